"""swb200: host side of the B200 time stepper for ShallowWaters.jl models.

The public names mirror the reference's API (src/ShallowWaters.jl:3):
``run_model`` and ``Parameter``; ``model_setup``/``initial_conditions`` expose
the set-up steps of src/run_model.jl:25-36 so that state can be prepared,
modified (seeded inputs) and handed to the device.
"""
from .parameter import Parameter
from .model_setup import Grid, Constants, Forcing, ModelSetup, model_setup
from .initial_conditions import (PrognosticVars, initial_conditions, add_halo, remove_halo,
                                 ghost_points, ghost_points_sst)
from .run_model import run_model, time_integration, NaNsDetected
from .model import Model
from . import abi

__all__ = ["Parameter", "Grid", "Constants", "Forcing", "ModelSetup", "model_setup",
           "PrognosticVars", "initial_conditions", "add_halo", "remove_halo",
           "ghost_points", "ghost_points_sst", "run_model", "time_integration",
           "NaNsDetected", "Model", "abi"]
