"""NetCDF output and restart (src/output.jl, src/initial_conditions.jl:39-150).

The writer and the restart reader are host code: these tests need no GPU.
The GPU run with output=true is in test_gpu_parity.py.
"""
import os

import numpy as np
from scipy.io import netcdf_file

import oracle as O
from conftest import seeded_inputs
from swb200 import Parameter, initial_conditions, model_setup
from swb200.initial_conditions import PrognosticVars, remove_halo
from swb200.output import NcFiles, VARS, vorticities

ALL = ["u", "v", "η", "sst", "q", "ζ", "du", "dv", "dη"]


def _read(path, name):
    with netcdf_file(os.path.join(path, name + ".nc"), "r", mmap=False) as nc:
        return np.array(nc.variables[name][:]), np.array(nc.variables["t"][:]), \
            nc.variables[name].units.decode(), np.array(nc.variables["x"][:])


def test_frames_run_folders_and_increments(tmp_path):
    P = Parameter(nx=20, output=True, outpath=str(tmp_path), output_vars=ALL)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 3))
    later = PrognosticVars(*(a + np.asarray(0.125, a.dtype) for a in Prog))
    nc = NcFiles(S)
    nc.write(0, Prog, Prog)
    nc.write(S.grid.nout, later, Prog)
    nc.close()
    assert os.path.basename(nc.runpath) == "run0000"
    un, vn, en, sn = remove_halo(*later, S)
    uo = remove_halo(*Prog, S)[0]
    u, t, unit, x = _read(nc.runpath, "u")
    assert u.shape == (2,) + un.shape and unit == "m/s"
    np.testing.assert_array_equal(u[1], un.astype(np.float32))
    np.testing.assert_array_equal(t, [0, S.grid.nout * S.grid.dtint])
    np.testing.assert_array_equal(x, S.grid.x_u)
    du = _read(nc.runpath, "du")[0]
    np.testing.assert_array_equal(du[1], un.astype(np.float32) - uo.astype(np.float32))
    np.testing.assert_array_equal(du[0], 0)
    for key in ALL:
        assert os.path.exists(os.path.join(nc.runpath, VARS[key][0] + ".nc"))
    # get_id_mode "continue": the next run takes the next folder
    nc2 = NcFiles(S)
    nc2.close()
    assert os.path.basename(nc2.runpath) == "run0001"


def test_vorticity_matches_oracle_pv():
    """q written for the initial state equals PV! of the oracle's prologue."""
    P = Parameter(nx=24, bc="nonperiodic", topography="seamount")
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 4))
    o = O.Oracle(S)
    o.set_state(Prog)
    q_ref = o.field("q")
    q, _ = vorticities(Prog.u, Prog.v, Prog.η, S)
    np.testing.assert_array_equal(q, q_ref[:q.shape[0], :q.shape[1]].astype(np.float32))


def test_restart_reads_last_frame(tmp_path):
    P = Parameter(nx=20, output=True, outpath=str(tmp_path))
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 5))
    nc = NcFiles(S)
    nc.write(0, Prog, Prog)
    nc.close()
    R = model_setup(Parameter(nx=20, initial_cond="ncfile", initpath=str(tmp_path), init_run_id=0))
    Prog2 = initial_conditions(R.parameters.Tprog, R)
    for a, b in zip(remove_halo(*Prog2, R)[:3], remove_halo(*Prog, S)[:3]):
        np.testing.assert_array_equal(a, b)


def test_restart_interpolates_to_another_grid(tmp_path):
    """Gridded linear interpolation with flat extrapolation reproduces a field
    linear in x exactly (src/initial_conditions.jl:71-116)."""
    P = Parameter(nx=20, output=True, outpath=str(tmp_path))
    S = model_setup(P)
    G = S.grid
    η = np.tile(np.arange(G.nx, dtype=float) + 0.5, (G.ny, 1))
    Prog = initial_conditions(P.Tprog, S, η0=η)
    nc = NcFiles(S)
    nc.write(0, Prog, Prog)
    nc.close()
    R = model_setup(Parameter(nx=10, initial_cond="ncfile", initpath=str(tmp_path), init_run_id=0))
    eta = remove_halo(*initial_conditions(R.parameters.Tprog, R), R)[2]
    expect = np.tile(np.arange(10) * 2.0 + 1.0, (R.grid.ny, 1))
    np.testing.assert_allclose(eta, expect, rtol=1e-6)
