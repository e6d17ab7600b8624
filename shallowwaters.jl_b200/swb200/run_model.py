"""run_model: the reference's user-facing entry point, executed on the B200.

``run_model(T=np.float32, **kwargs)``, ``run_model(P)`` and
``run_model(T, P)`` mirror src/run_model.jl:12-39: build Parameter, Grid,
Constants, Forcing and the initial conditions on the host, then hand the time
loop (src/time_integration.jl:2-250) to libswb200.so, which runs it as CUDA
kernels.  The returned PrognosticVars holds u, v, η, sst without halo, in
Tprog, like the reference.  There is no CPU fallback: without the library or a
GPU the call raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .initial_conditions import PrognosticVars, initial_conditions, remove_halo
from .model_setup import ModelSetup, model_setup
from .parameter import Parameter


class NaNsDetected(RuntimeError):
    """The run stopped because NaNs appeared (feedback.nans_detected)."""


def time_integration(Prog: PrognosticVars, S: ModelSetup, *, nt=None, storage="native",
                     storage_scale_uv=1024.0, build="parity", lib=None):
    """Drop-in for time_integration(Prog, Diag, S) (src/time_integration.jl:2-250).

    Runs on the GPU through ``sw_time_integration``.  Returns
    ``(PrognosticVars without halo, sw_status)``.  On NaN detection the state
    is the one the reference returns (u, v, η before the failing step) and
    ``status.code == SW_NAN_DETECTED``.
    """
    lib = lib or abi.load_library(build=build)
    cfg = abi.make_config(S, nt=nt, storage=storage, storage_scale_uv=storage_scale_uv)
    st = abi.StaticFields(S)
    Tp = S.parameters.Tprog
    u, v, η, sst = (np.ascontiguousarray(a, dtype=Tp).copy() for a in Prog)
    status = abi.SwStatus()
    rc = lib.sw_time_integration(C.byref(cfg), st.ptr(), *abi.state_ptrs(u, v, η, sst), C.byref(status))
    if rc not in (abi.SW_OK, abi.SW_NAN_DETECTED):
        abi.check(lib, rc)
    return PrognosticVars(*remove_halo(u, v, η, sst, S)), status


def run_model(T=np.float32, P: Parameter | None = None, **kwargs) -> PrognosticVars:
    """src/run_model.jl:12-39.

    ``run_model(np.float32, Ndays=10, nx=200)`` or ``run_model(P)`` or
    ``run_model(T, P)``.  Seeded initial fields may be given as ``u0, v0, η0,
    sst0`` (interiors, [j][i] storage); ``storage="bf16"/"f16"`` selects the
    16-bit device storage form.
    """
    if isinstance(T, Parameter):
        P, T = T, T.T
    init = {k: kwargs.pop(k) for k in ("u0", "v0", "η0", "sst0") if k in kwargs}
    storage = kwargs.pop("storage", "native")
    scale = kwargs.pop("storage_scale_uv", 1024.0)
    if P is None:
        P = Parameter(T=T, **kwargs)
    elif kwargs:
        P = P.replace(**kwargs)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **init)
    if P.output:
        out, status = _time_integration_with_output(Prog, S, storage=storage, storage_scale_uv=scale)
    else:
        out, status = time_integration(Prog, S, storage=storage, storage_scale_uv=scale)
    if status.code == abi.SW_NAN_DETECTED:
        print(f" NaNs detected at time step {status.nan_step}")
    return out


def _time_integration_with_output(Prog: PrognosticVars, S: ModelSetup, *, storage="native",
                                  storage_scale_uv=1024.0):
    """The time loop with output_nc! every nout steps (src/time_integration.jl:41,233):
    the state stays on the GPU and is read back only for the frames."""
    from .model import Model
    from .output import NcFiles
    G = S.grid
    nc = NcFiles(S)
    m = Model(S, storage=storage, storage_scale_uv=storage_scale_uv)
    try:
        m.set_state(Prog)
        state = m.get_state()
        # q and relvort: the reference computes them from the initial state before
        # its loop (src/time_integration.jl:27-29), then in every right-hand
        # side of nonlinear dynamics; linear dynamics never recomputes them
        # (the 16-bit storage form keeps its stage values in 16 bits: its frames
        # take them from the new state)
        initial = (np.asarray(Prog.u), np.asarray(Prog.v), np.asarray(Prog.η))

        def rhs_state():
            if S.parameters.dynamics != "nonlinear":
                return initial
            return m.get_rhs_input() if storage == "native" else None

        nc.write(0, state, state, initial)              # output_nc!(0, ...) of the initial state
        i = 0
        status = abi.SwStatus()
        while i < G.nt:
            n = min(G.nout - i % G.nout, G.nt - i)
            if (i + n) % G.nout == 0:
                # the frame needs the state one step before it for du, dv, dη
                if n > 1:
                    status = m.run(n - 1)
                    if status.code != abi.SW_OK:
                        break
                before = m.get_state()
                status = m.run(1)
                if status.code != abi.SW_OK:
                    break
                i += n
                nc.write(i, m.get_state(), before, rhs_state())
            else:
                status = m.run(n)
                if status.code != abi.SW_OK:
                    break
                i += n
        u, v, η, sst = m.get_state()
    finally:
        nc.close()
        m.close()
    return PrognosticVars(*remove_halo(u, v, η, sst, S)), status
