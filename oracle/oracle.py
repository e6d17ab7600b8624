"""ctypes driver of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py, never by the shipped package.  It feeds the
oracle exactly the config/static/state buffers the GPU library receives.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "shallowwaters.jl_b200"))

from swb200 import abi  # noqa: E402
from swb200.initial_conditions import PrognosticVars, initial_conditions, remove_halo  # noqa: E402
from swb200.model_setup import model_setup  # noqa: E402
from swb200.parameter import Parameter  # noqa: E402

LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_create.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
        L.oracle_set_state.argtypes = [C.c_void_p] * 5
        L.oracle_get_state.argtypes = [C.c_void_p] * 5
        L.oracle_run.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.oracle_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int)]
        L.oracle_last_error.argtypes = [C.c_void_p]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_set_threads.restype = C.c_int
        L.oracle_jvp.argtypes = [C.c_void_p, C.c_void_p] + [C.c_void_p] * 8 + [C.c_int64, C.POINTER(C.c_double),
                                                                                 C.POINTER(C.c_double)]
        L.oracle_jvp.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    """OpenMP threads for the oracle's loops; returns the count in effect."""
    return int(lib().oracle_set_threads(int(n)))


class Oracle:
    """One restated model instance: ``set_state``, ``run``, ``get_state``."""

    def __init__(self, S, nt=None):
        self.S = S
        self.cfg = abi.make_config(S, nt=nt)
        self.static = abi.StaticFields(S)
        self.h = C.c_void_p()
        rc = lib().oracle_create(C.byref(self.cfg), self.static.ptr(), C.byref(self.h))
        if rc:
            raise RuntimeError(f"oracle_create failed ({rc}): {lib().oracle_last_error(None).decode()}")
        self.Tp = S.parameters.Tprog

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            lib().oracle_destroy(self.h)
            self.h = C.c_void_p()

    def set_state(self, Prog):
        arrs = [np.ascontiguousarray(a, dtype=self.Tp) for a in Prog]
        rc = lib().oracle_set_state(self.h, *[a.ctypes.data for a in arrs])
        if rc:
            raise RuntimeError(lib().oracle_last_error(self.h).decode())

    def get_state(self) -> PrognosticVars:
        G = self.S.grid
        Tp = self.Tp
        u = np.zeros((G.nuy + 4, G.nux + 4), Tp)
        v = np.zeros((G.nvy + 4, G.nvx + 4), Tp)
        e = np.zeros((G.ny + 2, G.nx + 2), Tp)
        s = np.zeros((G.ny, G.nx + 2), Tp)
        lib().oracle_get_state(self.h, u.ctypes.data, v.ctypes.data, e.ctypes.data, s.ctypes.data)
        return PrognosticVars(u, v, e, s)

    def run(self, nsteps):
        st = abi.SwStatus()
        lib().oracle_run(self.h, int(nsteps), C.byref(st))
        return st

    def field(self, name):
        m, n, es = C.c_int64(), C.c_int64(), C.c_int()
        if not lib().oracle_field(self.h, name.encode(), None, C.byref(m), C.byref(n), C.byref(es)):
            raise KeyError(name)
        dt = {2: np.float16, 4: np.float32, 8: np.float64}[es.value]
        out = np.zeros((n.value, m.value), dt)
        lib().oracle_field(self.h, name.encode(), out.ctypes.data, C.byref(m), C.byref(n), C.byref(es))
        return out


def run_model(T=np.float32, P=None, *, nsteps=None, **kwargs):
    """run_model through the oracle; returns (PrognosticVars without halo, status)."""
    init = {k: kwargs.pop(k) for k in ("u0", "v0", "η0", "sst0") if k in kwargs}
    if P is None:
        P = Parameter(T=T, **kwargs)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **init)
    o = Oracle(S)
    o.set_state(Prog)
    st = o.run(S.grid.nt if nsteps is None else nsteps)
    return PrognosticVars(*remove_halo(*o.get_state(), S)), st


def jvp(S, Prog, eta_obs, nsteps, du=None, dv=None, deta=None, dFx=None):
    """(J, dJ) with J = sum over the interior of (eta after nsteps - eta_obs)^2
    and dJ its directional derivative along (du, dv, deta, dFx) (state shapes
    with halo, dFx (nuy, nux); None is zero), from the restated loop run with
    forward-mode dual numbers.  Float64 setups only."""
    cfg = abi.make_config(S, nt=nsteps)
    st = abi.StaticFields(S)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in list(Prog)[:3]]
    dirs = [None if d is None else np.ascontiguousarray(d, dtype=np.float64) for d in (du, dv, deta, dFx)]
    obs = np.ascontiguousarray(eta_obs, dtype=np.float64)
    J, dJ = C.c_double(), C.c_double()
    ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    rc = lib().oracle_jvp(C.byref(cfg), st.ptr(), *[a.ctypes.data for a in arrs], *[ptr(d) for d in dirs],
                          obs.ctypes.data, int(nsteps), C.byref(J), C.byref(dJ))
    if rc:
        raise RuntimeError(f"oracle_jvp failed ({rc}): {lib().oracle_last_error(None).decode()}")
    return J.value, dJ.value


def cost(S, Prog, eta_obs, nsteps):
    """J = sum over the interior of (eta after nsteps - eta_obs)^2 from the
    restated loop in S's number type (summed in float64)."""
    o = Oracle(S)
    o.set_state(Prog)
    o.run(nsteps)
    e = remove_halo(*o.get_state(), S)[2].astype(np.float64)
    return float(np.sum((e - np.asarray(eta_obs, np.float64)) ** 2))
