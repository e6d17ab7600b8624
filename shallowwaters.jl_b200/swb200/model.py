"""Model: a device-resident run, the context half of the C ABI.

``Model(S)`` wraps ``sw_create``; ``set_state``/``run``/``get_state`` move a
state with halo (PrognosticVars) to and from the GPU and advance it, so many
steps can run without host round trips.  It is the stepping counterpart of
``time_integration`` (src/time_integration.jl:2-250).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .initial_conditions import PrognosticVars
from .model_setup import ModelSetup


class Model:
    def __init__(self, S: ModelSetup, *, storage="native", storage_scale_uv=1024.0, build="parity", lib=None):
        """build: "parity" (libswb200.so, bit-exact with the reference's
        arithmetic) or "fast" (libswb200_fast.so, FMA contraction)."""
        self.lib = lib or abi.load_library(build=build)
        self.S = S
        self.cfg = abi.make_config(S, storage=storage, storage_scale_uv=storage_scale_uv)
        self.static = abi.StaticFields(S)
        self.ctx = C.c_void_p()
        rc = self.lib.sw_create(C.byref(self.cfg), self.static.ptr(), C.byref(self.ctx))
        abi.check(self.lib, rc)
        self.Tp = S.parameters.Tprog

    def close(self):
        if getattr(self, "ctx", None) and self.ctx.value:
            self.lib.sw_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, Prog: PrognosticVars):
        arrs = [np.ascontiguousarray(a, dtype=self.Tp) for a in Prog]
        self._keep = arrs
        rc = self.lib.sw_set_state(self.ctx, *abi.state_ptrs(*arrs))
        abi.check(self.lib, rc, self.ctx)

    def get_state(self) -> PrognosticVars:
        G, Tp = self.S.grid, self.Tp
        u = np.zeros((G.nuy + 4, G.nux + 4), Tp)
        v = np.zeros((G.nvy + 4, G.nvx + 4), Tp)
        e = np.zeros((G.ny + 2, G.nx + 2), Tp)
        s = np.zeros((G.ny, G.nx + 2), Tp)
        rc = self.lib.sw_get_state(self.ctx, *abi.state_ptrs(u, v, e, s))
        abi.check(self.lib, rc, self.ctx)
        return PrognosticVars(u, v, e, s)

    def get_rhs_input(self):
        """u, v, η (with halo) that the last right-hand-side evaluation of the
        last step read (the input of its last RK stage or SSP sub-stage): the
        state the reference's vorticity work arrays describe after a step."""
        G, Tp = self.S.grid, self.Tp
        u = np.zeros((G.nuy + 4, G.nux + 4), Tp)
        v = np.zeros((G.nvy + 4, G.nvx + 4), Tp)
        e = np.zeros((G.ny + 2, G.nx + 2), Tp)
        rc = self.lib.sw_get_rhs_input(self.ctx, *abi.state_ptrs(u, v, e, e)[:3])
        abi.check(self.lib, rc, self.ctx)
        return u, v, e

    def run(self, nsteps: int) -> abi.SwStatus:
        st = abi.SwStatus()
        rc = self.lib.sw_run(self.ctx, int(nsteps), C.byref(st))
        if rc not in (abi.SW_OK, abi.SW_NAN_DETECTED):
            abi.check(self.lib, rc, self.ctx)
        return st

    def run_profiled(self, nsteps: int, l2_flush_bytes: int = 0):
        prof, st = abi.SwProfile(), abi.SwStatus()
        rc = self.lib.sw_run_profiled(self.ctx, int(nsteps), int(l2_flush_bytes), C.byref(prof), C.byref(st))
        if rc not in (abi.SW_OK, abi.SW_NAN_DETECTED):
            abi.check(self.lib, rc, self.ctx)
        return prof, st

    def run_timed(self, nsteps: int, l2_flush_bytes: int = 0):
        """Run nsteps steps as sw_run does; returns (sum of per-step device ms, status)."""
        ms, st = C.c_double(0.0), abi.SwStatus()
        rc = self.lib.sw_run_timed(self.ctx, int(nsteps), int(l2_flush_bytes), C.byref(ms), C.byref(st))
        if rc not in (abi.SW_OK, abi.SW_NAN_DETECTED):
            abi.check(self.lib, rc, self.ctx)
        return ms.value, st

    def diagnostics(self) -> abi.SwDiag:
        d = abi.SwDiag()
        abi.check(self.lib, self.lib.sw_diagnostics(self.ctx, C.byref(d)), self.ctx)
        return d

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.sw_kernel_launches(self.ctx))
