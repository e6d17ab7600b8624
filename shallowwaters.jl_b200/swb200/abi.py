"""ctypes mirror of include/swb200.h and the loader of libswb200.so.

``make_config(S)`` fills ``sw_config`` from a ModelSetup the way a Julia
``ccall`` wrapper fills it from ``S.grid``/``S.constants``: every constant is
the reference's value already rounded to T or Tprog.  ``make_static(S)`` packs
the static fields (f_q, Fx, Fy, H, ...) as contiguous T arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .model_setup import ModelSetup

ABI_VERSION = 1

FMT = {np.float16: 1, np.float32: 2, np.float64: 3}
FMT_DTYPE = {1: np.float16, 2: np.float32, 3: np.float64}
SCHEME = {"RK": 0, "SSPRK2": 1, "SSPRK3": 2, "4SSPRK3": 3}
DYNAMICS = {"nonlinear": 0, "linear": 1}
ADV = {"ArakawaHsu": 0, "Sadourny": 1}
DRAG = {"quadratic": 0, "linear": 1, "none": 2}
DIFF = {"constant": 0, "Smagorinsky": 1}
STORAGE = {"native": 0, "bf16": 1, "f16": 2}

SW_OK, SW_ERR_ARG, SW_ERR_CUDA, SW_NAN_DETECTED, SW_ERR_TIMEOUT = 0, 1, 2, 3, 4
SW_ERR_UNSUPPORTED, SW_ERR_NOMEM, SW_ERR_DEPARTURE, SW_ERR_NODEVICE = 5, 6, 7, 8


class SwConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("periodic", C.c_int32),
        ("halo", C.c_int32), ("haloeta", C.c_int32),
        ("halosstx", C.c_int32), ("halossty", C.c_int32),
        ("T", C.c_int32), ("Tprog", C.c_int32), ("Tcomm", C.c_int32),
        ("time_scheme", C.c_int32),
        ("RKo", C.c_int32), ("RKs", C.c_int32), ("RKn", C.c_int32),
        ("nstep_diff", C.c_int32), ("nstep_advcor", C.c_int32),
        ("nadvstep", C.c_int32), ("nadvstep_half", C.c_int32),
        ("nout", C.c_int32),
        ("dtint", C.c_int32),
        ("nt", C.c_int64),
        ("dynamics", C.c_int32), ("adv_scheme", C.c_int32),
        ("bottom_drag", C.c_int32), ("diffusion", C.c_int32),
        ("tracer_advection", C.c_int32), ("tracer_consumption", C.c_int32),
        ("surface_relax", C.c_int32), ("surface_forcing", C.c_int32),
        ("seasonal_wind_x", C.c_int32), ("seasonal_wind_y", C.c_int32),
        ("RKaDt", C.c_double * 4), ("RKbDt", C.c_double * 3),
        ("Dt_Ds", C.c_double), ("Dt_D", C.c_double), ("Dt_D_half", C.c_double),
        ("one_minus_alpha", C.c_double),
        ("Dt_diff", C.c_double),
        ("ssp_n", C.c_int32), ("ssp_s", C.c_int32), ("ssp_kn", C.c_int32), ("ssp_mn", C.c_int32),
        ("ssp_Dt_Dn", C.c_double), ("ssp_kna", C.c_double), ("ssp_knb", C.c_double),
        ("ssp_Dt_Dnc", C.c_double),
        ("g", C.c_double), ("cD", C.c_double), ("rD", C.c_double), ("gamma", C.c_double),
        ("cSmag", C.c_double), ("nuB", C.c_double), ("rSST", C.c_double), ("jSST", C.c_double),
        ("SSTmin", C.c_double),
        ("dtadvu", C.c_double), ("dtadvv", C.c_double),
        ("half_dtadvu", C.c_double), ("half_dtadvv", C.c_double),
        ("omegaFeta", C.c_double), ("omegaFx", C.c_double), ("omegaFy", C.c_double),
        ("storage", C.c_int32),
        ("storage_scale_uv", C.c_double),
        ("reserved", C.c_int32 * 8),
    ]


class SwStatic(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("f_q", "f_u", "f_v", "Fx", "Fy", "H", "eta_ref", "Feta")]


class SwStatus(C.Structure):
    _fields_ = [("steps_done", C.c_int64), ("step", C.c_int64), ("nan_step", C.c_int64),
                ("code", C.c_int32), ("reserved", C.c_int32)]


class SwAdjointStats(C.Structure):
    _fields_ = [("forward_ms", C.c_double), ("reverse_ms", C.c_double), ("forward_steps", C.c_int64),
                ("adjoint_steps", C.c_int64), ("checkpoints", C.c_int32), ("launches_per_forward_step", C.c_int32),
                ("launches_per_adjoint_step", C.c_int32), ("stored_stage_states", C.c_int32)]


class SwDiag(C.Structure):
    _fields_ = [("mass", C.c_double), ("energy", C.c_double), ("max_speed", C.c_double),
                ("nan_count", C.c_int64)]


PROFILE_KINDS = 6
PROFILE_NAMES = ("rk_stage", "tail", "tracer", "advcor", "nan_check", "other")


class SwProfile(C.Structure):
    _fields_ = [("step_ms_total", C.c_double),
                ("kernel_ms", C.c_double * PROFILE_KINDS),
                ("launches", C.c_int64 * PROFILE_KINDS),
                ("steps", C.c_int64)]


def make_config(S: ModelSetup, *, nt=None, storage="native", storage_scale_uv=1024.0) -> SwConfig:
    P, G, K = S.parameters, S.grid, S.constants
    c = SwConfig()
    c.abi_version = ABI_VERSION
    c.nx, c.ny = G.nx, G.ny
    c.periodic = 1 if P.bc == "periodic" else 0
    c.halo, c.haloeta, c.halosstx, c.halossty = G.halo, G.haloη, G.halosstx, G.halossty
    c.T, c.Tprog, c.Tcomm = FMT[P.T], FMT[P.Tprog], FMT[P.Tcomm]
    c.time_scheme = SCHEME[P.time_scheme]
    c.RKo, c.RKs, c.RKn = P.RKo, P.RKs, P.RKn
    c.nstep_diff, c.nstep_advcor = P.nstep_diff, P.nstep_advcor
    c.nadvstep, c.nadvstep_half = G.nadvstep, G.nadvstep_half
    c.nout = G.nout
    c.dtint = G.dtint
    c.nt = G.nt if nt is None else int(nt)
    c.dynamics, c.adv_scheme = DYNAMICS[P.dynamics], ADV[P.adv_scheme]
    c.bottom_drag, c.diffusion = DRAG[P.bottom_drag], DIFF[P.diffusion]
    c.tracer_advection = int(bool(P.tracer_advection))
    c.tracer_consumption = int(bool(P.tracer_consumption))
    c.surface_relax, c.surface_forcing = int(bool(P.surface_relax)), int(bool(P.surface_forcing))
    c.seasonal_wind_x, c.seasonal_wind_y = int(bool(P.seasonal_wind_x)), int(bool(P.seasonal_wind_y))
    for k in range(4):
        c.RKaDt[k] = float(K.RKaΔt[k]) if k < len(K.RKaΔt) else 0.0
    for k in range(3):
        c.RKbDt[k] = float(K.RKbΔt[k]) if k < len(K.RKbΔt) else 0.0
    c.Dt_Ds, c.Dt_D, c.Dt_D_half = float(K.Δt_Δs), float(K.Δt_Δ), float(K.Δt_Δ_half)
    c.one_minus_alpha = float(K.one_minus_α)
    c.Dt_diff = float(G.Δt_diff)
    s3 = K.SSPRK3c
    c.ssp_n, c.ssp_s, c.ssp_kn, c.ssp_mn = s3["n"], s3["s"], s3["kn"], s3["mn"]
    c.ssp_Dt_Dn, c.ssp_kna = float(s3["Δt_Δn"]), float(s3["kna"])
    c.ssp_knb, c.ssp_Dt_Dnc = float(s3["knb"]), float(s3["Δt_Δnc"])
    c.g, c.cD, c.rD, c.gamma = float(K.g), float(K.cD), float(K.rD), float(K.γ)
    c.cSmag, c.nuB, c.rSST, c.jSST = float(K.cSmag), float(K.νB), float(K.rSST), float(K.jSST)
    c.SSTmin = float(K.SSTmin)
    c.dtadvu, c.dtadvv = float(G.dtadvu), float(G.dtadvv)
    c.half_dtadvu, c.half_dtadvv = float(G.half_dtadvu), float(G.half_dtadvv)
    c.omegaFeta, c.omegaFx, c.omegaFy = K.ωFη, K.ωFx, K.ωFy
    c.storage = STORAGE[storage]
    c.storage_scale_uv = float(storage_scale_uv)
    return c


class StaticFields:
    """Keeps the contiguous T arrays alive while the library reads them."""

    def __init__(self, S: ModelSetup):
        T = S.parameters.T
        G, F = S.grid, S.forcing
        self.arrays = {
            "f_q": np.ascontiguousarray(G.f_q, dtype=T),
            "f_u": np.ascontiguousarray(G.f_u, dtype=T),
            "f_v": np.ascontiguousarray(G.f_v, dtype=T),
            "Fx": np.ascontiguousarray(F.Fx, dtype=T),
            "Fy": np.ascontiguousarray(F.Fy, dtype=T),
            "H": np.ascontiguousarray(F.H, dtype=T),
            "eta_ref": np.ascontiguousarray(F.η_ref, dtype=T),
            "Feta": np.ascontiguousarray(F.Fη, dtype=T),
        }
        self.struct = SwStatic(**{k: a.ctypes.data for k, a in self.arrays.items()})

    def ptr(self):
        return C.byref(self.struct)


def state_ptrs(u, v, η, sst):
    for a in (u, v, η, sst):
        if not (isinstance(a, np.ndarray) and a.flags.c_contiguous):
            raise ValueError("state arrays must be C-contiguous numpy arrays ([j][i] storage)")
    return tuple(C.c_void_p(a.ctypes.data) for a in (u, v, η, sst))


# --------------------------------------------------------------------------

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("SWB200_LIB", os.path.join(_PKG_DIR, "libswb200.so"))
# the two builds of the same sources: "parity" (no FMA contraction, bit-exact
# with the reference's arithmetic) and "fast" (FMA contraction, equal to
# rounding); see include/swb200.h sw_build_kind
BUILDS = {"parity": LIB_PATH, "fast": os.path.join(_PKG_DIR, "libswb200_fast.so")}
SW_BUILD_PARITY, SW_BUILD_FAST = 0, 1
_libs = {}

EXPORTS = {
    "sw_time_integration": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "sw_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_run": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p]),
    "sw_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_get_rhs_input": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_diagnostics": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sw_run_profiled": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]),
    "sw_run_timed": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.POINTER(C.c_double), C.c_void_p]),
    "sw_diagnostics_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_trim_memory": (C.c_int, []),
    "sw_batch_create": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "sw_batch_set_state": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_batch_run": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p]),
    "sw_batch_get_state": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_batch_launches": (C.c_int64, [C.c_void_p]),
    "sw_batch_tile_rows": (C.c_int32, [C.c_void_p]),
    "sw_batch_member": (C.c_void_p, [C.c_void_p, C.c_int32]),
    "sw_batch_destroy": (None, [C.c_void_p]),
    "sw_adjoint_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_int64, C.c_int32, C.POINTER(C.c_double), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sw_kernel_launches": (C.c_int64, [C.c_void_p]),
    "sw_destroy": (None, [C.c_void_p]),
    "sw_strerror": (C.c_char_p, [C.c_int]),
    "sw_last_error": (C.c_char_p, [C.c_void_p]),
    "sw_abi_version": (C.c_int, []),
    "sw_build_kind": (C.c_int, []),
}


def load_library(path: str | None = None, build: str = "parity"):
    """Load libswb200.so (build="parity") or libswb200_fast.so (build="fast");
    raises if it is missing (there is no CPU fallback)."""
    if path is None and build in _libs:
        return _libs[build]
    if build not in BUILDS:
        raise ValueError(f"build must be one of {sorted(BUILDS)}")
    p = path or BUILDS[build]
    if not os.path.exists(p):
        raise RuntimeError(f"{os.path.basename(p)} not found at {p}; build it with "
                           f"`python __graft_entry__.py` or `make -C shallowwaters.jl_b200/csrc`")
    lib = C.CDLL(p)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.sw_abi_version() != ABI_VERSION:
        raise RuntimeError(f"libswb200 ABI {lib.sw_abi_version()} != {ABI_VERSION}")
    if path is None:
        want = SW_BUILD_FAST if build == "fast" else SW_BUILD_PARITY
        if lib.sw_build_kind() != want:
            raise RuntimeError(f"{p} is not the {build} build")
        _libs[build] = lib
    return lib


class SwError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"swb200 error {code}: {msg}")
        self.code = code


def check(lib, code, ctx=None):
    if code != SW_OK:
        msg = lib.sw_last_error(ctx) if ctx else lib.sw_strerror(code)
        raise SwError(code, (msg or b"").decode(errors="replace"))
