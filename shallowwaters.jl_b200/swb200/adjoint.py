"""Gradients of an eta misfit through the time loop (sw_adjoint_run).

    J(u0, v0, eta0, Fx) = sum over the interior of (eta after nsteps - eta_obs)^2

``gradient`` returns J and its gradients with respect to the initial state
(u, v, eta with halo) and the wind forcing Fx, computed on the GPU by the
library's hand-written adjoint of every pass of the RK step and of the tail
(drag and diffusion), with the step states kept at checkpoints in device
memory (binomial recomputation when there are fewer checkpoint slots than
steps).  It is the counterpart of a ChainRules ``rrule`` around the Julia
time loop: ``J`` is the primal value and the gradients are its pullback of 1.

``twin`` builds the identical-twin experiment the adjoint is measured on: a
periodic flat channel (RK4, Arakawa-Hsu, Smagorinsky, quadratic drag, no
tracer), the seeded eta noise of the other workloads as initial state, and
observations eta_obs taken from a run whose wind Fx_obs = Fx + dFx adds eight
seeded Fourier modes of 0.02 Pa peak, converted to the model's units by
Delta / (rho H) like the wind itself (src/forcing.jl:57-64).
"""
from __future__ import annotations

import copy
import ctypes as C
import dataclasses
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import abi


@dataclass
class AdjointResult:
    J: float
    u: np.ndarray          # dJ/du0, shape of u with halo
    v: np.ndarray
    eta: np.ndarray
    Fx: np.ndarray         # dJ/dFx, (nuy, nux)
    eta_final: np.ndarray  # eta after nsteps, with halo
    stats: abi.SwAdjointStats


def with_Fx(S, Fx):
    """A copy of ModelSetup S whose forcing has the wind field Fx."""
    F = copy.copy(S.forcing)
    F.Fx = np.ascontiguousarray(Fx, dtype=S.parameters.T)
    return dataclasses.replace(S, forcing=F)


def gradient(S, Prog, eta_obs, nsteps: Optional[int] = None, ncheckpoints: Optional[int] = None,
             lib=None) -> AdjointResult:
    """J and its gradients for ModelSetup S from the initial state Prog
    (PrognosticVars with halo).  eta_obs is (ny, nx).  nsteps defaults to
    S.grid.nt, ncheckpoints to nsteps (every state kept)."""
    lib = lib or abi.load_library()
    P, G = S.parameters, S.grid
    T = P.T
    n = int(G.nt if nsteps is None else nsteps)
    nc = int(n if ncheckpoints is None else ncheckpoints)
    cfg = abi.make_config(S, nt=n)
    static = abi.StaticFields(S)
    u, v, e = (np.ascontiguousarray(a, dtype=T) for a in list(Prog)[:3])
    obs = np.ascontiguousarray(eta_obs, dtype=T)
    if obs.shape != (G.ny, G.nx):
        raise ValueError(f"eta_obs must be (ny, nx) = {(G.ny, G.nx)}")
    gu, gv, ge = np.zeros_like(u), np.zeros_like(v), np.zeros_like(e)
    gF = np.zeros((G.nuy, G.nux), T)
    ef = np.zeros_like(e)
    J = C.c_double()
    stats = abi.SwAdjointStats()
    rc = lib.sw_adjoint_run(C.byref(cfg), static.ptr(), u.ctypes.data, v.ctypes.data, e.ctypes.data,
                            obs.ctypes.data, n, nc, C.byref(J), gu.ctypes.data, gv.ctypes.data, ge.ctypes.data,
                            gF.ctypes.data, ef.ctypes.data, C.byref(stats))
    abi.check(lib, rc)
    return AdjointResult(J.value, gu, gv, ge, gF, ef, stats)


def fourier_modes(S, seed: int, nmodes: int = 8, peak_pa: float = 0.02) -> np.ndarray:
    """dFx on the u-grid: nmodes seeded 2-D Fourier modes (wavenumbers 1-4 in
    x and y, random phases and amplitudes), scaled to peak_pa Pa at their
    maximum and converted by Delta / (rho H)."""
    P, G = S.parameters, S.grid
    rng = np.random.default_rng(seed)
    x = (np.arange(G.nux) + 0.5) / G.nux
    y = (np.arange(G.nuy) + 0.5) / G.nuy
    X, Y = np.meshgrid(x, y)
    f = np.zeros_like(X)
    for _ in range(nmodes):
        kx, ky = rng.integers(1, 5, size=2)
        a, ph = rng.uniform(0.5, 1.0), rng.uniform(0, 2 * np.pi, size=2)
        f += a * np.cos(2 * np.pi * kx * X + ph[0]) * np.cos(np.pi * ky * Y + ph[1])
    f *= peak_pa / np.max(np.abs(f))
    return (G.Δ / P.ρ / P.H) * f


def twin(nx: int = 512, nsteps: int = 2000, seed: int = 5, T=np.float64, **kw):
    """(S, Prog, eta_obs, dFx) of the identical-twin experiment, eta_obs from
    the library's forward run with Fx + dFx."""
    from . import Model, Parameter, initial_conditions, model_setup
    from .initial_conditions import remove_halo
    pkw = dict(nx=nx, L_ratio=2, bc="periodic", wind_forcing_x="channel", Fx0=0.12, topography="flat", H=500,
               g=10, cfl=1, time_scheme="RK", RKo=4, adv_scheme="ArakawaHsu", diffusion="Smagorinsky",
               bottom_drag="quadratic", tracer_advection=False, Ndays=1.0)
    pkw.update(kw)
    P = Parameter(T=T, **pkw)
    S = model_setup(P)
    rng = np.random.default_rng(seed)
    eta0 = rng.normal(0.0, 0.01, (S.grid.ny, S.grid.nx))
    Prog = initial_conditions(P.Tprog, S, η0=eta0)
    dFx = fourier_modes(S, seed + 1)
    S_obs = with_Fx(S, S.forcing.Fx + dFx)
    with Model(S_obs) as m:
        m.set_state(Prog)
        m.run(nsteps)
        eta_obs = remove_halo(*m.get_state(), S)[2]
    return S, Prog, np.ascontiguousarray(eta_obs, dtype=T), dFx
