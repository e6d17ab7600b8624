"""Prognostic variables, initial conditions and halos (host side).

Restates src/initial_conditions.jl:1-164 and the halo helpers of
src/ghost_points.jl:1-241 for the one-off set-up on the host.  All 2-D arrays
are stored ``[j][i]`` (x fastest), which is the memory order of Julia's
column-major ``Array{T,2}`` with element ``(i,j)``.

Seeded inputs (noise on eta, a checkerboard tracer, ...) are injected by
overwriting interiors *before* the halo is added, so the halo always satisfies
the boundary conditions, as after ``add_halo`` in the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .model_setup import PI, ModelSetup, _meshgrid_x, _meshgrid_y


@dataclass
class PrognosticVars:
    """src/initial_conditions.jl:6-11: u, v, η, sst."""
    u: np.ndarray
    v: np.ndarray
    η: np.ndarray
    sst: np.ndarray

    def __iter__(self):
        return iter((self.u, self.v, self.η, self.sst))


# --------------------------------------------------------------------------
# ghost points on the host (src/ghost_points.jl:46-241), used by add_halo

def _tcomm(x, T, Tcomm):
    """T(Tcomm(x)) (src/ghost_points.jl:65-68)."""
    return T(Tcomm(x)) if Tcomm is not T else x


def ghost_points_u_nonperiodic(u, one_minus_α):
    """src/ghost_points.jl:47-57 (Julia u[i,1] is u[0,i] here)."""
    u[0, :] = one_minus_α * u[3, :]
    u[1, :] = one_minus_α * u[2, :]
    u[-2, :] = one_minus_α * u[-3, :]
    u[-1, :] = one_minus_α * u[-4, :]


def ghost_points_u_periodic(Tcomm, u):
    """src/ghost_points.jl:60-73."""
    T = u.dtype.type
    u[:, 0] = _tcomm(u[:, -4], T, Tcomm)
    u[:, 1] = _tcomm(u[:, -3], T, Tcomm)
    u[:, -2] = _tcomm(u[:, 2], T, Tcomm)
    u[:, -1] = _tcomm(u[:, 3], T, Tcomm)


def ghost_points_v_nonperiodic(v, one_minus_α):
    """src/ghost_points.jl:76-86."""
    v[:, 0] = one_minus_α * v[:, 3]
    v[:, 1] = one_minus_α * v[:, 2]
    v[:, -2] = one_minus_α * v[:, -3]
    v[:, -1] = one_minus_α * v[:, -4]


def ghost_points_v_periodic(Tcomm, v):
    """src/ghost_points.jl:89-99."""
    T = v.dtype.type
    v[:, 0] = _tcomm(v[:, -4], T, Tcomm)
    v[:, 1] = _tcomm(v[:, -3], T, Tcomm)
    v[:, -2] = _tcomm(v[:, 2], T, Tcomm)
    v[:, -1] = _tcomm(v[:, 3], T, Tcomm)


def ghost_points_η_nonperiodic(η):
    """src/ghost_points.jl:102-116."""
    η[:, 0] = η[:, 1]
    η[:, -1] = η[:, -2]
    η[0, :] = η[1, :]
    η[-1, :] = η[-2, :]


def ghost_points_η_periodic(Tcomm, η):
    """src/ghost_points.jl:119-133."""
    T = η.dtype.type
    η[:, 0] = _tcomm(η[:, -2], T, Tcomm)
    η[:, -1] = _tcomm(η[:, 1], T, Tcomm)
    η[0, :] = η[1, :]
    η[-1, :] = η[-2, :]


def ghost_points_sst_nonperiodic(sst, halosstx, halossty):
    """src/ghost_points.jl:136-156."""
    for i in range(halosstx):
        sst[:, i] = sst[:, halosstx]
        sst[:, -1 - i] = sst[:, -1 - halosstx]
    for j in range(halossty):
        sst[j, :] = sst[halossty, :]
        sst[-1 - j, :] = sst[-1 - halossty, :]


def ghost_points_sst_periodic(Tcomm, sst, halosstx, halossty):
    """src/ghost_points.jl:159-179."""
    T = sst.dtype.type
    m = sst.shape[1]
    for i in range(1, halosstx + 1):
        sst[:, i - 1] = _tcomm(sst[:, m - 2 * halosstx + i - 1], T, Tcomm)
        sst[:, m - halosstx + i - 1] = _tcomm(sst[:, halosstx + i - 1], T, Tcomm)
    for j in range(halossty):
        sst[j, :] = sst[halossty, :]
        sst[-1 - j, :] = sst[-1 - halossty, :]


def ghost_points(u, v, η, S: ModelSetup):
    """src/ghost_points.jl:182-199."""
    P, C = S.parameters, S.constants
    if P.bc == "periodic":
        ghost_points_u_periodic(P.Tcomm, u)
        ghost_points_v_periodic(P.Tcomm, v)
        ghost_points_η_periodic(P.Tcomm, η)
    else:
        ghost_points_u_nonperiodic(u, C.one_minus_α)
        ghost_points_v_nonperiodic(v, C.one_minus_α)
        ghost_points_η_nonperiodic(η)


def ghost_points_sst(sst, S: ModelSetup):
    """src/ghost_points.jl:232-241."""
    G = S.grid
    if S.parameters.bc == "periodic":
        ghost_points_sst_periodic(S.parameters.Tcomm, sst, G.halosstx, G.halossty)
    else:
        ghost_points_sst_nonperiodic(sst, G.halosstx, G.halossty)


def add_halo(u, v, η, sst, S: ModelSetup):
    """src/ghost_points.jl:2-27: zero halo, then the boundary conditions."""
    G = S.grid
    T = u.dtype.type
    h, he, hx, hy = G.halo, G.haloη, G.halosstx, G.halossty
    U = np.zeros((G.nuy + 2 * h, G.nux + 2 * h), dtype=T)
    U[h:h + G.nuy, h:h + G.nux] = u
    V = np.zeros((G.nvy + 2 * h, G.nvx + 2 * h), dtype=T)
    V[h:h + G.nvy, h:h + G.nvx] = v
    E = np.zeros((G.ny + 2 * he, G.nx + 2 * he), dtype=T)
    E[he:he + G.ny, he:he + G.nx] = η
    SST = np.zeros((G.ny + 2 * hy, G.nx + 2 * hx), dtype=T)
    SST[hy:hy + G.ny, hx:hx + G.nx] = sst
    ghost_points(U, V, E, S)
    ghost_points_sst(SST, S)
    return U, V, E, SST


def remove_halo(u, v, η, sst, S: ModelSetup):
    """src/ghost_points.jl:30-44."""
    G = S.grid
    h, he, hx, hy = G.halo, G.haloη, G.halosstx, G.halossty
    return (u[h:u.shape[0] - h, h:u.shape[1] - h].copy(),
            v[h:v.shape[0] - h, h:v.shape[1] - h].copy(),
            η[he:η.shape[0] - he, he:η.shape[1] - he].copy(),
            sst[hy:sst.shape[0] - hy, hx:sst.shape[1] - hx].copy())


# --------------------------------------------------------------------------

def initial_sst(S: ModelSetup) -> np.ndarray:
    """The SST profile of src/initial_conditions.jl:115-140, in Float64."""
    P, G = S.parameters, S.grid
    SSTmin, SSTmax, SSTw, SSTϕ = P.SSTmin, P.SSTmax, P.SSTw, P.SSTϕ
    xx_T = _meshgrid_x(G.x_T, G.ny)
    yy_T = _meshgrid_y(G.y_T, G.nx)
    if P.sst_initial == "south":
        return (SSTmin + SSTmax) / 2 + np.tanh(2 * PI * (G.Ly / (4 * SSTw)) * (yy_T / G.Ly - SSTϕ)) \
            * (SSTmin - SSTmax) / 2
    if P.sst_initial == "west":
        return (SSTmin + SSTmax) / 2 + np.tanh(2 * PI * (G.Lx / (4 * SSTw)) * (xx_T / G.Lx - SSTϕ)) \
            * (SSTmin - SSTmax) / 2
    if P.sst_initial == "flat":
        return np.full(xx_T.shape, float(SSTmin))
    if P.sst_initial == "rect":
        x0, x1, y0, y1 = P.sst_rect_coords
        sst = np.full(xx_T.shape, float(SSTmin))
        inside = (xx_T / G.Lx > x0) & (xx_T / G.Lx < x1) & (yy_T / G.Ly > y0) & (yy_T / G.Ly < y1)
        sst[inside] = SSTmax
        return sst
    raise ValueError(f"sst_initial '{P.sst_initial}' unsupported without a restart file")


def initial_conditions(Tprog, S: ModelSetup, *, u0=None, v0=None, η0=None, sst0=None) -> PrognosticVars:
    """src/initial_conditions.jl:26-164 for ``initial_cond == "rest"``.

    ``u0, v0, η0, sst0`` optionally replace the interior fields (no halo, in
    Float64 or Tprog) before they are rounded to Tprog and the halo is added;
    this is how seeded synthetic inputs enter, since the reference has no hook
    for custom initial states.  ``initial_cond == "ncfile"`` reads u, v, η (and
    sst with ``sst_initial == "restart"``) from a previous run's NetCDF output
    (src/initial_conditions.jl:39-120,144-150; ``output.read_restart``).
    """
    P, G = S.parameters, S.grid
    if P.initial_cond == "ncfile" and u0 is None:
        from .output import read_restart
        u0, v0, η0, sst_r = read_restart(S)
        if sst0 is None and sst_r is not None:
            sst0 = sst_r
    u = np.zeros((G.nuy, G.nux)) if u0 is None else np.asarray(u0)
    v = np.zeros((G.nvy, G.nvx)) if v0 is None else np.asarray(v0)
    η = np.zeros((G.ny, G.nx)) if η0 is None else np.asarray(η0)
    sst = initial_sst(S) if sst0 is None else np.asarray(sst0)
    for name, a, shp in (("u", u, (G.nuy, G.nux)), ("v", v, (G.nvy, G.nvx)),
                         ("η", η, (G.ny, G.nx)), ("sst", sst, (G.ny, G.nx))):
        if a.shape != shp:
            raise ValueError(f"{name} has shape {a.shape}, expected {shp} ([j][i] storage)")
    u, v, η, sst = (Tprog(a).astype(Tprog) for a in (u, v, η, sst))
    return PrognosticVars(*add_halo(u, v, η, sst, S))
