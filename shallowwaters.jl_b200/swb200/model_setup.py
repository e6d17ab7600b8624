"""Grid, Constants, Forcing and ModelSetup: the host-side inputs of the time loop.

These stay on the host (they run once) and are restated here from
ShallowWaters.jl with the reference's Float64 operation order, rounding to
T/Tprog only where the reference does:

* ``Grid``      src/grid.jl:1-159
* ``Constants`` src/constants.jl:1-115 (``SSPRK3coeff`` :4-27)
* ``Forcing``   src/forcing.jl:1-217
* ``ModelSetup`` src/model_setup.jl:1-6

Python floats are IEEE binary64 and every expression below keeps the
reference's evaluation order, so the Float64 intermediates match Julia's.
Transcendentals (cos, tanh, exp, sin) come from the C library; Julia's own
implementations agree with them to within one unit in the last place of the
Float64 value, which the final rounding to Float32 hides except in rare ties.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from decimal import Decimal, getcontext

import numpy as np

from .parameter import Parameter

PI = math.pi  # Float64(π)


# --------------------------------------------------------------------------
# degree-exact trigonometry (Julia's sind/cosd reduce in degrees and evaluate
# in extended precision; computing the exactly rounded value gives the same
# Float64 for the latitudes used by the model)

def _dec_pi():
    getcontext().prec = 50
    # Machin's formula
    def arctan_inv(x):
        x = Decimal(x)
        s, t, n, sign = Decimal(0), 1 / x, 1, 1
        x2 = x * x
        while True:
            term = t / n
            if term == 0 or abs(term) < Decimal(10) ** -48:
                break
            s += sign * term
            t /= x2
            n += 2
            sign = -sign
        return s
    return 4 * (4 * arctan_inv(5) - arctan_inv(239))


_DPI = None


def _dec_sin_cos(xdeg: float):
    global _DPI
    if _DPI is None:
        _DPI = _dec_pi()
    getcontext().prec = 50
    x = Decimal(xdeg) * _DPI / 180
    # Taylor series (|x| <= 2π after reduction)
    s, c = Decimal(0), Decimal(0)
    term_s, term_c = x, Decimal(1)
    n = 0
    while True:
        s += term_s
        c += term_c
        term_s = -term_s * x * x / ((2 * n + 2) * (2 * n + 3))
        term_c = -term_c * x * x / ((2 * n + 1) * (2 * n + 2))
        n += 1
        if abs(term_s) < Decimal(10) ** -45 and abs(term_c) < Decimal(10) ** -45:
            break
    return s, c


def sind(x: float) -> float:
    """sin of x degrees, rounded once to Float64."""
    r = math.fmod(x, 360.0)
    if r == 0.0:
        return math.copysign(0.0, x)
    return float(_dec_sin_cos(r)[0])


def cosd(x: float) -> float:
    """cos of x degrees, rounded once to Float64."""
    r = math.fmod(x, 360.0)
    return float(_dec_sin_cos(r)[1])


def coriolis_at_lat(ω, ϕ):
    """src/grid.jl:130-132."""
    return 2 * ω * sind(ϕ)


def β_at_lat(ω, R, ϕ):
    """src/grid.jl:136-138."""
    return 2 * ω / R * cosd(ϕ)


def _arange(a, b):
    """Julia's Array(a:b) as Float64 values."""
    return np.arange(a, b + 1, dtype=np.float64)


def _as_real(x):
    """Julia keeps Int/Float64 as given for ``::Real`` fields."""
    return x


# --------------------------------------------------------------------------

class Grid:
    """src/grid.jl:1-96."""

    def __init__(self, P: Parameter):
        T, Tprog = P.T, P.Tprog
        self.T, self.Tprog = T, Tprog
        nx, Lx, L_ratio, bc = P.nx, P.Lx, P.L_ratio, P.bc
        self.nx, self.Lx, self.L_ratio, self.bc = nx, Lx, L_ratio, bc
        self.g, self.H, self.cfl, self.Ndays = P.g, P.H, P.cfl, P.Ndays
        self.nstep_diff, self.nstep_advcor = P.nstep_diff, P.nstep_advcor
        self.Uadv, self.output_dt = P.Uadv, P.output_dt
        self.ω, self.ϕ, self.R = P.ω, P.ϕ, P.R

        # DOMAIN SIZES (:21-23)
        Δ = Lx / nx
        ny = int(round(Lx / L_ratio / Δ))          # round half to even, like Julia
        Ly = ny * Δ
        self.Δ, self.ny, self.Ly = Δ, ny, Ly

        # NUMBER OF GRID POINTS (:26-37)
        per = bc == "periodic"
        self.nux = nx if per else nx - 1
        self.nuy = ny
        self.nvx = nx
        self.nvy = ny - 1
        self.nqx = nx if per else nx + 1
        self.nqy = ny + 1
        self.nT = nx * ny
        self.nu = self.nux * self.nuy
        self.nv = self.nvx * self.nvy
        self.nq = self.nqx * self.nqy

        # GRID VECTORS (:40-47)
        self.x_T = Δ * _arange(1, nx) - Δ / 2
        self.y_T = Δ * _arange(1, ny) - Δ / 2
        self.x_u = Δ * _arange(0, nx - 1) if per else Δ * _arange(1, nx - 1)
        self.y_u = self.y_T
        self.x_v = self.x_T
        self.y_v = Δ * _arange(1, ny - 1)
        self.x_q = self.x_u if per else Δ * _arange(1, nx + 1) - Δ
        self.y_q = Δ * _arange(1, ny + 1) - Δ

        # HALO SIZES (:50-53)
        self.halo, self.haloη, self.halosstx, self.halossty = 2, 1, 1, 0

        # EDGE POINT (:56)
        self.ep = 1 if per else 0

        # GRID VECTORS WITH HALO (:59-66)
        self.x_T_halo = Δ * _arange(0, nx + 1) - Δ / 2
        self.y_T_halo = Δ * _arange(0, ny + 1) - Δ / 2
        self.x_u_halo = Δ * _arange(-2, nx + 1) if per else Δ * _arange(-1, nx + 1)
        self.y_u_halo = Δ * _arange(-1, ny + 2) - Δ / 2
        self.x_v_halo = Δ * _arange(-1, nx + 2) - Δ / 2
        self.y_v_halo = Δ * _arange(-1, ny + 1)
        self.x_q_halo = self.x_u_halo if per else Δ * _arange(-1, nx + 3) - Δ
        self.y_q_halo = Δ * _arange(-1, ny + 3) - Δ

        # TIME STEPS (:69-74)
        self.c = math.sqrt(self.g * self.H)
        self.dtint = int(math.floor(self.cfl * Δ / self.c))
        if self.dtint < 1:
            raise ValueError("time step dtint rounds to 0 s; lower the resolution or raise cfl")
        self.nt = int(math.ceil(self.Ndays * 3600 * 24 / self.dtint))
        self.dt = T(self.dtint)
        self.Δt = T(self.dtint / Δ)
        self.Δt_diff = Tprog(self.nstep_diff * self.dtint / Δ)

        # TIME STEPS FOR ADVECTION (:77-83)
        self.nadvstep = max(1, int(math.floor(Δ / self.Uadv / self.dtint)))
        self.nadvstep_half = self.nadvstep // 2
        self.dtadvint = self.nadvstep * self.dtint
        self.dtadvu = T(self.dtadvint * nx / Lx)
        self.dtadvv = T(self.dtadvint * ny / Ly)
        self.half_dtadvu = T(self.dtadvint * nx / Lx / 2)
        self.half_dtadvv = T(self.dtadvint * ny / Ly / 2)

        # N TIME STEPS FOR OUTPUT (:86-88)
        self.nout = int(math.floor(self.output_dt * 3600 / self.dtint))
        if self.nout < 1:
            self.nout = 1  # the reference would divide by zero in `i % nout`
        self.nout_total = (self.nt // self.nout) + 1

        # CORIOLIS (:91-95)
        self.f0 = coriolis_at_lat(self.ω, self.ϕ)
        self.β = β_at_lat(self.ω, self.R, self.ϕ)
        f0, β = self.f0, self.β
        # meshgrid(x,y)[2] repeats y along x: value depends on the y index only
        self.f_u = np.tile(T(Δ * (f0 + β * (self.y_u - Ly / 2))), (self.nux, 1)).T.copy()
        self.f_v = np.tile(T(Δ * (f0 + β * (self.y_v - Ly / 2))), (self.nvx, 1)).T.copy()
        yq = self.y_q_halo[2:-2]                     # y_q_halo[3:end-2] (:99-108)
        nfq = nx + 1                                 # x_q_halo[3:end-1] or [3:end-2]
        self.f_q = np.tile(T(Δ * (f0 + β * (yq - Ly / 2))), (nfq, 1)).T.copy()
        # all 2-D fields here are stored [j][i] (x fastest), i.e. Julia's layout


def _ssprk3(P: Parameter, Δt_Δ, Tprog):
    """SSPRK3coeff (src/constants.jl:4-27)."""
    n = P.RKn
    s = n ** 2
    kn = n * (n + 1) // 2 + 1
    mn = (n - 1) * (n - 2) // 2 + 1
    Δt_Δn = Tprog(float(Δt_Δ) / (n ** 2 - n))
    kna = Tprog((n - 1) / (2 * n - 1))
    knb = Tprog(n / (2 * n - 1))
    Δt_Δnc = Tprog(float(Δt_Δ) / (n * (2 * n - 1)))
    return dict(n=n, s=s, kn=kn, mn=mn, Δt_Δn=Δt_Δn, kna=kna, knb=knb, Δt_Δnc=Δt_Δnc)


class Constants:
    """src/constants.jl:29-115."""

    def __init__(self, P: Parameter, G: Grid):
        T, Tprog = P.T, P.Tprog
        dtint, Δ = G.dtint, G.Δ
        # RK coefficients (:63-72): ([a...]*dtint)/Δ element-wise in Float64
        if P.RKo == 2:
            a, b = [1 / 2, 1 / 2], [1.0]
        elif P.RKo == 3:
            a, b = [1 / 4, 0., 3 / 4], [1 / 3, 2 / 3]
        else:
            a, b = [1 / 6, 1 / 3, 1 / 3, 1 / 6], [.5, .5, 1.]
        self.RKaΔt = [Tprog(x * dtint / Δ) for x in a]
        self.RKbΔt = [Tprog(x * dtint / Δ) for x in b]
        self.Δt_Δs = Tprog(dtint / Δ / (P.RKs - 1))                      # :76
        self.Δt_Δ = Tprog(dtint / Δ)                                      # :79
        self.Δt_Δ_half = Tprog(dtint / Δ / 2)                             # :80
        # SSPRK3coeff{Tprog}(P,Δt_Δ): Δt_Δ enters already rounded to Tprog
        self.SSPRK3c = _ssprk3(P, self.Δt_Δ, Tprog)                      # :83
        self.one_minus_α = Tprog(1 - P.α)                                 # :86
        self.g = T(P.g)                                                   # :87
        self.cD = T(-Δ * P.cD)                                            # :91
        self.rD = T(-Δ / (P.τD * 24 * 3600)) if P.τD != 0 else T(-math.inf)  # :92
        self.γ = T(Δ / (P.t_relax * 3600 * 24))                          # :96
        self.cSmag = T(-P.cSmag)                                          # :99
        self.νB = T(-P.νB / 30000)                                        # :100
        self.rSST = T(G.dtadvint / (P.τSST * 3600 * 24))                  # :103
        self.jSST = T(G.dtadvint / (P.jSST * 3600 * 24))                  # :104
        self.SSTmin = T(P.SSTmin)                                         # :105
        self.ωFη = -2 * PI * P.ωFη / 24 / 365.25 / 3600                  # :108
        self.ωFx = 2 * PI * P.ωFx / 24 / 365.25 / 3600                   # :109
        self.ωFy = 2 * PI * P.ωFy / 24 / 365.25 / 3600                   # :110


def _meshgrid_y(y, nxx):
    """meshgrid(x,y)[2] in [j][i] storage: row j holds y[j]."""
    return np.tile(y[:, None], (1, nxx))


def _meshgrid_x(x, nyy):
    """meshgrid(x,y)[1] in [j][i] storage: column i holds x[i]."""
    return np.tile(x[None, :], (nyy, 1))


class Forcing:
    """src/forcing.jl:1-53.  Fields stored [j][i] (x fastest)."""

    def __init__(self, P: Parameter, G: Grid):
        T = P.T
        wx, wy = P.wind_forcing_x, P.wind_forcing_y
        winds = {"channel": self.channel_wind, "shear": self.shear_wind,
                 "double_gyre": self.double_gyre_wind, "constant": self.constant_wind,
                 "none": self.no_wind}
        self.Fx = winds[wx](T, P, G)[0]
        if wy == "none" and wx != "none":
            # src/forcing.jl:35 tests wind_forcing_x in the Fy "none" branch,
            # which leaves Fy undefined in the reference.
            raise ValueError("wind_forcing_y='none' requires wind_forcing_x='none' "
                             "(src/forcing.jl:35 leaves Fy undefined otherwise)")
        self.Fy_raw = winds[wy](T, P, G)[1]
        self.Fy = self.fy_as_read(self.Fy_raw, G)

        topo = P.topography
        if topo == "ridge":
            self.H = self.ridge(T, P, G)[0]
        elif topo == "ridges":
            self.H = self.ridges(T, P, G)
        elif topo == "seamount":
            self.H = self.seamount(T, P, G)
        else:
            self.H = self.flat_bottom(T, P, G)

        self.η_ref = self.interface_relaxation(T, P, G)
        self.Fη = self.kelvin_pump(T, P, G)

    @staticmethod
    def fy_as_read(Fy_raw, G):
        """The N x (M-1) values momentum_v! reads from Fy.

        momentum_v! (src/rhs.jl:269-273) reads ``Fy[i,j]`` for i<=nvx, j<=nvy
        under @inbounds, i.e. at linear index (i-1)+(j-1)*size(Fy,1).  The
        channel/shear/double-gyre winds build Fy on the u-grid (nux x nuy,
        src/forcing.jl:63-65), whose first dimension is N-1 in the nonperiodic
        case, so the values read there come from that linear indexing.
        """
        m_raw = Fy_raw.shape[1]
        flat = Fy_raw.reshape(-1)                    # Julia's linear order
        i = np.arange(G.nvx)[None, :]
        j = np.arange(G.nvy)[:, None]
        return flat[i + j * m_raw].copy()

    # --- winds (src/forcing.jl:57-123) ------------------------------------
    @staticmethod
    def channel_wind(T, P, G):
        xx_u = _meshgrid_x(G.x_u, G.ny)
        yy_u = _meshgrid_y(G.y_u, len(G.x_u))
        Fx = (G.Δ * P.Fx0 / P.ρ / P.H) * np.cos(PI * (yy_u / G.Ly - 1 / 2)) ** 2
        Fy = (G.Δ * P.Fy0 / P.ρ / P.H) * np.cos(PI * (xx_u / G.Lx - 1 / 2)) ** 2
        return T(Fx), T(Fy)

    @staticmethod
    def shear_wind(T, P, G):
        xx_u = _meshgrid_x(G.x_u, G.ny)
        yy_u = _meshgrid_y(G.y_u, len(G.x_u))
        Fx = (G.Δ * P.Fx0 / P.ρ / P.H) * np.tanh(2 * PI * (yy_u / G.Ly - 1 / 2))
        Fy = (G.Δ * P.Fy0 / P.ρ / P.H) * np.tanh(2 * PI * (xx_u / G.Lx - 1 / 2))
        return T(Fx), T(Fy)

    @staticmethod
    def double_gyre_wind(T, P, G):
        xx_u = _meshgrid_x(G.x_u, G.ny)
        yy_u = _meshgrid_y(G.y_u, len(G.x_u))
        Fx = (G.Δ * P.Fx0 / P.ρ / P.H) * (np.cos(2 * PI * (yy_u / G.Ly - 1 / 2))
                                          + 2 * np.sin(PI * (yy_u / G.Ly - 1 / 2)))
        Fy = (G.Δ * P.Fy0 / P.ρ / P.H) * (np.cos(2 * PI * (xx_u / G.Lx - 1 / 2))
                                          + 2 * np.sin(PI * (xx_u / G.Lx - 1 / 2)))
        return T(Fx), T(Fy)

    @staticmethod
    def constant_wind(T, P, G):
        Fx = np.full((G.nuy, G.nux), T(T(G.Δ * P.Fx0 / P.ρ / P.H) * T(1)), dtype=T)
        Fy = np.full((G.nvy, G.nvx), T(T(G.Δ * P.Fy0 / P.ρ / P.H) * T(1)), dtype=T)
        return Fx, Fy

    @staticmethod
    def no_wind(T, P, G):
        return np.zeros((G.nuy, G.nux), dtype=T), np.zeros((G.nvy, G.nvx), dtype=T)

    # --- relaxation / pumping (src/forcing.jl:127-136, 198-212) -----------
    @staticmethod
    def interface_relaxation(T, P, G):
        yy_T = _meshgrid_y(G.y_T, G.nx)
        η_ref = -(P.η_refh / 2) * np.tanh(2 * PI * (G.Ly / (4 * P.η_refw)) * (yy_T / G.Ly - 1 / 2))
        return T(η_ref)

    @staticmethod
    def kelvin_pump(T, P, G):
        yy_T = _meshgrid_y(G.y_T, G.nx)
        mϕ = 2 * PI * G.R / 360.
        y0 = G.Ly / 2 - (G.ϕ - P.ϕk) * mϕ
        Fη = P.A * G.Δ * np.exp(-(yy_T - y0) ** 2 / (2 * P.wk ** 2))
        return T(Fη)

    # --- topography (src/forcing.jl:141-195) --------------------------------
    @staticmethod
    def seamount(T, P, G):
        xx_T = _meshgrid_x(G.x_T_halo, len(G.y_T_halo))
        yy_T = _meshgrid_y(G.y_T_halo, len(G.x_T_halo))
        bumpx = np.exp(-((xx_T - G.Lx / 2) ** 2) / (2 * P.topo_width ** 2))
        bumpy = np.exp(-((yy_T - G.Ly / 2) ** 2) / (2 * P.topo_width ** 2))
        return T(P.H - P.topo_height * bumpx * bumpy)

    @staticmethod
    def ridge(T, P, G):
        xx_T = _meshgrid_x(G.x_T_halo, len(G.y_T_halo))
        yy_T = _meshgrid_y(G.y_T_halo, len(G.x_T_halo))
        bumpx = np.exp(-((xx_T - G.Lx / 2) ** 2) / (2 * P.topo_width ** 2))
        bumpy = np.exp(-((yy_T - G.Ly / 2) ** 2) / (2 * P.topo_width ** 2))
        Hx = P.H - P.topo_height * bumpx
        Hy = P.H - P.topo_height * bumpy
        return T(Hx), T(Hy)

    @staticmethod
    def ridges(T, P, G):
        xx_T = _meshgrid_x(G.x_T_halo, len(G.y_T_halo))
        w2 = 2 * P.topo_width ** 2
        b0x = np.exp(-(xx_T ** 2) / w2)
        b1x = np.exp(-((xx_T - 0.99 * G.Lx / 4) ** 2) / w2)
        b2x = np.exp(-((xx_T - 1.01 * G.Lx / 2) ** 2) / w2)
        b3x = np.exp(-((xx_T - 0.99 * 3 * G.Lx / 4) ** 2) / w2)
        b4x = np.exp(-((xx_T - G.Lx) ** 2) / w2)
        th = P.topo_height
        return T(P.H - th * b0x - th * b1x - th * b2x - th * b3x - th * b4x)

    @staticmethod
    def flat_bottom(T, P, G):
        return np.full((G.ny + 2 * G.haloη, G.nx + 2 * G.haloη), T(P.H), dtype=T)


def ftime(T, t: int, ω: float):
    """Ftime (src/forcing.jl:215-217)."""
    return T(math.sin(ω * t))


@dataclass
class ModelSetup:
    """src/model_setup.jl:1-6."""
    parameters: Parameter
    grid: Grid
    constants: Constants
    forcing: Forcing


def model_setup(P: Parameter) -> ModelSetup:
    """The setup half of run_model(T,P) (src/run_model.jl:25-33)."""
    G = Grid(P)
    C = Constants(P, G)
    F = Forcing(P, G)
    return ModelSetup(P, G, C, F)
