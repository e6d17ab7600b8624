"""The host mirror of Grid, Constants and Forcing, pinned to independent values.

The oracle and the GPU both take their grid, constants and forcing from
``swb200.model_setup``, so an error there would pass every parity test.  These
checks recompute what the reference's setup produces directly from its
formulas (src/grid.jl:21-95, src/constants.jl:58-115, src/forcing.jl:57-151)
in plain Python, without calling into the mirror's helpers, and compare:

* the integer time-stepping quantities of the benchmark configurations (the
  literal values below were worked out by hand from src/grid.jl:70-86);
* the array shapes of the prognostic fields with halo;
* spot rows of f_q, the channel and double-gyre winds Fx and the seamount H;
* the rounded RK and diffusion constants handed to the library.
"""
import math

import numpy as np
import pytest

from swb200 import Parameter, initial_conditions, model_setup
from swb200.abi import make_config

# (configuration, Parameter keywords, Δ, dtint, nt, nadvstep at Uadv = 0.25)
CONFIGS = [
    ("C1 channel 100x50, 10 days", dict(nx=100, L_ratio=2, Ndays=10), 20000.0, 282, 3064, 283),
    ("C2 double gyre 512x512, 100 days", dict(nx=512, L_ratio=1, bc="nonperiodic", Ndays=100),
     3906.25, 55, 157091, 284),
    ("C3 channel 2048x1024, 100 days", dict(nx=2048, L_ratio=2, Ndays=100), 976.5625, 13, 664616, 300),
    ("C4 member nx=64, 30 days", dict(nx=64, L_ratio=1, Ndays=30), 31250.0, 441, 5878, None),
    ("C4 member nx=96, 30 days", dict(nx=96, L_ratio=2, Ndays=30), 2000e3 / 96, 294, 8817, None),
    ("C4 member nx=128, 30 days", dict(nx=128, L_ratio=1, Ndays=30), 15625.0, 220, 11782, None),
    ("C4 member nx=192, 30 days", dict(nx=192, L_ratio=2, Ndays=30), 2000e3 / 192, 147, 17633, None),
    ("C4 member nx=256, 30 days", dict(nx=256, L_ratio=1, Ndays=30), 7812.5, 110, 23564, None),
    ("C5 adjoint 512x256", dict(nx=512, L_ratio=2), 3906.25, 55, None, None),
    ("C5 Dual check 128x64", dict(nx=128, L_ratio=2), 15625.0, 220, None, None),
]


@pytest.mark.parametrize("name,kw,delta,dtint,nt,nadv", CONFIGS, ids=[c[0] for c in CONFIGS])
def test_time_stepping_integers(name, kw, delta, dtint, nt, nadv):
    P = Parameter(**kw)
    G = model_setup(P).grid
    assert G.Δ == delta
    assert G.ny == round(2000e3 / kw["L_ratio"] / delta)
    assert G.dtint == dtint                                   # floor(cfl Δ / sqrt(g H)), g = 10, H = 500
    assert G.dtint == math.floor(1.0 * delta / math.sqrt(10.0 * 500.0))
    if nt is not None:
        assert G.nt == nt                                     # ceil(Ndays 86400 / dtint)
        assert G.nt == math.ceil(kw["Ndays"] * 86400 / dtint)
    if nadv is not None:
        assert G.nadvstep == nadv                             # max(1, floor(Δ / Uadv / dtint))
    assert G.nadvstep == max(1, math.floor(delta / 0.25 / dtint))
    assert G.nadvstep_half == G.nadvstep // 2
    assert G.nout == math.floor(6 * 3600 / dtint)             # output_dt = 6 hours
    # Uadv = 1000 (tracer every step) as in the benchmark workloads
    assert model_setup(Parameter(Uadv=1000, **kw)).grid.nadvstep == 1


@pytest.mark.parametrize("bc,ushape,vshape,eshape", [
    ("periodic", (54, 104), (53, 104), (52, 102)),
    ("nonperiodic", (54, 103), (53, 104), (52, 102)),
])
def test_state_shapes_with_halo(bc, ushape, vshape, eshape):
    """u (nux+4) x (M+4), v (N+4) x (M+3), η (N+2) x (M+2), sst (N+2) x M at 100 x 50."""
    P = Parameter(nx=100, L_ratio=2, bc=bc)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S)
    assert Prog.u.shape == ushape and Prog.v.shape == vshape and Prog.η.shape == eshape
    assert Prog.sst.shape == (50, 102)


SIN45 = math.sqrt(0.5)   # sind(45) = cosd(45), correctly rounded


@pytest.mark.parametrize("bc", ["periodic", "nonperiodic"])
def test_coriolis_f_q(bc):
    """f_q = Float32(Δ (f0 + β (y_q - Ly/2))) on the q rows y = jΔ, j = 0..M,
    with f0 = 2ω sind(45°), β = 2ω/R cosd(45°) (src/grid.jl:91-108)."""
    P = Parameter(nx=64, L_ratio=2, bc=bc)
    G = model_setup(P).grid
    omega, R = 2 * math.pi / (24 * 3600), 6.371e6
    f0, beta = 2 * omega * SIN45, 2 * omega / R * SIN45
    delta, M = 2000e3 / 64, G.ny
    Ly = M * delta
    assert G.f_q.shape == (M + 1, 65)
    for j in (0, 1, M // 2, M):
        want = np.float32(delta * (f0 + beta * (j * delta - Ly / 2)))
        assert np.all(G.f_q[j] == want), (j, G.f_q[j][0], want)
    assert abs(float(G.f_q[M // 2, 0]) - delta * f0) < 1e-6 * delta * f0    # f0 at mid-channel


def test_channel_wind():
    """Fx = Float32((Δ Fx0 / ρ / H) cos²(π (y_u/Ly - 1/2))) on the u rows
    y_u = (j + 1/2)Δ (src/forcing.jl:57-68): zero-ish at the walls, Fx0 Δ/(ρH) mid-channel."""
    P = Parameter(nx=100, L_ratio=2, Fx0=0.12)
    F = model_setup(P).forcing
    delta, M = 20000.0, 50
    amp = delta * 0.12 / 1000.0 / 500.0
    assert F.Fx.shape == (M, 100)
    for j in (0, 7, 24, 25, 49):
        y = (j + 0.5) * delta
        want = np.float32(amp * math.cos(math.pi * (y / (M * delta) - 0.5)) ** 2)
        np.testing.assert_allclose(F.Fx[j], want, rtol=2e-7, atol=0)
        assert np.all(F.Fx[j] == F.Fx[j, 0])
    assert np.float32(amp) >= F.Fx[24, 0] > np.float32(0.99 * amp)


def test_double_gyre_wind():
    """Fx = (Δ Fx0/ρ/H)(cos(2π(y/Ly - 1/2)) + 2 sin(π(y/Ly - 1/2))) (src/forcing.jl:88-98)."""
    P = Parameter(nx=128, L_ratio=1, bc="nonperiodic", wind_forcing_x="double_gyre", Fx0=0.12)
    F = model_setup(P).forcing
    delta, M = 15625.0, 128
    amp = delta * 0.12 / 1000.0 / 500.0
    assert F.Fx.shape == (M, 127)
    for j in (0, 31, 64, 100, 127):
        s = ((j + 0.5) * delta) / (M * delta) - 0.5
        want = np.float32(amp * (math.cos(2 * math.pi * s) + 2 * math.sin(math.pi * s)))
        np.testing.assert_allclose(F.Fx[j], want, rtol=2e-7, atol=1e-12)
    # the sign change between the gyres: negative in the south, positive in the north
    assert F.Fx[0, 0] < 0 < F.Fx[M - 1, 0]


def test_seamount_depth():
    """H = Float32(H0 - h exp(-(x-Lx/2)²/2w²) exp(-(y-Ly/2)²/2w²)) on the T grid
    with halo, x_T_halo = (i - 1/2)Δ for i = 0..N+1 (src/forcing.jl:141-151)."""
    P = Parameter(nx=128, L_ratio=1, bc="nonperiodic", topography="seamount", topo_height=50, H=500)
    F = model_setup(P).forcing
    delta, N, w = 15625.0, 128, 300e3
    assert F.H.shape == (N + 2, N + 2)
    for (j, i) in [(0, 0), (65, 65), (64, 65), (30, 90), (N + 1, N + 1)]:
        x, y = (i - 0.5) * delta, (j - 0.5) * delta
        bump = math.exp(-((x - N * delta / 2) ** 2) / (2 * w ** 2)) * math.exp(-((y - N * delta / 2) ** 2) / (2 * w ** 2))
        want = np.float32(500 - 50 * bump)
        np.testing.assert_allclose(F.H[j, i], want, rtol=2e-7)
    assert float(F.H.min()) > 450 and float(F.H.max()) < 500


def test_flat_bottom_and_rk_constants():
    """Flat H = 500; RKaΔt = (1/6, 1/3, 1/3, 1/6) dtint/Δ and RKbΔt = (1/2, 1/2, 1)
    dtint/Δ in Tprog, Δt_diff = nstep_diff dtint/Δ (src/constants.jl:58-72,
    src/grid.jl:74), g and cD = -Δ cD rounded to T."""
    P = Parameter(nx=2048, L_ratio=2, topography="flat", H=500, diffusion="Smagorinsky", nstep_diff=1)
    S = model_setup(P)
    assert np.all(S.forcing.H == np.float32(500))
    cfg = make_config(S)
    # Julia's [a...]*dtint/Δ multiplies each coefficient by dtint, then divides by Δ
    for k, a in enumerate((1 / 6, 1 / 3, 1 / 3, 1 / 6)):
        assert cfg.RKaDt[k] == float(np.float32(a * 13 / 976.5625))
    for k, b in enumerate((0.5, 0.5, 1.0)):
        assert cfg.RKbDt[k] == float(np.float32(b * 13 / 976.5625))
    assert cfg.Dt_diff == float(np.float32(1 * 13 / 976.5625))
    assert cfg.g == 10.0
    assert cfg.cD == float(np.float32(-976.5625 * 1e-5))
    assert cfg.cSmag == float(np.float32(-0.15))
    assert cfg.dtint == 13 and cfg.nx == 2048 and cfg.ny == 1024
