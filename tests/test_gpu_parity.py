"""GPU parity: the CUDA time loop against the CPU oracle, through the C ABI.

Both receive the same config, static fields and seeded state; the library is
built without FMA contraction, so the comparison is bit for bit on the full
arrays with halo (u, v, η, sst) after every checked step count.  Sizes are
small and odd where possible so partial tiles and all boundary code paths run.
"""
import numpy as np
import pytest

import oracle as O
from conftest import assert_bitwise, seeded_inputs
from swb200 import Model, Parameter, initial_conditions, model_setup, run_model

pytestmark = pytest.mark.gpu


def both(kw, nsteps, seed=1, checkpoints=None):
    P = Parameter(**kw)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, seed))
    o = O.Oracle(S)
    o.set_state(Prog)
    m = Model(S)
    m.set_state(Prog)
    done = 0
    for n in (checkpoints or [nsteps]):
        so = o.run(n - done)
        sg = m.run(n - done)
        done = n
        assert so.code == sg.code, (so.code, sg.code)
        a, b = o.get_state(), m.get_state()
        for x, y, name in zip(a, b, ("u", "v", "η", "sst")):
            assert_bitwise(y, x, f"{name} after {n} steps")
    return S, m


BASE = dict(nx=40, Ndays=0.5, Uadv=1000)

CASES = {
    "periodic_const": dict(),
    "periodic_smag": dict(diffusion="Smagorinsky"),
    "nonperiodic": dict(bc="nonperiodic"),
    "nonperiodic_freeslip_seamount_gyre": dict(bc="nonperiodic", α=0, topography="seamount",
                                               wind_forcing_x="double_gyre"),
    "periodic_seamount_smag": dict(topography="seamount", diffusion="Smagorinsky"),
    "periodic_ridges_linear_drag": dict(topography="ridges", bottom_drag="linear"),
    "partial_slip_no_drag": dict(bc="nonperiodic", α=0.5, bottom_drag="none"),
    "rk3": dict(RKo=3, cfl=0.6),
    "rk2": dict(RKo=2, cfl=0.3),
    "seasonal_wind": dict(seasonal_wind_x=True, seasonal_wind_y=True, wind_forcing_y="channel", Fy0=0.05),
    "fy_channel_nonperiodic": dict(bc="nonperiodic", wind_forcing_y="channel", Fy0=0.05),
    "tracer_consumption": dict(tracer_consumption=True),
    "tracer_every_30": dict(Uadv=2.0, Ndays=1),
    "tracer_default_uadv": dict(Uadv=0.25, nx=24, Ndays=2),
    "nstep_diff_3": dict(nstep_diff=3),
    "tcomm_float16": dict(Tcomm=np.float16),
    "float64": dict(T=np.float64),
    "float64_nonperiodic_smag": dict(T=np.float64, bc="nonperiodic", diffusion="Smagorinsky"),
    "mixed_f32_f64": dict(T=np.float32, Tprog=np.float64),
    "odd_37": dict(nx=37),
    "odd_37_nonperiodic": dict(nx=37, bc="nonperiodic", diffusion="Smagorinsky"),
    "wide_130": dict(nx=130, L_ratio=4, Ndays=0.2),
    "square_64_nonperiodic": dict(nx=64, L_ratio=1, bc="nonperiodic", Ndays=0.2),
    # semi-implicit strong-stability-preserving schemes (src/time_integration.jl:80-196)
    "ssprk2_s3": dict(time_scheme="SSPRK2", RKs=3, cfl=1.2),
    "ssprk2_s2_smag": dict(time_scheme="SSPRK2", RKs=2, cfl=0.7, diffusion="Smagorinsky"),
    "ssprk3_n2": dict(time_scheme="SSPRK3", RKn=2, cfl=1.2),
    "ssprk3_n3_nonperiodic": dict(time_scheme="SSPRK3", RKn=3, cfl=2.5, bc="nonperiodic"),
    "4ssprk3": dict(time_scheme="4SSPRK3", cfl=1.0),
    "4ssprk3_nonperiodic_f64": dict(time_scheme="4SSPRK3", bc="nonperiodic", diffusion="Smagorinsky",
                                    T=np.float64),
    "ssprk3_mixed_f32_f64": dict(time_scheme="SSPRK3", RKn=2, T=np.float32, Tprog=np.float64),
    "ssprk2_tcomm_float16": dict(time_scheme="SSPRK2", RKs=3, Tcomm=np.float16, α=0.5, bc="nonperiodic"),
    # continuity! variants (src/continuity.jl:3-49)
    "surface_relax": dict(surface_relax=True),
    "surface_forcing_nonperiodic": dict(surface_forcing=True, bc="nonperiodic"),
    "ssprk2_surface_relax": dict(time_scheme="SSPRK2", RKs=3, cfl=1.2, surface_relax=True),
    "4ssprk3_surface_forcing": dict(time_scheme="4SSPRK3", surface_forcing=True),
    # linear dynamics (src/rhs.jl:59-86); with RK, continuity! sees the never-computed U = V = 0
    "linear": dict(dynamics="linear"),
    "linear_nonperiodic_relax": dict(dynamics="linear", bc="nonperiodic", surface_relax=True),
    "linear_rk3_mixed_f32_f64": dict(dynamics="linear", RKo=3, cfl=0.6, T=np.float32, Tprog=np.float64),
    "linear_advcor_ignored": dict(dynamics="linear", nstep_advcor=2),
    "linear_ssprk2": dict(dynamics="linear", time_scheme="SSPRK2", cfl=0.7),
    "linear_4ssprk3_nonperiodic_f64": dict(dynamics="linear", time_scheme="4SSPRK3", bc="nonperiodic",
                                           T=np.float64),
    # Sadourny's enstrophy-conserving PV advection (src/PV_advection.jl:31-59)
    "sadourny": dict(adv_scheme="Sadourny"),
    "sadourny_nonperiodic_smag": dict(adv_scheme="Sadourny", bc="nonperiodic", diffusion="Smagorinsky"),
    "sadourny_mixed_f32_f64": dict(adv_scheme="Sadourny", T=np.float32, Tprog=np.float64),
    "sadourny_ssprk3_f64": dict(adv_scheme="Sadourny", time_scheme="SSPRK3", RKn=2, cfl=1.2, T=np.float64),
    # advection/Coriolis terms refreshed every nstep_advcor steps (src/time_integration.jl:208-211)
    "advcor_1": dict(nstep_advcor=1),
    "advcor_2_smag": dict(nstep_advcor=2, diffusion="Smagorinsky"),
    "advcor_3_nonperiodic_nstep_diff_2": dict(nstep_advcor=3, nstep_diff=2, bc="nonperiodic"),
    "advcor_2_linear_drag": dict(nstep_advcor=2, bottom_drag="linear"),
    "advcor_2_sadourny_f64": dict(nstep_advcor=2, adv_scheme="Sadourny", T=np.float64),
    "advcor_ssprk2": dict(time_scheme="SSPRK2", RKs=3, cfl=1.2, nstep_advcor=1),
    "advcor_ssprk3_n3_nonperiodic": dict(time_scheme="SSPRK3", RKn=3, cfl=2.5, nstep_advcor=1, bc="nonperiodic"),
    "advcor_2_mixed_f32_f64": dict(nstep_advcor=2, T=np.float32, Tprog=np.float64),
    # Float16 compute with Julia's Float16 arithmetic (test/runtests.jl:37)
    "float16_T_f32_prog": dict(T=np.float16, Tprog=np.float32),
    "float16_all": dict(T=np.float16, Tprog=np.float16),
    "float16_nonperiodic_smag": dict(T=np.float16, Tprog=np.float32, bc="nonperiodic", diffusion="Smagorinsky",
                                     topography="seamount"),
    "float16_ssprk2_advcor": dict(T=np.float16, Tprog=np.float32, time_scheme="SSPRK2", RKs=3, cfl=1.2,
                                  nstep_advcor=1),
    "float16_tracer_every_30_linear_drag": dict(T=np.float16, Tprog=np.float32, Uadv=2.0, Ndays=1,
                                                bottom_drag="linear"),
}


@pytest.mark.parametrize("stage", ["auto", "tma"])
@pytest.mark.parametrize("name", list(CASES))
def test_bitwise_parity(name, stage, monkeypatch):
    """Every option case, bit for bit, with the stage kernel the grid size picks
    (short streaming strips at these sizes) and with the TMA stage kernel
    forced (SWB200_TMA=1; options it does not serve stay streaming)."""
    if stage == "tma":
        monkeypatch.setenv("SWB200_TMA", "1")
    kw = dict(BASE)
    kw.update(CASES[name])
    both(kw, 0, checkpoints=[1, 2, 7, 20])


def test_reference_config_c1_one_day():
    """The periodic wind-driven channel at 100x50 (Smagorinsky, quadratic drag,
    tracer every step) for one day: identical to the oracle."""
    kw = dict(nx=100, L_ratio=2, bc="periodic", wind_forcing_x="channel", Fx0=0.12, topography="flat",
              H=500, g=10, cfl=1, adv_scheme="ArakawaHsu", diffusion="Smagorinsky",
              bottom_drag="quadratic", tracer_advection=True, Uadv=1000, Ndays=1)
    both(kw, 0, checkpoints=[1, 50, 307])


def test_no_forcing_known_answer():                       # test/runtests.jl:4-9
    prog = run_model(Ndays=1, Fx0=0)
    assert np.all(prog.u == 0) and np.all(prog.v == 0) and np.all(prog.η == 0)


@pytest.mark.parametrize("kw", [dict(bc="periodic"), dict(bc="nonperiodic"), dict(α=0)])
def test_boundary_conditions(kw):                         # test/runtests.jl:11-20
    prog = run_model(Ndays=1, **kw)
    assert np.all(np.abs(prog.η) < 10)


def test_mixed_precision_f32_f64():                       # test/runtests.jl:33-35
    prog = run_model(np.float32, Tprog=np.float64, Ndays=1)
    assert prog.u.dtype == np.float64
    assert np.all(np.abs(prog.η) < 10) and np.all(prog.u != 0)


def test_rk3():                                           # test/runtests.jl:42-46
    prog = run_model(time_scheme="RK", RKo=3, cfl=0.6, nstep_advcor=0)
    assert np.all(np.abs(prog.η) < 10) and np.all(prog.u != 0)


def test_nan_detection_matches_reference():
    """NaNs in the state stop the run at the first multiple of nout, returning
    u, v, η from before that step (src/time_integration.jl:235-237)."""
    P = Parameter(nx=20, Ndays=2, Uadv=1000, tracer_advection=False)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S)
    Prog.u[5, 7] = np.nan
    o = O.Oracle(S)
    o.set_state(Prog)
    so = o.run(S.grid.nt)
    m = Model(S)
    m.set_state(Prog)
    sg = m.run(S.grid.nt)
    assert sg.code == so.code == 3
    assert sg.nan_step == so.nan_step == S.grid.nout
    for x, y, name in zip(o.get_state(), m.get_state(), ("u", "v", "η", "sst")):
        assert_bitwise(y, x, name)


def test_time_integration_drop_in_equals_stepping():
    """sw_time_integration (host buffers in/out) equals the context API."""
    from swb200 import time_integration
    P = Parameter(nx=40, Ndays=0.3, Uadv=1000, diffusion="Smagorinsky")
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 3))
    out, st = time_integration(Prog, S)
    assert st.code == 0 and st.steps_done == S.grid.nt
    ref, sto = O.run_model(P=P, **seeded_inputs(S, 3))
    for x, y, name in zip(ref, out, ("u", "v", "η", "sst")):
        assert_bitwise(y, x, name)


def test_kernel_launch_count():
    P = Parameter(nx=40, Ndays=0.3, Uadv=1000)
    S = model_setup(P)
    m = Model(S)
    m.set_state(initial_conditions(P.Tprog, S))
    n0 = m.kernel_launches
    m.run(10)
    # 4 stages + tail + tracer per step, plus NaN checks every nout steps
    assert m.kernel_launches - n0 >= 60


@pytest.mark.parametrize("rows", ["1", "2", "4", "8", "16", "32"])
@pytest.mark.parametrize("kw", [dict(diffusion="Smagorinsky"), dict(bc="nonperiodic", α=0.5, T=np.float64)])
def test_every_tail_strip_height_is_bit_exact(rows, kw, monkeypatch):
    """The streaming tail's strip height (chosen by grid size, forced here with
    SWB200_TAIL_TY) does not change a bit of the result."""
    monkeypatch.setenv("SWB200_TAIL_TY", rows)
    k = dict(BASE)
    k.update(kw)
    both(k, 0, checkpoints=[1, 5])


@pytest.mark.parametrize("rows", ["1", "2", "4", "8", "16", "32"])
@pytest.mark.parametrize("kw", [dict(adv_scheme="Sadourny", diffusion="Smagorinsky"),
                                dict(bc="nonperiodic", α=0.5, topography="seamount"),
                                dict(time_scheme="SSPRK2", RKs=3, cfl=1.0, bc="nonperiodic", α=0.5, T=np.float64),
                                dict(time_scheme="SSPRK3", RKn=2, cfl=1.2, diffusion="Smagorinsky"),
                                dict(time_scheme="4SSPRK3", cfl=1.0, bc="nonperiodic", α=1.0)])
def test_every_stage_strip_height_is_bit_exact(rows, kw, monkeypatch):
    """The streaming stage and SSP momentum kernels' strip height (chosen by
    grid size, forced here with SWB200_STAGE_TY) does not change a bit."""
    monkeypatch.setenv("SWB200_TMA", "0")
    monkeypatch.setenv("SWB200_STAGE_TY", rows)
    k = dict(BASE)
    k.update(kw)
    both(k, 0, checkpoints=[1, 5])


def test_graph_replay_equals_direct_launches(monkeypatch):
    """Steps replayed from CUDA graphs equal steps launched one kernel at a
    time, over enough steps to use every graph key (parities, tracer and
    diffusion sub-steps)."""
    P = Parameter(nx=40, Ndays=0.5, Uadv=2.0, nstep_diff=3, diffusion="Smagorinsky")
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 5))
    out = []
    for graphs in ("1", "0"):
        monkeypatch.setenv("SWB200_GRAPHS", graphs)
        m = Model(S)
        m.set_state(Prog)
        st = m.run(37)
        assert st.code == 0
        out.append(m.get_state())
        m.close()
    for x, y, name in zip(out[0], out[1], ("u", "v", "η", "sst")):
        assert_bitwise(x, y, name)


def test_diagnostics_fp64_reductions():
    """sw_diagnostics: FP64 mass, energy, max speed and NaN count of the
    current state, against numpy in double on the downloaded state."""
    P = Parameter(nx=40, Ndays=0.2, Uadv=1000, bc="nonperiodic", topography="seamount")
    S = model_setup(P)
    m = Model(S)
    m.set_state(initial_conditions(P.Tprog, S, **seeded_inputs(S, 7)))
    m.run(25)
    d = m.diagnostics()
    u, v, e, sst = (np.asarray(a, dtype=np.float64) for a in m.get_state())
    G = S.grid
    N, M, ep = G.nx, G.ny, G.ep
    eta = e[1:M + 1, 1:N + 1]
    H = np.asarray(S.forcing.H, dtype=np.float64)[1:M + 1, 1:N + 1]
    # ([j][i] arrays) u at face F, row b: u[b + 2, F + 1 + ep]; v at column a, face G: v[G + 1, a + 2]
    uu = u[2:M + 2, 1 + ep:N + 2 + ep]
    vv = v[1:M + 2, 2:N + 2]
    energy = np.sum(0.5 * (eta + H) * (0.5 * (uu[:, :-1] ** 2 + uu[:, 1:] ** 2) + 0.5 * (vv[:-1] ** 2 + vv[1:] ** 2))
                    + 0.5 * float(S.parameters.g) * eta ** 2)
    assert uu.shape == (M, N + 1) and vv.shape == (M + 1, N)
    np.testing.assert_allclose(d.mass, eta.sum(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(d.energy, energy, rtol=1e-12)
    assert d.max_speed == max(np.abs(uu[:, :-1]).max(), np.abs(vv[:-1]).max())
    assert d.nan_count == 0


def test_output_frames_match_oracle(tmp_path):
    """run_model(output=true): each frame is the state after step k*nout, the
    du frame the change over that step (src/output.jl:63-133)."""
    import os
    from scipy.io import netcdf_file
    from swb200.initial_conditions import remove_halo
    P = Parameter(nx=40, Ndays=0.3, Uadv=1000, output=True, outpath=str(tmp_path), output_dt=1,
                  output_vars=["u", "η", "sst", "du"])
    S = model_setup(P)
    init = seeded_inputs(S, 8)
    out = run_model(P, **init)
    nout, nt = S.grid.nout, S.grid.nt
    path = os.path.join(str(tmp_path), "run0000")

    def frames(name):
        with netcdf_file(os.path.join(path, name + ".nc"), "r", mmap=False) as nc:
            return np.array(nc.variables[name][:], dtype=np.float32), np.array(nc.variables["t"][:], dtype=np.int64)

    u, t = frames("u")
    du, _ = frames("du")
    assert len(t) == nt // nout + 1
    np.testing.assert_array_equal(t, np.arange(len(t)) * nout * S.grid.dtint)
    o = O.Oracle(S)
    o.set_state(initial_conditions(P.Tprog, S, **init))
    k = 2
    o.run(k * nout - 1)
    before = remove_halo(*o.get_state(), S)[0].astype(np.float32)
    o.run(1)
    after = remove_halo(*o.get_state(), S)[0].astype(np.float32)
    assert_bitwise(u[k], after, "u frame")
    assert_bitwise(du[k], after - before, "du frame")
    if nt % nout == 0:
        assert_bitwise(u[-1], out.u.astype(np.float32), "last frame")


@pytest.mark.parametrize("kw", [dict(), dict(bc="nonperiodic", diffusion="Smagorinsky"),
                                dict(time_scheme="SSPRK2", RKs=3, cfl=1.2)])
def test_vorticity_frames_equal_the_reference_work_arrays(kw):
    """q from the last right-hand-side input (sw_get_rhs_input) equals the
    oracle's q work array after the same steps, bit for bit: the values the
    reference's q frame writes (src/output.jl:105-108)."""
    from swb200.output import vorticities
    P = Parameter(nx=40, Ndays=0.3, Uadv=1000, **kw)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 17))
    o = O.Oracle(S)
    o.set_state(Prog)
    m = Model(S)
    m.set_state(Prog)
    for n in (1, 5):
        o.run(n)
        m.run(n)
        q, _ = vorticities(*m.get_rhs_input(), S)
        qo = o.field("q")[:q.shape[0], :q.shape[1]].astype(np.float32)
        assert_bitwise(q, qo, f"q after {n} more steps")


def test_contexts_reuse_memory_and_trim():
    """Destroyed contexts leave their blocks to the next context of the same
    shape (zeroed again at creation); sw_trim_memory returns them to CUDA."""
    from swb200 import abi
    P = Parameter(nx=40, Ndays=0.2, Uadv=1000)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 13))
    states = []
    for _ in range(2):
        m = Model(S)
        m.set_state(Prog)
        m.run(7)
        states.append(m.get_state())
        m.close()
    for x, y, name in zip(states[0], states[1], ("u", "v", "η", "sst")):
        assert_bitwise(x, y, name)
    lib = abi.load_library()
    assert lib.sw_trim_memory() == abi.SW_OK
    m = Model(S)
    m.set_state(Prog)
    m.run(7)
    for x, y, name in zip(m.get_state(), states[0], ("u", "v", "η", "sst")):
        assert_bitwise(x, y, name)
    m.close()
