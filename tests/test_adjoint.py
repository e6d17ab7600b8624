"""The adjoint (sw_adjoint_run): gradients of J = sum (eta_T - eta_obs)^2.

CPU: the Dual-number oracle (forward-mode directional derivative of the
restated loop) against central finite differences of the Float64 oracle; and
a host check build of the adjoint's own passes (sw_adjoint.cu compiled with
SWA_HOST_CHECK: the same code in host loops, every array access checked
against its reference shape) against the oracle and the Dual derivative.
GPU: the adjoint's own forward recomputation is bit-identical with the time
loop; <gradient, direction> equals the Dual directional derivative to 1e-4
relative (and finite differences of the GPU forward); the checkpoint schedule
does not change the gradient.
"""
import ctypes as C
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO

sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle  # noqa: E402

from swb200 import Parameter, PrognosticVars, abi, initial_conditions, model_setup  # noqa: E402
from swb200.adjoint import gradient, twin, with_Fx  # noqa: E402

DUAL_RTOL = 1e-4       # adjoint vs Dual directional derivative (Float64)

# option sets covered (stable at their cfl)
OPTIONS = [dict(), dict(bc="nonperiodic", α=0.5), dict(diffusion="constant"),
           dict(bottom_drag="linear", bc="nonperiodic", α=0.0), dict(RKo=3, bottom_drag="none", cfl=0.5),
           dict(RKo=2, bc="nonperiodic", α=2.0, cfl=0.3),
           dict(time_scheme="SSPRK2", RKs=3, cfl=1.0),
           dict(time_scheme="SSPRK2", RKs=2, cfl=0.6, bc="nonperiodic", α=0.5, diffusion="constant"),
           dict(adv_scheme="Sadourny"), dict(adv_scheme="Sadourny", bc="nonperiodic", α=1.0, time_scheme="SSPRK2",
                                             RKs=3, cfl=1.0),
           dict(surface_relax=True), dict(surface_relax=True, time_scheme="SSPRK2", RKs=3, cfl=1.0),
           dict(nstep_diff=3), dict(nstep_diff=2, time_scheme="SSPRK2", RKs=2, cfl=0.6),
           dict(seasonal_wind_x=True, ωFx=40.0), dict(surface_forcing=True, ωFη=40.0, seasonal_wind_y=True, ωFy=30.0,
                                                     time_scheme="SSPRK2", RKs=3, cfl=1.0),
           dict(dynamics="linear", surface_relax=True), dict(dynamics="linear", time_scheme="SSPRK2", RKs=3, cfl=1.0,
                                                             bc="nonperiodic", α=0.5),
           dict(time_scheme="4SSPRK3", cfl=1.0), dict(time_scheme="4SSPRK3", cfl=1.0, bc="nonperiodic", α=0.5,
                                                      adv_scheme="Sadourny"),
           dict(time_scheme="SSPRK3", RKn=2, cfl=1.2),
           dict(time_scheme="SSPRK3", RKn=3, cfl=2.0, bc="nonperiodic", α=0.5, surface_relax=True)]


def setup(T=np.float64, seed=3, **kw):
    pkw = dict(nx=32, L_ratio=2, bc="periodic", tracer_advection=False, Fx0=0.12, diffusion="Smagorinsky")
    pkw.update(kw)
    P = Parameter(T=T, **pkw)
    S = model_setup(P)
    rng = np.random.default_rng(seed)
    Prog = initial_conditions(P.Tprog, S, η0=rng.normal(0, 0.01, (S.grid.ny, S.grid.nx)))
    obs = rng.normal(0, 0.01, (S.grid.ny, S.grid.nx)).astype(T)
    return S, Prog, obs, rng


def direction(S, Prog, rng, uv=True):
    """A seeded direction in the interior of u, v, eta and in Fx."""
    u, v, e, _ = Prog
    du, dv, de = np.zeros_like(u), np.zeros_like(v), np.zeros_like(e)
    if uv:
        du[2:-2, 2:-2] = rng.normal(0, 1e-4, du[2:-2, 2:-2].shape)
        dv[2:-2, 2:-2] = rng.normal(0, 1e-4, dv[2:-2, 2:-2].shape)
    de[1:-1, 1:-1] = rng.normal(0, 1e-3, de[1:-1, 1:-1].shape)
    dF = rng.normal(0, 1e-2, S.forcing.Fx.shape) * np.abs(S.forcing.Fx).max()
    return du, dv, de, dF


@pytest.mark.parametrize("bc", ["periodic", "nonperiodic"])
def test_dual_oracle_matches_central_differences(bc):
    S, Prog, obs, rng = setup(bc=bc, α=0.5)
    n = 40
    du, dv, de, dF = direction(S, Prog, rng)
    J, dJ = oracle.jvp(S, Prog, obs, n, du=du, dv=dv, deta=de, dFx=dF)
    u, v, e, sst = Prog

    def J_at(s):
        return oracle.cost(with_Fx(S, S.forcing.Fx + s * dF), PrognosticVars(u + s * du, v + s * dv, e + s * de, sst),
                           obs, n)

    assert J == pytest.approx(J_at(0.0), rel=1e-14)
    eps = 1e-3
    fd = (J_at(eps) - J_at(-eps)) / (2 * eps)
    assert fd == pytest.approx(dJ, rel=1e-7)


def test_adjoint_entry_rejects_bad_arguments_and_unbuilt_options():
    """sw_adjoint_run's checks: bad arguments give SW_ERR_ARG and option
    combinations outside the differentiated loop SW_ERR_UNSUPPORTED, before any
    device work; on a machine without a GPU a valid call gives SW_ERR_NODEVICE."""
    import torch
    from swb200.adjoint import gradient as grad
    S, Prog, obs, _ = setup()
    with pytest.raises(abi.SwError) as e:
        grad(S, Prog, obs, 0)
    assert e.value.code == abi.SW_ERR_ARG
    for kw in (dict(time_scheme="SSPRK3", RKn=4, cfl=2.0), dict(nstep_advcor=2),
               dict(T=np.float32, Tprog=np.float64)):
        S2, P2, o2, _ = setup(**kw)
        with pytest.raises(abi.SwError) as e:
            grad(S2, P2, o2, 3)
        assert e.value.code == abi.SW_ERR_UNSUPPORTED, kw
    if not torch.cuda.is_available():
        with pytest.raises(abi.SwError) as e:
            grad(S, Prog, obs, 3)
        assert e.value.code == abi.SW_ERR_NODEVICE


def _production_eta(S, Prog, n):
    from swb200 import Model
    with Model(S) as m:
        m.set_state(Prog)
        m.run(n)
        return m.get_state().η


def directional(r, d):
    """<gradient, direction> over the controls given (None skipped)."""
    return float(sum(np.sum(g * x) for g, x in zip((r[0], r[1], r[2], r[3]), d) if x is not None))


@pytest.fixture(scope="module")
def host_check_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available for the host check build")
    out = str(tmp_path_factory.mktemp("hc") / "libswadj_host.so")
    src = os.path.join(REPO, "shallowwaters.jl_b200", "csrc", "sw_adjoint.cu")
    ccbin = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []
    subprocess.run([nvcc, "-O1", "-std=c++17", "--fmad=false", "--extended-lambda", "-DSWA_HOST_CHECK",
                    "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(REPO, "include"), *ccbin,
                    "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", out, src], check=True)
    L = C.CDLL(out)
    L.swa_host_check_run.argtypes = [C.c_void_p] * 6 + [C.c_int64, C.c_int32, C.POINTER(C.c_double)] + \
        [C.c_void_p] * 5 + [C.POINTER(C.c_longlong)]
    return L


def host_check_gradient(L, S, Prog, obs, n, nc):
    T = S.parameters.T
    cfg, st = abi.make_config(S, nt=n), abi.StaticFields(S)
    u, v, e = (np.ascontiguousarray(a, dtype=T) for a in list(Prog)[:3])
    obs = np.ascontiguousarray(obs, dtype=T)
    g = [np.zeros_like(u), np.zeros_like(v), np.zeros_like(e), np.zeros(S.forcing.Fx.shape, T)]
    ef = np.zeros_like(e)
    J, bad = C.c_double(), C.c_longlong()
    rc = L.swa_host_check_run(C.byref(cfg), st.ptr(), u.ctypes.data, v.ctypes.data, e.ctypes.data, obs.ctypes.data,
                              n, nc, C.byref(J), *[x.ctypes.data for x in g], ef.ctypes.data, C.byref(bad))
    assert rc == 0
    return J.value, g, ef, bad.value


@pytest.mark.parametrize("opts", OPTIONS)
def test_host_check_of_the_adjoint_passes(host_check_lib, opts):
    """Every access of every forward and reverse pass stays inside its array;
    the recomputed forward is the oracle's bit for bit; the gradient matches
    the Dual derivative per control; a 3-slot checkpoint schedule gives the
    same numbers."""
    S, Prog, obs, rng = setup(nx=32, seed=11, **opts)
    n = 12
    J, g, ef, bad = host_check_gradient(host_check_lib, S, Prog, obs, n, n)
    assert bad == 0
    o = oracle.Oracle(S)
    o.set_state(Prog)
    o.run(n)
    assert np.array_equal(ef, o.get_state().η)
    du, dv, de, dF = direction(S, Prog, rng)
    for d in ((du, dv, de, dF), (du, None, None, None), (None, dv, None, None), (None, None, de, None),
              (None, None, None, dF)):
        Jd, dJ = oracle.jvp(S, Prog, obs, n, du=d[0], dv=d[1], deta=d[2], dFx=d[3])
        assert J == pytest.approx(Jd, rel=1e-13)
        assert directional(g, d) == pytest.approx(dJ, rel=1e-10)
    J3, g3, _, bad3 = host_check_gradient(host_check_lib, S, Prog, obs, n, 3)     # two-level schedule
    assert bad3 == 0 and J3 == J
    for a, b in zip(g3, g):
        assert np.array_equal(a, b)
    os.environ["SWB200_ADJ_SCHEDULE"] = "binomial"
    try:
        J3b, g3b, _, bad3b = host_check_gradient(host_check_lib, S, Prog, obs, n, 3)
    finally:
        del os.environ["SWB200_ADJ_SCHEDULE"]
    assert bad3b == 0 and J3b == J
    for a, b in zip(g3b, g):
        assert np.array_equal(a, b)
    os.environ["SWB200_ADJ_STORE"] = "0"       # every state kept, steps recomputed instead of stored
    try:
        J0, g0, _, bad0 = host_check_gradient(host_check_lib, S, Prog, obs, n, n)
    finally:
        del os.environ["SWB200_ADJ_STORE"]
    assert bad0 == 0 and J0 == J
    for a, b in zip(g0, g):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("opts", OPTIONS)
def test_adjoint_forward_is_the_time_loop(T, opts):
    """The states the adjoint differentiates are the time loop's, bit for bit."""
    S, Prog, obs, _ = setup(T=T, nx=48, **opts)
    n = 25
    r = gradient(S, Prog, obs, n)
    ref = _production_eta(S, Prog, n)
    assert np.array_equal(r.eta_final.view(np.uint8), np.ascontiguousarray(ref, dtype=T).view(np.uint8))
    e = r.eta_final[1:-1, 1:-1].astype(np.float64)
    assert r.J == pytest.approx(float(np.sum((e - obs.astype(np.float64)) ** 2)), rel=1e-12)
    assert r.stats.adjoint_steps == n


@pytest.mark.gpu
@pytest.mark.parametrize("opts", OPTIONS)
def test_gradient_matches_dual_directional_derivative(opts):
    """<gradient, direction> against the Dual-number oracle at 128 x 64."""
    S, Prog, obs, rng = setup(nx=128, seed=11, **opts)
    n = 60
    du, dv, de, dF = direction(S, Prog, rng)
    r = gradient(S, Prog, obs, n)
    J, dJ = oracle.jvp(S, Prog, obs, n, du=du, dv=dv, deta=de, dFx=dF)
    assert r.J == pytest.approx(J, rel=1e-12)
    g = (r.u, r.v, r.eta, r.Fx)
    assert directional(g, (du, dv, de, dF)) == pytest.approx(dJ, rel=DUAL_RTOL)
    for d in ((du, None, None, None), (None, dv, None, None), (None, None, de, None), (None, None, None, dF)):
        _, dJk = oracle.jvp(S, Prog, obs, n, du=d[0], dv=d[1], deta=d[2], dFx=d[3])
        assert directional(g, d) == pytest.approx(dJk, rel=DUAL_RTOL)


@pytest.mark.gpu
def test_float32_gradient_agrees_with_float64():
    """The Float32 adjoint of the same problem gives the Float64 directional
    derivative to about the precision of the Float32 forward run."""
    n = 40
    r64, r32 = [gradient(*setup(T=T, nx=64, seed=13)[:3], n) for T in (np.float64, np.float32)]
    rng = np.random.default_rng(2)
    S, Prog, _, _ = setup(nx=64, seed=13)
    du, dv, de, dF = direction(S, Prog, rng)
    d64 = directional((r64.u, r64.v, r64.eta, r64.Fx), (du, dv, de, dF))
    d32 = directional(tuple(np.asarray(x, np.float64) for x in (r32.u, r32.v, r32.eta, r32.Fx)), (du, dv, de, dF))
    assert d32 == pytest.approx(d64, rel=1e-3)
    assert r32.J == pytest.approx(r64.J, rel=1e-3)


@pytest.mark.gpu
def test_checkpoint_schedule_does_not_change_the_gradient(monkeypatch):
    S, Prog, obs, _ = setup(nx=64, seed=5)
    n = 37
    full = gradient(S, Prog, obs, n)
    assert full.stats.forward_steps == n and full.stats.stored_stage_states == 1
    monkeypatch.setenv("SWB200_ADJ_STORE", "0")
    rec = gradient(S, Prog, obs, n)
    monkeypatch.delenv("SWB200_ADJ_STORE")
    assert rec.stats.stored_stage_states == 0 and rec.J == full.J
    for a, b in ((rec.u, full.u), (rec.v, full.v), (rec.eta, full.eta), (rec.Fx, full.Fx)):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())
    # two-level schedule (state slots per segment, stage inputs kept per
    # segment: each step recomputed once), with the recomputation overlapped
    # with the reverse steps (default) or after them, and the binomial one
    for schedule in ("segments", "segments_in_turn", "binomial"):
        if schedule == "segments_in_turn":
            monkeypatch.setenv("SWB200_ADJ_OVERLAP", "0")
        if schedule == "binomial":
            monkeypatch.delenv("SWB200_ADJ_OVERLAP")
            monkeypatch.setenv("SWB200_ADJ_SCHEDULE", "binomial")
        for nc in (6, 2, 1):
            r = gradient(S, Prog, obs, n, ncheckpoints=nc)
            assert r.J == full.J
            assert r.stats.checkpoints == nc and r.stats.forward_steps > n
            if schedule == "segments":
                assert r.stats.stored_stage_states == 3 and r.stats.forward_steps == 2 * n
            elif schedule == "segments_in_turn":
                assert r.stats.stored_stage_states == 2 and r.stats.forward_steps == 2 * n
            else:
                assert r.stats.stored_stage_states == 0
            for a, b in ((r.u, full.u), (r.v, full.v), (r.eta, full.eta), (r.Fx, full.Fx)):
                np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())
    monkeypatch.delenv("SWB200_ADJ_SCHEDULE")


@pytest.mark.gpu
def test_twin_gradient_matches_finite_differences():
    """The 512 x 256 twin experiment: the gradient along the true forcing error
    dFx and along an eta perturbation matches central differences of the GPU
    forward (eps = 1e-3 of the perturbation)."""
    n = 300
    S, Prog, obs, dFx = twin(nx=512, nsteps=n)
    r = gradient(S, Prog, obs, n, ncheckpoints=40)
    u, v, e, sst = Prog
    rng = np.random.default_rng(9)
    de = np.zeros_like(e)
    de[1:-1, 1:-1] = rng.normal(0, 1e-3, de[1:-1, 1:-1].shape)

    def J_at(SS, PP):
        eta = _production_eta(SS, PP, n)[1:-1, 1:-1]
        return float(np.sum((eta - obs) ** 2))

    eps = 1e-3
    fd_F = (J_at(with_Fx(S, S.forcing.Fx + eps * dFx), Prog) - J_at(with_Fx(S, S.forcing.Fx - eps * dFx), Prog)) / (2 * eps)
    assert float(np.sum(r.Fx * dFx)) == pytest.approx(fd_F, rel=1e-4)
    fd_e = (J_at(S, PrognosticVars(u, v, e + eps * de, sst)) - J_at(S, PrognosticVars(u, v, e - eps * de, sst))) / (2 * eps)
    assert float(np.sum(r.eta * de)) == pytest.approx(fd_e, rel=1e-4)
    assert r.J > 0 and float(np.sum(r.Fx * dFx)) < 0     # moving towards Fx_obs lowers the misfit
