"""The fast build (libswb200_fast.so) against the oracle, to a stated tolerance.

The fast build compiles the same kernels with FMA contraction, so a*b+c is
rounded once instead of twice.  Results then differ from the reference's
Float32 (and Float64) arithmetic by rounding, and the comparison is normwise:

    max |gpu - oracle| <= TOL * max |oracle|     for u, v, η and sst,

with TOL = 1e-5 for Float32 and 1e-12 for Float64 after one step (the
tolerance the drop-in promises), and a looser 1e-4 (Float32) after 20 steps,
where rounding differences have been carried through the nonlinear terms.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import seeded_inputs
from swb200 import Model, Parameter, initial_conditions, model_setup

pytestmark = pytest.mark.gpu

TOL_ONE_STEP = {np.float32: 1e-5, np.float64: 1e-12}
TOL_20_STEPS = {np.float32: 1e-4, np.float64: 1e-10}

CASES = {
    "channel_smag": dict(nx=64, diffusion="Smagorinsky"),
    "nonperiodic_seamount_gyre": dict(nx=64, L_ratio=1, bc="nonperiodic", α=0, topography="seamount",
                                      wind_forcing_x="double_gyre"),
    "partial_slip_linear_drag": dict(nx=48, bc="nonperiodic", α=0.5, bottom_drag="linear"),
    "ssprk2": dict(nx=64, time_scheme="SSPRK2", RKs=3, cfl=1.2),
    "4ssprk3_sadourny": dict(nx=64, time_scheme="4SSPRK3", adv_scheme="Sadourny"),
    "float64_smag": dict(nx=64, T=np.float64, diffusion="Smagorinsky"),
    "tracer_every_30": dict(nx=64, Uadv=2.0),
}


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run_both(kw, steps, seed=31):
    P = Parameter(Uadv=kw.pop("Uadv", 1000), Ndays=1, **kw)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, seed))
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(S)
    o.set_state(Prog)
    m = Model(S, build="fast")
    m.set_state(Prog)
    out, done = {}, 0
    for n in steps:
        assert o.run(n - done).code == 0 and m.run(n - done).code == 0
        done = n
        out[n] = {name: relerr(y, x) for x, y, name in zip(o.get_state(), m.get_state(), ("u", "v", "η", "sst"))}
    m.close()
    return P.T, out


@pytest.mark.parametrize("name", list(CASES))
def test_fast_build_within_tolerance(name):
    T, errs = run_both(dict(CASES[name]), [1, 20])
    print(name, errs)
    for field, e in errs[1].items():
        assert e <= TOL_ONE_STEP[T], f"{field} after 1 step: {e:.3e} > {TOL_ONE_STEP[T]:.0e}"
    for field, e in errs[20].items():
        assert e <= TOL_20_STEPS[T], f"{field} after 20 steps: {e:.3e} > {TOL_20_STEPS[T]:.0e}"


def test_fast_build_headline_channel_one_step():
    """The benchmark workload (2048 x 1024 channel) after one step."""
    from swb200.precision import channel_params, channel_state
    kw, rng = channel_params(2048)
    P = Parameter(**kw)
    S = model_setup(P)
    Prog = channel_state(S, rng)
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(S)
    o.set_state(Prog)
    m = Model(S, build="fast")
    m.set_state(Prog)
    assert o.run(1).code == 0 and m.run(1).code == 0
    errs = {name: relerr(y, x) for x, y, name in zip(o.get_state(), m.get_state(), ("u", "v", "η", "sst"))}
    print("headline", errs)
    for field, e in errs.items():
        assert e <= TOL_ONE_STEP[np.float32], f"{field}: {e:.3e}"
    m.close()
