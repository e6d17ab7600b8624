"""The 16-bit storage form (storage="bf16" or "f16") on the GPU.

Every array the time loop keeps in HBM holds scaled 16-bit numbers: the state
as compensated pairs hi + lo, the RK stage values and the accumulated
increment as single 16-bit numbers, the tracer as one 16-bit number.  Its
arithmetic is FP32, so it is not bit-identical with any reference run; these
tests check:

* set_state / get_state: the stored state is exactly the pair rounding of the
  uploaded state after the ghost rules (a numpy emulation of the rounding);
* one step: the change of u, v, η over the step agrees with the Float32
  oracle's change to the precision of the 16-bit format the tendencies are
  computed from;
* many steps: the state stays close to the Float32 oracle's;
* the run is deterministic and its graph replay equals direct launches;
* options the form is not built for are refused with SW_ERR_UNSUPPORTED.
"""
import numpy as np
import pytest

import oracle as O
from conftest import assert_bitwise, seeded_inputs
from swb200 import Model, Parameter, abi, initial_conditions, model_setup
from swb200.initial_conditions import remove_halo

pytestmark = pytest.mark.gpu

SCALE = 1024.0
# normwise bound on the one-step change of u, v, η: max|Δ16 - Δ32| / max|Δ32|
STEP_TOL = {"bf16": 3e-2, "f16": 4e-3}
# RMSE / std of the state against Float32 after 100 steps from rest: the
# velocities are still small and shaped by the noise in η, so their relative
# difference is largest (measured: v 3.4e-2 for bf16, 4.3e-3 for f16)
RUN_TOL = {"bf16": 1e-1, "f16": 1.5e-2}


def _r16(x, form):
    """float32 -> nearest 16-bit value (ties to even), back as float32."""
    x = np.asarray(x, np.float32)
    if form == "f16":
        return x.astype(np.float16).astype(np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32)


def _pair(x, s, form):
    """The value a compensated pair holds: (round16(s x) + round16(s x - hi)) / s."""
    y = np.asarray(x, np.float32) * np.float32(s)
    hi = _r16(y, form)
    lo = _r16(y - hi, form)
    return ((hi + lo) * np.float32(1.0 / s)).astype(np.float32)


def _setup(bc="periodic", **kw):
    P = Parameter(nx=64, Ndays=1, Uadv=1000, bc=bc, diffusion="Smagorinsky",
                  α=0.5 if bc == "nonperiodic" else 1.0, **kw)
    S = model_setup(P)
    return S, initial_conditions(P.Tprog, S, **seeded_inputs(S, 9))


@pytest.mark.parametrize("form,bc", [("bf16", "periodic"), ("f16", "periodic"), ("bf16", "nonperiodic")])
def test_stored_state_is_the_pair_rounding(form, bc):
    from swb200.initial_conditions import ghost_points
    S, Prog = _setup(bc)
    m = Model(S, storage=form, storage_scale_uv=SCALE)
    m.set_state(Prog)
    u, v, e = (np.array(a, np.float32) for a in (Prog.u, Prog.v, Prog.η))
    ghost_points(u, v, e, S)
    ref = [_pair(u, SCALE, form), _pair(v, SCALE, form), _pair(e, SCALE, form), _r16(Prog.sst, form)]
    for x, y, name in zip(m.get_state(), ref, ("u", "v", "η", "sst")):
        assert_bitwise(x, y, f"{name} stored at set_state ({form}, {bc})")


def _increment_errors(form, bc, steps):
    S, Prog = _setup(bc)
    o = O.Oracle(S)
    o.set_state(Prog)
    o.run(steps)
    m = Model(S, storage=form, storage_scale_uv=SCALE)
    m.set_state(Prog)
    x0 = m.get_state()
    assert m.run(steps).code == 0
    # interiors: the change of each field over the steps, in both runs
    i0, i16, i32, ip = (remove_halo(*st, S) for st in (x0, m.get_state(), o.get_state(), Prog))
    out = {}
    for k, name in enumerate(("u", "v", "η")):
        d16 = np.asarray(i16[k], np.float64) - np.asarray(i0[k], np.float64)
        d32 = np.asarray(i32[k], np.float64) - np.asarray(ip[k], np.float64)
        out[name] = float(np.max(np.abs(d16 - d32)) / np.max(np.abs(d32)))
    return out


@pytest.mark.parametrize("form,bc", [("bf16", "periodic"), ("f16", "periodic"), ("bf16", "nonperiodic"),
                                     ("f16", "nonperiodic")])
def test_one_step_change_matches_float32(form, bc):
    errs = _increment_errors(form, bc, 1)
    print(form, bc, errs)
    for name, e in errs.items():
        assert e <= STEP_TOL[form], f"{name}: {e:.3e} > {STEP_TOL[form]:.0e}"


@pytest.mark.parametrize("form", ["bf16", "f16"])
def test_hundred_steps_stay_close_to_float32(form):
    S, Prog = _setup()
    o = O.Oracle(S)
    o.set_state(Prog)
    o.run(100)
    m = Model(S, storage=form, storage_scale_uv=SCALE)
    m.set_state(Prog)
    assert m.run(100).code == 0
    for a16, a32, name in zip(m.get_state(), o.get_state(), ("u", "v", "η", "sst")):
        a16, a32 = np.asarray(a16, np.float64), np.asarray(a32, np.float64)
        rel = float(np.sqrt(np.mean((a16 - a32) ** 2)) / np.std(a32))
        print(form, name, rel)
        assert rel <= RUN_TOL[form], f"{name}: {rel:.3e}"


def test_deterministic_and_graphs_equal_direct_launches(monkeypatch):
    S, Prog = _setup(nstep_diff=2)
    out = []
    for graphs in ("1", "1", "0"):
        monkeypatch.setenv("SWB200_GRAPHS", graphs)
        m = Model(S, storage="bf16", storage_scale_uv=SCALE)
        m.set_state(Prog)
        assert m.run(13).code == 0
        out.append(m.get_state())
        m.close()
    for other in out[1:]:
        for x, y, name in zip(out[0], other, ("u", "v", "η", "sst")):
            assert_bitwise(x, y, name)


def test_diagnostics_of_the_stored_state():
    S, Prog = _setup()
    m = Model(S, storage="f16", storage_scale_uv=SCALE)
    m.set_state(Prog)
    m.run(5)
    d = m.diagnostics()
    e = np.asarray(m.get_state().η, np.float64)[1:-1, 1:-1]
    np.testing.assert_allclose(d.mass, e.sum(), rtol=1e-12, atol=1e-12)
    assert d.nan_count == 0


@pytest.mark.parametrize("kw", [dict(time_scheme="SSPRK2"), dict(dynamics="linear"), dict(adv_scheme="Sadourny"),
                                dict(nstep_advcor=2), dict(surface_relax=True)])
def test_options_outside_the_form_are_refused(kw):
    S, _ = _setup(**kw)
    with pytest.raises(abi.SwError) as e:
        Model(S, storage="bf16", storage_scale_uv=SCALE)
    assert e.value.code == abi.SW_ERR_UNSUPPORTED
