"""The CPU oracle: the reference's own tests, and a second restatement.

The reference's test/runtests.jl holds one known-answer test (zero forcing
gives exactly zero fields) and stability bounds for seven option sets; they
are run here against the C++ restatement (oracle/sw_oracle.hpp).  The oracle
is further checked bit for bit against an independent numpy restatement
(oracle/numpy_port.py) over the option space.
"""
import numpy as np
import pytest

import numpy_port as NP
import oracle as O
from conftest import assert_bitwise, seeded_inputs
from swb200 import Parameter, initial_conditions, model_setup


# ------------------------------------------------ test/runtests.jl, verbatim options
def test_no_forcing():                                   # test/runtests.jl:4-9
    prog, st = O.run_model(Ndays=1, Fx0=0)
    assert st.code == 0 and st.steps_done == 307
    assert np.all(prog.u == 0) and np.all(prog.v == 0) and np.all(prog.η == 0)


@pytest.mark.parametrize("kw", [dict(bc="periodic"), dict(bc="nonperiodic"), dict(α=0)])
def test_boundary_conditions(kw):                        # test/runtests.jl:11-20
    prog, st = O.run_model(Ndays=1, **kw)
    assert st.code == 0
    assert np.all(np.abs(prog.η) < 10)


@pytest.mark.parametrize("kw", [dict(surface_relax=True), dict(surface_forcing=True)])
def test_continuity_forcing(kw):                         # test/runtests.jl:22-30
    prog, st = O.run_model(Ndays=1, **kw)
    assert np.all(np.abs(prog.η) < 10)
    assert np.all(prog.u != 0)


@pytest.mark.parametrize("T,Tprog", [(np.float32, np.float64), (np.float16, np.float32)])
def test_mixed_precision(T, Tprog):                      # test/runtests.jl:32-40
    prog, st = O.run_model(T, Tprog=Tprog, Ndays=1)
    assert prog.u.dtype == Tprog
    assert np.all(np.abs(prog.η) < 10)
    assert np.all(prog.u != 0)


def test_rk3():                                          # test/runtests.jl:42-46
    prog, st = O.run_model(time_scheme="RK", RKo=3, cfl=0.6, nstep_advcor=0)
    assert np.all(np.abs(prog.η) < 10)
    assert np.all(prog.u != 0)


@pytest.mark.parametrize("RKs,cfl,advcor", [(2, 0.7, 1), (3, 1.2, 1), (4, 1.4, 1),
                                            (2, 0.7, 0), (3, 1.2, 0), (4, 1.4, 0)])
def test_ssprk2(RKs, cfl, advcor):                       # test/runtests.jl:48-72
    prog, st = O.run_model(time_scheme="SSPRK2", RKs=RKs, cfl=cfl, nstep_advcor=advcor)
    assert np.all(np.abs(prog.η) < 10)
    assert np.all(prog.u != 0)


@pytest.mark.parametrize("RKn,cfl", [(2, 1.2), (3, 2.5)])
def test_ssprk3(RKn, cfl):                               # test/runtests.jl:74-82
    prog, st = O.run_model(time_scheme="SSPRK3", RKn=RKn, cfl=cfl, nstep_advcor=1)
    assert np.all(np.abs(prog.η) < 10)
    assert np.all(prog.u != 0)


# ------------------------------------------------ C++ oracle == numpy restatement
CASES = {
    "per_rk4_const": dict(),
    "per_rk4_smag": dict(diffusion="Smagorinsky"),
    "nonper_rk4": dict(bc="nonperiodic"),
    "nonper_seamount_dg": dict(bc="nonperiodic", topography="seamount", wind_forcing_x="double_gyre", α=0),
    "per_seamount_smag": dict(topography="seamount", diffusion="Smagorinsky"),
    "per_ridges_lin": dict(topography="ridges", bottom_drag="linear"),
    "nodrag_partialslip": dict(bottom_drag="none", α=0.5, bc="nonperiodic"),
    "sadourny": dict(adv_scheme="Sadourny"),
    "sadourny_np": dict(adv_scheme="Sadourny", bc="nonperiodic"),
    "rk3": dict(RKo=3, cfl=0.6),
    "rk2": dict(RKo=2, cfl=0.3),
    "ssprk2": dict(time_scheme="SSPRK2", RKs=3, cfl=1.2, nstep_advcor=1),
    "ssprk2_0": dict(time_scheme="SSPRK2", RKs=2, cfl=0.7),
    "ssprk3": dict(time_scheme="SSPRK3", RKn=2, cfl=1.2, nstep_advcor=1),
    "ssprk3n3_np": dict(time_scheme="SSPRK3", RKn=3, cfl=2.5, nstep_advcor=1, bc="nonperiodic"),
    "4ssprk3": dict(time_scheme="4SSPRK3", cfl=1.0),
    "relax": dict(surface_relax=True),
    "pump_np": dict(surface_forcing=True, bc="nonperiodic"),
    "seasonal": dict(seasonal_wind_x=True, wind_forcing_y="channel", Fy0=0.05, seasonal_wind_y=True),
    "fy_channel_np": dict(wind_forcing_y="channel", Fy0=0.05, bc="nonperiodic"),
    "linear": dict(dynamics="linear"),
    "linear_ssprk2": dict(dynamics="linear", time_scheme="SSPRK2", cfl=0.7),
    "consumption": dict(tracer_consumption=True),
    "uadv_default": dict(Uadv=0.25, Ndays=1),
    "uadv_30": dict(Uadv=30.0),
    "f64": dict(T=np.float64),
    "f64_np_smag": dict(T=np.float64, bc="nonperiodic", diffusion="Smagorinsky"),
    "tcomm16": dict(Tcomm=np.float16),
    "nstep_diff3": dict(nstep_diff=3),
    "advcor2": dict(nstep_advcor=2),
}


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_equals_numpy_port(name):
    kw = dict(nx=40, Ndays=0.2, Uadv=1000)
    kw.update(CASES[name])
    P = Parameter(**kw)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S))
    o = O.Oracle(S)
    o.set_state(Prog)
    st = o.run(6)
    assert st.code == 0
    a = o.get_state()
    b = NP.NumpyModel(S).run(Prog, 6)
    for x, y, nm in zip(a, b, ("u", "v", "η", "sst")):
        assert_bitwise(x, y, f"{name}:{nm}")


def test_nan_detection_stops_like_reference():
    """NaNs are looked for every nout steps in (u,v,η before the step, sst after
    it); the loop breaks before the copy-back (src/feedback.jl:134-148,
    src/time_integration.jl:235-237)."""
    P = Parameter(nx=20, Ndays=2, Uadv=1000, tracer_advection=False)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S)
    Prog.u[5, 7] = np.nan
    o = O.Oracle(S)
    o.set_state(Prog)
    st = o.run(S.grid.nt)
    assert st.code == 3
    assert st.nan_step == S.grid.nout
    assert st.steps_done == S.grid.nout
