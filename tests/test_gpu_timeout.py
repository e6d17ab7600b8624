"""A bounded device wait that runs out, and the context that carries on.

Every mbarrier wait of the TMA stage kernel gives up after a number of polls,
records SW_ERR_TIMEOUT in the device status, sets the stop flag and returns,
so a lost copy can never hang the GPU.  Here the wait is made to run out on
purpose, without any fault: two test-only settings read at context creation
shorten the limit (SWB200_TEST_WAIT_LIMIT polls) and make the producer leave
one chunk of block 0's first tile unfilled (SWB200_TEST_SKIP_CHUNK), so no
copy is in flight for it and its consumers' wait cannot complete.  The run
must return SW_ERR_TIMEOUT, and a new context in the same process must then
compute the oracle's results bit for bit.
"""
import pytest

import oracle as O
from conftest import assert_bitwise, seeded_inputs
from swb200 import Model, Parameter, abi, initial_conditions, model_setup

pytestmark = pytest.mark.gpu


def _setup():
    P = Parameter(nx=256, L_ratio=2, Uadv=1000, Ndays=1, diffusion="Smagorinsky")
    S = model_setup(P)
    return S, initial_conditions(P.Tprog, S, **seeded_inputs(S, 41))


@pytest.mark.parametrize("chunk", ["0", "1"])
def test_stage_wait_runs_out_and_reports_timeout(chunk, monkeypatch):
    S, Prog = _setup()
    monkeypatch.setenv("SWB200_TMA", "1")      # the TMA stage kernel at this size too
    monkeypatch.setenv("SWB200_TEST_WAIT_LIMIT", "4096")
    monkeypatch.setenv("SWB200_TEST_SKIP_CHUNK", chunk)
    m = Model(S)
    m.set_state(Prog)
    with pytest.raises(abi.SwError) as e:
        m.run(2)
    assert e.value.code == abi.SW_ERR_TIMEOUT
    m.close()

    # the same CUDA context, a new model context: the oracle's results
    monkeypatch.delenv("SWB200_TEST_WAIT_LIMIT")
    monkeypatch.delenv("SWB200_TEST_SKIP_CHUNK")
    m = Model(S)
    m.set_state(Prog)
    assert m.run(3).code == abi.SW_OK
    o = O.Oracle(S)
    o.set_state(Prog)
    o.run(3)
    for x, y, name in zip(o.get_state(), m.get_state(), ("u", "v", "η", "sst")):
        assert_bitwise(y, x, f"{name} after the timed-out context")
    m.close()
