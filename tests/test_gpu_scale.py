"""GPU parity at full size and on the tile scheduler's multi-tile path.

The TMA stage kernel runs persistent blocks that take tiles (112 columns x 8
rows) from a device counter.  On the small grids of the option table every
block takes at most one tile, so these tests cover the other path:

* the benchmark's own workload, the 2048 x 1024 periodic channel (2,432 tiles
  on at most 888 blocks), for 3 steps against the oracle, bit for bit;
* the double gyre over a seamount at 512 x 512, nonperiodic free slip, for
  3 steps, bit for bit;
* every case of the option table with the persistent blocks capped at 1 and
  at 2 (SWB200_STAGE_BLOCKS), so one block walks every tile of a launch and
  the slot ring and mbarrier phases carry across tiles.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import assert_bitwise, seeded_inputs
from swb200 import Model, Parameter, initial_conditions, model_setup

from test_gpu_parity import BASE, CASES, both

pytestmark = pytest.mark.gpu


def _compare(S, Prog, steps):
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(S)
    o.set_state(Prog)
    m = Model(S)
    m.set_state(Prog)
    done = 0
    for n in steps:
        so, sg = o.run(n - done), m.run(n - done)
        done = n
        assert so.code == sg.code == 0, (so.code, sg.code)
        for x, y, name in zip(o.get_state(), m.get_state(), ("u", "v", "η", "sst")):
            assert_bitwise(y, x, f"{name} after {n} steps")
    m.close()


def test_headline_channel_2048x1024_bitwise():
    """The benchmark workload (seeded wind amplitude, η noise and tracer
    checkerboard; RK4, Arakawa-Hsu, Smagorinsky, quadratic drag, tracer every
    step) equals the oracle after 1 and 3 steps."""
    from swb200.precision import channel_params, channel_state
    kw, rng = channel_params(2048)
    P = Parameter(**kw)
    S = model_setup(P)
    assert (S.grid.nx, S.grid.ny) == (2048, 1024)
    _compare(S, channel_state(S, rng), [1, 3])


def test_double_gyre_seamount_512x512_bitwise():
    """Nonperiodic free slip (α = 0), double-gyre wind, 50 m seamount on 500 m,
    RK4, tracer every step, at 512 x 512: equals the oracle after 1 and 3 steps."""
    P = Parameter(nx=512, L_ratio=1, bc="nonperiodic", α=0, wind_forcing_x="double_gyre", Fx0=0.12,
                  topography="seamount", topo_height=50, H=500, Uadv=1000, Ndays=100)
    S = model_setup(P)
    Prog = initial_conditions(P.Tprog, S, **seeded_inputs(S, 22))
    _compare(S, Prog, [1, 3])


def test_channel_100x50_ten_days_bitwise():
    """The 100 x 50 periodic channel (Fx0 = 0.12 Pa, Smagorinsky, quadratic
    drag, tracer every step) for its full 10 days, 3064 steps: equal to the
    Float32 oracle at day 1, 5 and 10."""
    from swb200.precision import channel_state, workload_params
    kw, rng = workload_params("c1", days=10)
    S = model_setup(Parameter(**kw))
    assert S.grid.nt == 3064
    _compare(S, channel_state(S, rng), [307, 1532, 3064])


@pytest.mark.parametrize("blocks", ["1", "2"])
@pytest.mark.parametrize("name", list(CASES))
def test_option_table_with_capped_stage_blocks(name, blocks, monkeypatch):
    """The option table's cases with at most `blocks` persistent blocks in the
    TMA stage kernel: still bit for bit the oracle's results."""
    monkeypatch.setenv("SWB200_TMA", "1")      # the TMA stage kernel at these sizes too
    monkeypatch.setenv("SWB200_STAGE_BLOCKS", blocks)
    kw = dict(BASE)
    kw.update(CASES[name])
    both(kw, 0, checkpoints=[1, 2, 7])
