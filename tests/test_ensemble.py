"""Ensemble sharding: the member assignment, the cross-rank gather (gloo,
world size 2, on CPU) and, on the GPU, concurrent members equal lone runs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from swb200.ensemble import COLUMNS, Member, c4_members, partition, run_ensemble, run_local


def test_c4_members_are_seeded_and_uneven():
    a, b = c4_members(16, seed=7), c4_members(16, seed=7)
    assert [m.kwargs for m in a] == [m.kwargs for m in b] and [m.seed for m in a] == [m.seed for m in b]
    assert {m.kwargs["nx"] for m in c4_members(64)} <= {64, 96, 128, 192, 256}
    assert [m.kwargs["bc"] for m in a[:4]] == ["periodic", "nonperiodic"] * 2
    assert all(0.05 <= m.kwargs["Fx0"] <= 0.2 for m in a)


@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_partition_covers_each_member_once_and_balances(nranks):
    rng = np.random.default_rng(nranks)
    costs = [int(c) for c in rng.integers(1, 1000, size=37)]
    parts = partition(costs, nranks)
    assert sorted(i for p in parts for i in p) == list(range(37))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)          # LPT bound
    assert parts == partition(costs, nranks)               # every rank derives the same split


def _fake_runner(m: Member):
    # a deterministic stand-in for a GPU run: a row that identifies the member
    return np.array([m.index * 1.5, m.seed % 97, m.kwargs["nx"], 0, 10 + m.index, m.kwargs["nx"] ** 2], float)


def _gloo_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        members = c4_members(11, seed=3)
        costs = [m.kwargs["nx"] ** 2 for m in members]
        table, _ = run_ensemble(members, threads=2, costs=costs, runner=_fake_runner)
        np.save(os.path.join(out, f"rank{rank}.npy"), table)
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_equals_one_process(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_gloo_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    members = c4_members(11, seed=3)
    ref = np.array([_fake_runner(m) for m in members])
    for r in range(2):
        np.testing.assert_array_equal(np.load(os.path.join(tmp_path, f"rank{r}.npy")), ref)
    assert ref.shape == (11, len(COLUMNS))


@pytest.mark.gpu
def test_concurrent_members_equal_lone_runs():
    """Members run four at a time (one context and stream each) give the same
    results, bit for bit, as the same members run one after another."""
    members = [Member(k, dict(nx=[24, 32, 40][k % 3], L_ratio=1 + k % 2, Ndays=0.3,
                              bc="periodic" if k % 2 else "nonperiodic", α=0.0,
                              Fx0=0.05 + 0.02 * k), seed=100 + k) for k in range(8)]
    together = run_local(members, threads=4)
    alone = run_local(members, threads=1)
    for k in range(8):
        np.testing.assert_array_equal(together[k], alone[k])
        assert together[k][COLUMNS.index("nan_count")] == 0


def _batch_members():
    return [
        Member(0, dict(nx=24, Ndays=0.3, Uadv=1000), seed=1),
        Member(1, dict(nx=40, L_ratio=1, Ndays=0.2, bc="nonperiodic", α=0.0, topography="seamount"), seed=2),
        Member(2, dict(nx=64, Ndays=0.25, Uadv=1000, diffusion="Smagorinsky"), seed=3),
        Member(3, dict(nx=30, Ndays=0.4, Uadv=1000, bc="nonperiodic", α=0.5), seed=4),
        Member(4, dict(nx=32, Ndays=0.5, Uadv=2.0), seed=5),                      # tracer every few steps
        Member(5, dict(nx=36, Ndays=0.5, Uadv=2.5, tracer_consumption=True), seed=6),
        Member(6, dict(nx=28, Ndays=0.3, Uadv=1000, adv_scheme="Sadourny", surface_relax=True), seed=7),
    ]


def _lone_states(members, storage="native"):
    from swb200.ensemble import member_setup
    from swb200 import Model
    from swb200.initial_conditions import remove_halo
    out = {}
    for m in members:
        P, S, Prog = member_setup(m)
        with Model(S, storage=storage) as model:
            model.set_state(Prog)
            st = model.run(S.grid.nt)
            out[m.index] = (remove_halo(*model.get_state(), S), st.steps_done, S.grid.nt)
    return out


@pytest.mark.gpu
def test_pipelined_batches_equal_lone_runs():
    """Members split into two batches that run on worker threads while the
    next is set up end where each member ends alone, bit for bit."""
    from swb200.ensemble import run_batched
    members = _batch_members()
    info = {}
    table, states = run_batched(members, return_states=True, info=info, chunks=2)
    assert len(info["chunk_tile_rows"]) == 2
    for k, (ref, done, nt) in _lone_states(members).items():
        assert table[k][COLUMNS.index("steps")] == done == nt
        for x, y in zip(states[k], ref):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("rows", ["4", "8", "16", "32", "tuned"])
def test_every_batch_tile_height_equals_lone_runs(rows, monkeypatch):
    """The autotuner's candidates (forced with SWB200_BATCH_TY) and its own
    choice all give the lone runs' results bit for bit."""
    from swb200.ensemble import run_batched
    if rows != "tuned":
        monkeypatch.setenv("SWB200_BATCH_TY", rows)
    else:
        monkeypatch.delenv("SWB200_BATCH_TY", raising=False)
    members = _batch_members()[:4]
    info = {}
    table, states = run_batched(members, return_states=True, info=info)
    if rows == "tuned":
        assert info["tile_rows"] in (4, 8, 16, 32)
    else:
        assert info["tile_rows"] == int(rows)
    for k, (ref, done, nt) in _lone_states(members).items():
        assert table[k][COLUMNS.index("steps")] == done == nt
        for x, y in zip(states[k], ref):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.gpu
def test_batched_members_equal_lone_runs():
    """sw_batch_*: members of different sizes, boundaries and tracer schedules,
    advanced with one launch per sub-step, end bit for bit where each ends alone
    (including members that finish earlier than others)."""
    from swb200.ensemble import member_setup, run_batched
    from swb200 import Model
    from swb200.initial_conditions import remove_halo
    members = [
        Member(0, dict(nx=24, Ndays=0.3, Uadv=1000), seed=1),
        Member(1, dict(nx=40, L_ratio=1, Ndays=0.2, bc="nonperiodic", α=0.0, topography="seamount"), seed=2),
        Member(2, dict(nx=64, Ndays=0.25, Uadv=1000, diffusion="Smagorinsky"), seed=3),
        Member(3, dict(nx=30, Ndays=0.4, Uadv=1000, bc="nonperiodic", α=0.5), seed=4),
        Member(4, dict(nx=32, Ndays=0.5, Uadv=2.0), seed=5),                      # tracer every few steps
        Member(5, dict(nx=36, Ndays=0.5, Uadv=2.5, tracer_consumption=True), seed=6),
        Member(6, dict(nx=28, Ndays=0.3, Uadv=1000, adv_scheme="Sadourny", surface_relax=True), seed=7),
    ]
    table, states = run_batched(members, return_states=True)
    for m in members:
        P, S, Prog = member_setup(m)
        with Model(S) as model:
            model.set_state(Prog)
            st = model.run(S.grid.nt)
            ref = remove_halo(*model.get_state(), S)
        assert table[m.index][COLUMNS.index("steps")] == st.steps_done == S.grid.nt
        for x, y, name in zip(states[m.index], ref, ("u", "v", "η", "sst")):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"member {m.index}: {name}"


@pytest.mark.gpu
@pytest.mark.parametrize("storage,rows", [("bf16", "8"), ("bf16", "tuned"), ("f16", "16"), ("f16", "tuned")])
def test_batched_16bit_members_equal_lone_runs(storage, rows, monkeypatch):
    """Members in the 16-bit storage form, batched (one launch per sub-step
    for all of them), end bit for bit where each ends alone in that form:
    periodic and nonperiodic members, Smagorinsky, topography, tracers every
    step and every few steps, tracer consumption, members finishing early."""
    from swb200.ensemble import run_batched
    if rows != "tuned":
        monkeypatch.setenv("SWB200_BATCH_TY", rows)
    else:
        monkeypatch.delenv("SWB200_BATCH_TY", raising=False)
    members = [m for m in _batch_members() if "adv_scheme" not in m.kwargs]
    info = {}
    table, states = run_batched(members, return_states=True, info=info, storage=storage)
    if rows != "tuned":
        assert info["tile_rows"] == int(rows)
    for k, (ref, done, nt) in _lone_states(members, storage).items():
        assert table[k][COLUMNS.index("steps")] == done == nt
        assert table[k][COLUMNS.index("nan_count")] == 0
        for x, y, name in zip(states[k], ref, ("u", "v", "η", "sst")):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"member {k}: {name}"
