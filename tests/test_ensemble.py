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
