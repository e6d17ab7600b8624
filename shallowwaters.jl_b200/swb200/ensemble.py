"""Ensembles of independent model runs, sharded over GPUs.

Members share nothing: each is a full run_model (its own grid, forcing, time
step and step count).  Members are therefore dealt out whole, with no data
exchange during the run.

* Across GPUs: one process per GPU (torch.distributed).  Every rank computes
  the same greedy longest-first assignment of members by their cost
  nx*ny*nt and runs its own share.  A single FP64 all-reduce of the
  per-member diagnostics table (mass, energy, max speed, NaN count, steps) at
  the end is the only collective.
* On one GPU, either as a batch (``run_batched``, sw_batch_*): one kernel
  launch per sub-step advances every member that shares the boundary type and
  options, so many small grids fill the GPU together; or several members at
  once, each a libswb200 context with its own CUDA stream driven from its own
  host thread (``run_local``; the library call releases the GIL).

``c4_members`` builds the seeded ensemble of uneven sizes used for
measurements: nx in {64, 96, 128, 192, 256}, L_ratio in {1, 2}, bc alternating
periodic / nonperiodic free-slip, Fx0 ~ U(0.05, 0.2) Pa and seeded eta noise
sigma = 0.01 m per member.
"""
from __future__ import annotations

import concurrent.futures as cf
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

COLUMNS = ("mass", "energy", "max_speed", "nan_count", "steps", "cells")


@dataclass
class Member:
    """One ensemble member: Parameter keyword arguments and its noise seed."""
    index: int
    kwargs: Dict = field(default_factory=dict)
    seed: int = 0


def c4_members(n: int = 256, seed: int = 2024, Ndays: float = 30.0, **extra) -> List[Member]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(rng.choice([64, 96, 128, 192, 256]))
        L_ratio = int(rng.choice([1, 2]))
        kw = dict(nx=nx, L_ratio=L_ratio, Ndays=Ndays, Fx0=float(rng.uniform(0.05, 0.2)),
                  bc="periodic" if k % 2 == 0 else "nonperiodic", α=0.0)
        kw.update(extra)
        out.append(Member(k, kw, int(rng.integers(0, 2**31 - 1))))
    return out


def member_setup(m: Member):
    """Parameter, ModelSetup and the seeded initial state of a member."""
    from . import Parameter, initial_conditions, model_setup
    P = Parameter(**m.kwargs)
    S = model_setup(P)
    rng = np.random.default_rng(m.seed)
    η0 = rng.normal(0.0, 0.01, size=(S.grid.ny, S.grid.nx))
    return P, S, initial_conditions(P.Tprog, S, η0=η0)


def member_cost(m: Member) -> int:
    """nx * ny * nt: the member's cell updates."""
    from . import Parameter, model_setup
    S = model_setup(Parameter(**m.kwargs))
    return S.grid.nx * S.grid.ny * S.grid.nt


def partition(costs: List[int], nranks: int) -> List[List[int]]:
    """Greedy longest-processing-time assignment: members by decreasing cost,
    each to the least loaded rank (lowest rank on ties).  Deterministic, so
    every rank derives the same assignment without communicating."""
    load = [0] * nranks
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def run_member(m: Member, storage: str = "native") -> np.ndarray:
    """Run one member to its end on the current GPU; returns its row of COLUMNS."""
    from .model import Model
    P, S, Prog = member_setup(m)
    with Model(S, storage=storage) as model:
        model.set_state(Prog)
        st = model.run(S.grid.nt)
        d = model.diagnostics()
    return np.array([d.mass, d.energy, d.max_speed, d.nan_count, st.steps_done, S.grid.nx * S.grid.ny],
                    dtype=np.float64)


def _batch_create(members: List[Member], lib, storage: str = "native"):
    """Host set-up of the members and the batch (sw_batch_create + states)."""
    import ctypes as C
    from . import abi
    setups = [member_setup(m) for m in members]
    cfgs = (abi.SwConfig * len(members))(*[abi.make_config(S, storage=storage) for _, S, _ in setups])
    statics = [abi.StaticFields(S) for _, S, _ in setups]
    sts = (abi.SwStatic * len(members))(*[st.struct for st in statics])
    b = C.c_void_p()
    abi.check(lib, lib.sw_batch_create(len(members), cfgs, sts, C.byref(b)))
    try:
        states = []
        for k, (P, S, Prog) in enumerate(setups):
            arrs = [np.ascontiguousarray(a, dtype=P.Tprog) for a in Prog]
            states.append(arrs)
            abi.check(lib, lib.sw_batch_set_state(b, k, *abi.state_ptrs(*arrs)))
    except Exception:
        lib.sw_batch_destroy(b)
        raise
    return b, setups, states


def _batch_run(lib, b, members, setups, states, return_states):
    """Runs a created batch to its end, collects each member's row (and state)
    and destroys it.  Returns (rows, states, info)."""
    import ctypes as C
    from . import abi
    from .initial_conditions import remove_halo
    try:
        status = (abi.SwStatus * len(members))()
        t0 = time.perf_counter()
        rc = lib.sw_batch_run(b, 1 << 62, status)
        run_seconds = time.perf_counter() - t0
        if rc not in (abi.SW_OK, abi.SW_NAN_DETECTED):
            abi.check(lib, rc)
        info = {"tile_rows": int(lib.sw_batch_tile_rows(b)), "launches": int(lib.sw_batch_launches(b)),
                "run_seconds": run_seconds}
        out, fin = {}, {}
        for k, (m, (P, S, _)) in enumerate(zip(members, setups)):
            d = abi.SwDiag()
            abi.check(lib, lib.sw_diagnostics(lib.sw_batch_member(b, k), C.byref(d)))
            out[m.index] = np.array([d.mass, d.energy, d.max_speed, d.nan_count, status[k].steps_done,
                                     S.grid.nx * S.grid.ny], dtype=np.float64)
            if return_states:
                arrs = [np.empty_like(a) for a in states[k]]
                abi.check(lib, lib.sw_batch_get_state(b, k, *abi.state_ptrs(*arrs)))
                fin[m.index] = remove_halo(*arrs, S)
    finally:
        lib.sw_batch_destroy(b)
    return out, fin, info


def run_batched(members: List[Member], lib=None, return_states: bool = False, info: Optional[dict] = None,
                chunks: int = 1, storage: str = "native"):
    """Run members as batches (sw_batch_*): one launch per sub-step for all
    members of a batch sharing the boundary type and options.  Returns
    {index: row of COLUMNS} (and the final states without halo when
    ``return_states``).  ``storage`` ("native", "bf16", "f16") is the state
    storage of every member (the 16-bit form keeps every array of the time
    loop in 16 bits; Float32 members only).

    ``chunks`` > 1 splits the members (round robin by decreasing cost) into
    that many batches and pipelines them: while a batch runs on a worker
    thread (the library call releases the GIL), the next one is set up on the
    host, and the batches' steps overlap on the GPU.  ``info``, if given,
    receives the tile heights ("tile_rows", "chunk_tile_rows"), kernel
    launches ("launches") and, for one batch, the seconds of the sw_batch_run
    call ("run_seconds": the steps only, without member set-up and uploads)."""
    from . import abi
    lib = lib or abi.load_library()
    if chunks <= 1 or len(members) < 2 * chunks:
        b, setups, states = _batch_create(members, lib, storage)
        out, fin, inf = _batch_run(lib, b, members, setups, states, return_states)
        if info is not None:
            info.update(inf)
            info["chunk_tile_rows"] = [inf["tile_rows"]]
        return (out, fin) if return_states else out
    order = sorted(members, key=lambda m: -(m.kwargs.get("nx", 0) ** 2))
    groups = [order[k::chunks] for k in range(chunks)]
    futs = []
    with cf.ThreadPoolExecutor(max_workers=chunks) as ex:
        try:
            for grp in groups:
                b, setups, states = _batch_create(grp, lib, storage)
                futs.append(ex.submit(_batch_run, lib, b, grp, setups, states, return_states))
        finally:
            results = [f.result() for f in futs]
    out, fin = {}, {}
    for o, f, _ in results:
        out.update(o)
        fin.update(f)
    if info is not None:
        infos = [r[2] for r in results]
        info["tile_rows"] = infos[0]["tile_rows"]
        info["chunk_tile_rows"] = [x["tile_rows"] for x in infos]
        info["launches"] = sum(x["launches"] for x in infos)
        info["run_seconds"] = None
    return (out, fin) if return_states else out


def run_local(members: List[Member], threads: int = 8,
              runner: Callable[[Member], np.ndarray] = run_member) -> Dict[int, np.ndarray]:
    """Run members on this process's GPU, ``threads`` at a time."""
    if threads <= 1:
        return {m.index: runner(m) for m in members}
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        futs = {m.index: ex.submit(runner, m) for m in members}
        return {k: f.result() for k, f in futs.items()}


def run_ensemble(members: List[Member], *, threads: int = 8, costs: Optional[List[int]] = None,
                 runner: Callable[[Member], np.ndarray] = run_member, batched: bool = False,
                 info: Optional[dict] = None, chunks: int = 1, storage: str = "native"):
    """Run an ensemble over all ranks of the default process group (or alone).

    Returns ``(table, seconds)``: the (len(members), len(COLUMNS)) FP64 table of
    every member's diagnostics, identical on all ranks, and this rank's time.
    ``storage`` is the state storage of batched members (run_batched).
    """
    import torch
    import torch.distributed as dist
    dist_on = dist.is_available() and dist.is_initialized()
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist_on else (0, 1)
    if costs is None:
        costs = [member_cost(m) for m in members]
    mine = [members[i] for i in partition(costs, world)[rank]]
    t0 = time.perf_counter()
    if batched and mine:
        local = run_batched(mine, info=info, chunks=chunks, storage=storage)
    else:
        local = run_local(mine, threads, runner)
    seconds = time.perf_counter() - t0
    table = np.zeros((len(members), len(COLUMNS)), dtype=np.float64)
    pos = {m.index: k for k, m in enumerate(members)}
    for idx, row in local.items():
        table[pos[idx]] = row
    if dist_on and world > 1:
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.from_numpy(table).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)      # each row is non-zero on exactly one rank
        table = t.cpu().numpy()
    return table, seconds
