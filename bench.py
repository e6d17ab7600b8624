#!/usr/bin/env python
"""Benchmark: RK4 cell-updates/s of the shallow-water time loop on B200.

Workload: the periodic wind-driven channel at 2048 x 1024 cells (Δ = 976.6 m,
dtint = 13 s): flat 500 m depth, channel wind with Fx0 drawn U(0.08, 0.16) Pa
from the seed, RK4 at CFL 1, Arakawa-Hsu advection, Smagorinsky biharmonic
diffusion, quadratic drag, semi-Lagrangian tracer every step (Uadv = 1000),
seeded η noise σ = 0.01 m and a ±1 tracer checkerboard.  Plain Float32.

One "step" is one model time step (4 RK stages + tail + tracer).  ``value`` is
device time (CUDA events on the library's stream) with the state resident in
HBM and a 256 MiB L2 flush between steps (outside the timed intervals);
``e2e`` times the drop-in ``sw_time_integration`` call with pinned host
buffers, uploads and downloads included.  With N GPUs (torchrun) every rank
runs an independent replica (the single domain is not decomposed) and values
are aggregates over ranks with the time taken as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "shallowwaters.jl_b200"))

import numpy as np  # noqa: E402

METRIC = "RK4 cell-updates/s on 1 B200, plain FP32 vs chosen form at stated η error"
UNIT = "cell-updates/s"
L2_FLUSH = 256 << 20
# algorithmic bytes per cell of one RK stage launch, Float32, averaged over the
# 4 stages: stage 1 reads X, H, Fx and writes X1, X0 (44 B); stages 2-3 read
# X1, X, X0, H, Fx and write X1, X0 (68 B); stage 4 reads X1, X0, H, Fx and
# writes X0 (44 B)
STAGE_BYTES_PER_CELL = (44 + 68 + 68 + 44) / 4
STEP_BYTES_PER_CELL = 264
# the 16-bit storage form (scaled 16-bit state pairs, stage increments and
# accumulated increments; FP32 X0 after the last stage): stage 1 reads the
# state's pair and writes the stage increment and D (32 B with H, Fx), stages
# 2-3 read the pair, the increment and D and write both increments (44 B),
# stage 4 reads the pair, the increment and D and writes the FP32 X0 and eta's
# new pair (48 B); the tail reads X0 (u, v, eta) and H and writes the u, v
# pairs (24 B); the tracer reads u, v (hi) and sst and writes sst (8 B)
STAGE_BYTES_PER_CELL_16 = (32 + 44 + 44 + 48) / 4
STEP_BYTES_PER_CELL_16 = 200


def packed_static_bytes(static):
    """Bytes the library uploads for the static fields: a field constant along
    x or y (or both) is stored as one row, one column or one value."""
    total = 0
    for a in static.arrays.values():
        a = np.asarray(a)
        cx = bool(np.all(a == a[:, :1]))
        cy = bool(np.all(a == a[:1, :]))
        total += a.itemsize * (1 if cx and cy else a.shape[0] if cx else a.shape[1] if cy else a.size)
    return total


def workload_params(nx=2048, seed=1234):
    from swb200.precision import channel_params
    return channel_params(nx, seed)


def make_state(S, rng):
    from swb200.precision import channel_state
    return channel_state(S, rng)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid=None):
        self.uuid = uuid
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except Exception:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and (self.uuid is None or f[0] == self.uuid):
                self.rows.append(f)

    def wait_first(self, timeout):
        """Wait (up to timeout seconds) for the first sample."""
        t0 = time.time()
        while self.proc and not self.rows and time.time() - t0 < timeout:
            time.sleep(0.02)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.th.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(cells):
    """DRAM bytes per stage launch from the committed ncu summary, scaled to cells."""
    p = os.path.join(REPO, "profiles", "rk_stage_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d["dram_bytes_per_launch"] * cells / d["cells"]
    except Exception:
        return None


def host_info():
    model = "unknown"
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True).stdout
        for line in out.splitlines():
            if line.startswith("Model name"):
                model = line.split(":", 1)[1].strip()
    except Exception:
        pass
    return {"nproc": os.cpu_count(), "model": model}


# -------------------------------------------------------------- CPU legs
def cpu_run(S, Prog, threads, target_s, max_steps):
    """Times the oracle on the workload: returns (cell-updates/s, steps, seconds, threads)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    used = O.set_threads(threads)
    o = O.Oracle(S)
    o.set_state(Prog)
    t0 = time.perf_counter()
    o.run(1)
    t1 = time.perf_counter() - t0
    n = int(max(2, min(max_steps, math.ceil(target_s / max(t1, 1e-3)))))
    o.set_state(Prog)
    t0 = time.perf_counter()
    o.run(n)
    dt = time.perf_counter() - t0
    cells = S.grid.nx * S.grid.ny
    return cells * n / dt, n, dt, used


# --------------------------------------------------------------- main
def bench_ensemble(args, rank, world, barrier, allmax):
    """Aggregate cell-updates/s of a seeded ensemble of uneven members (nx in
    {64..256}, L_ratio 1-2, periodic / nonperiodic), sharded over the ranks and
    run as one batch per GPU (one launch per sub-step for all members).  At
    N = 1 the same members are also run ``--threads`` contexts at a time and one
    after another, for comparison.  Each rank's span is taken between device
    synchronisations; the job time is the maximum over ranks."""
    from functools import partial
    from swb200.ensemble import COLUMNS, c4_members, member_cost, run_batched, run_ensemble, run_local, run_member
    storage = {"fp32": "native", "bf16": "bf16", "f16": "f16"}[args.form]
    members = c4_members(args.members, seed=2024, Ndays=args.days)
    costs = [member_cost(m) for m in members]
    warm = c4_members(4, seed=1, Ndays=0.05)                            # module load, graphs, caches
    runner = partial(run_member, storage=storage)
    run_local(warm, threads=2, runner=runner)
    run_batched(warm, storage=storage)
    barrier()
    binfo = {}
    table, secs = run_ensemble(members, threads=args.threads, costs=costs, batched=True, info=binfo,
                               chunks=args.chunks, storage=storage)
    barrier()
    t = allmax(secs)
    value = sum(costs) / t
    threaded = seq = None
    sample = members
    vs_fp32 = None
    if world == 1:
        one = {}                                    # a single batch, for the time of its steps alone
        run_ensemble(members, costs=costs, batched=True, info=one, chunks=1, storage=storage)
        binfo["run_seconds"] = one["run_seconds"]
        if storage != "native":
            # the same members batched in Float32: each member's energy
            # against its Float32 run (relative), and its mass (the sum of
            # eta) as the difference of mean eta in metres
            ref, _ = run_ensemble(members, costs=costs, batched=True, chunks=1)
            ke, ms, nc = COLUMNS.index("energy"), COLUMNS.index("mass"), COLUMNS.index("cells")
            de = np.abs(table[:, ke] - ref[:, ke]) / np.maximum(np.abs(ref[:, ke]), 1e-30)
            dm = np.abs(table[:, ms] - ref[:, ms]) / ref[:, nc]
            vs_fp32 = {"energy_rel_median": float(np.median(de)), "energy_rel_max": float(de.max()),
                       "mean_eta_diff_max_m": float(dm.max()),
                       "mean_eta_fp32_max_m": float((np.abs(ref[:, ms]) / ref[:, nc]).max())}
        # the looped single-member runs (contexts on threads, and one after
        # another) on every member, or on every k-th member when
        # --compare-members bounds their time; their value is their own
        # cell-updates over their own time
        if 0 < args.compare_members < len(members):
            step = len(members) / args.compare_members
            sample = [members[int(k * step)] for k in range(args.compare_members)]
        scost = sum(member_cost(m) for m in sample)
        t0 = time.perf_counter()
        run_local(sample, threads=args.threads, runner=runner)
        threaded = scost / (time.perf_counter() - t0)
        t0 = time.perf_counter()
        run_local(sample, threads=1, runner=runner)
        seq = scost / (time.perf_counter() - t0)
    if rank == 0:
        print(json.dumps({
            "metric": "ensemble cell-updates/s", "value": value, "unit": UNIT, "n_gpus": world,
            "higher_is_better": True, "scaling": "strong", "dtype": "f32", "storage": args.form,
            "data": "synthetic (seeded members)",
            "config": {"workload": f"{len(members)} members, nx in {{64..256}}, L_ratio 1-2, periodic/nonperiodic, "
                                   f"{args.days} days each", "mode": "batched: one launch per sub-step for all members",
                       "cell_updates": int(sum(costs)), "parallelism": f"members sharded over {world} GPU(s)",
                       "tile_rows": binfo.get("chunk_tile_rows"), "batches": args.chunks,
                       "pipelining": "each batch runs on a worker thread while the next is set up"},
            "seconds": t, "batch_run_seconds": binfo.get("run_seconds"),
            "batch_run_value": (sum(costs) / binfo["run_seconds"]) if world == 1 and binfo.get("run_seconds") else None,
            "threaded_value": threaded, "threads": args.threads, "sequential_value": seq,
            "compared_members": len(sample), "vs_fp32_members": vs_fp32,
            "nan_members": int((table[:, COLUMNS.index("nan_count")] > 0).sum())}))
    return 0


def bench_adjoint(args):
    """Gradient of the twin experiment's eta misfit (512 x 256 periodic channel,
    RK4, Arakawa-Hsu, Smagorinsky, quadratic drag; observations from a run
    with the wind perturbed by eight seeded Fourier modes): device time of
    the adjoint's forward sweep plus reverse sweep against the time loop's own
    forward run over the same window, both on the GPU."""
    import numpy as np
    from swb200 import Model
    from swb200.adjoint import gradient, twin
    T = {"f64": np.float64, "f32": np.float32}[args.adj_dtype]
    n = args.adj_steps
    scheme = {"rk4": {}, "ssprk2": dict(time_scheme="SSPRK2", RKs=3, cfl=1.0),
              "4ssprk3": dict(time_scheme="4SSPRK3", cfl=1.0)}[args.adj_scheme]
    S, Prog, obs, dFx = twin(nx=args.adj_nx, nsteps=n, T=T, **scheme)
    nc = args.checkpoints or n
    gradient(S, Prog, obs, 4, ncheckpoints=4)                              # warm-up
    with Model(S) as m:
        m.set_state(Prog)
        m.run(4)
        m.set_state(Prog)
        fwd_ms, st = m.run_timed(n)
    t0 = time.perf_counter()
    r = gradient(S, Prog, obs, n, ncheckpoints=nc)
    wall = time.perf_counter() - t0
    st_ = r.stats
    adj_ms = st_.forward_ms + st_.reverse_ms
    G = S.grid
    print(json.dumps({
        "metric": "adjoint cost / forward cost", "value": adj_ms / fwd_ms, "unit": "x", "n_gpus": 1,
        "higher_is_better": False, "dtype": args.adj_dtype, "data": "synthetic (seeded twin experiment)",
        "config": {"workload": f"twin experiment {G.nx}x{G.ny} periodic channel, "
                               f"{ {'rk4': 'RK4', 'ssprk2': 'SSPRK2 (3 sub-stages)', '4ssprk3': '4SSPRK3'}[args.adj_scheme] }, "
                               f"Arakawa-Hsu, Smagorinsky, "
                               f"quadratic drag, {n} steps, J = sum (eta_T - eta_obs)^2, gradient w.r.t. u0, v0, "
                               f"eta0 and Fx", "checkpoints": st_.checkpoints,
                   "schedule": {0: "checkpoint slots only (binomial, or every state kept)",
                                1: "every step's stage inputs kept",
                                2: "two-level: one slot per segment, segments recomputed in turn",
                                3: "two-level: one slot per segment, each segment recomputed on a second "
                                   "stream while the next is reversed"}[st_.stored_stage_states]},
        "forward_ms": fwd_ms, "adjoint_forward_sweep_ms": st_.forward_ms, "adjoint_reverse_sweep_ms": st_.reverse_ms,
        "adjoint_wall_s": wall, "forward_steps": st_.forward_steps, "adjoint_steps": st_.adjoint_steps,
        "launches_per_adjoint_step": st_.launches_per_adjoint_step,
        "launches_per_forward_step": st_.launches_per_forward_step,
        "J": r.J, "dJ_along_dFx": float(np.sum(r.Fx * dFx))}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="time only --form/--build, not the other forms")
    ap.add_argument("--workload", default="channel", choices=["channel", "ensemble", "adjoint"],
                    help="channel: the 2048x1024 headline run; ensemble: seeded members of uneven size; "
                         "adjoint: the gradient of the 512x256 twin experiment")
    ap.add_argument("--adj-steps", type=int, default=2000)
    ap.add_argument("--adj-nx", type=int, default=512)
    ap.add_argument("--adj-dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--adj-scheme", default="rk4", choices=["rk4", "ssprk2", "4ssprk3"])
    ap.add_argument("--checkpoints", type=int, default=0, help="adjoint checkpoint slots (0: one per step)")
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--days", type=float, default=1.0, help="model days per ensemble member")
    ap.add_argument("--threads", type=int, default=8, help="members run at once per GPU")
    ap.add_argument("--chunks", type=int, default=2, help="ensemble batches per GPU, pipelined with their set-up")
    ap.add_argument("--compare-members", type=int, default=0,
                    help="run the looped single-member comparison on this many members (0: all)")
    ap.add_argument("--build", default="parity", choices=["parity", "fast"],
                    help="parity: libswb200.so (no FMA contraction, bit-exact with the oracle); "
                         "fast: libswb200_fast.so (FMA contraction, equal to the oracle to rounding)")
    ap.add_argument("--form", default="fp32", choices=["fp32", "bf16", "f16"],
                    help="state storage between steps: plain FP32 or compensated 16-bit pairs (u, v scaled by 2^10)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from swb200 import Model, abi, model_setup, Parameter

    kw, rng = workload_params(args.nx)
    P = Parameter(**kw)
    S = model_setup(P)
    G = S.grid
    cells = G.nx * G.ny
    config = {"workload": f"periodic wind-driven channel {G.nx}x{G.ny}, RK4, Arakawa-Hsu, Smagorinsky, "
                          f"quadratic drag, tracer every step",
              "nx": G.nx, "ny": G.ny, "dtint_s": G.dtint, "form": args.form, "build": args.build,
              "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{args.gpus}",
              "step_launch": "one CUDA graph per time step"}
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded η noise, tracer checkerboard, seeded wind amplitude)", "config": config}

    if args.impl == "reference":
        if rank != 0:
            return 0
        Prog = make_state(S, rng)
        threads = os.cpu_count() or 1
        target = 20.0 * (args.steps + args.warmup) / max(args.steps + args.warmup, 1)
        v, n, dt, used = cpu_run(S, Prog, threads, min(60.0, target), args.steps)
        hi = host_info()
        line = dict(base)
        line.update({"impl": "reference", "value": v, "ms_per_step": 1e3 * dt / n,
                     "cpu_baseline": {"value": v, "unit": UNIT, "cores": used, "kind": "port",
                                      "sample": f"{n} steps of the {G.nx}x{G.ny} workload from the same state "
                                                f"({dt:.1f} s), OpenMP over {used} threads of {hi['model']}"},
                     "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        print(json.dumps(line))
        return 0

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev_uuid = None
    try:
        dev_uuid = "GPU-" + str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
    except Exception:
        pass

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.workload == "ensemble":
        return bench_ensemble(args, rank, world, barrier, allmax)
    if args.workload == "adjoint":
        return bench_adjoint(args) if rank == 0 else 0

    Prog = make_state(S, rng)
    storage = {"fp32": "native", "bf16": "bf16", "f16": "f16"}[args.form]
    # clocks are sampled from before the warm-up to after the end-to-end calls,
    # so that the record covers the timed steps whatever their length
    clk = ClockSampler(dev_uuid)
    clk.start()
    clk.wait_first(10.0)

    def time_form(storage, build):
        """Device time of args.steps steps (L2 flushed between steps), then a
        profiled pass for the per-kernel times; returns a dict."""
        m = Model(S, storage=storage, build=build)
        m.set_state(Prog)
        m.run(args.warmup)
        barrier()
        n0 = m.kernel_launches
        step_ms, st = m.run_timed(args.steps, L2_FLUSH)
        launches = m.kernel_launches - n0
        barrier()
        if st.code != 0:
            raise SystemExit(f"run failed with code {st.code}")
        t_dev = allmax(step_ms) / 1e3
        # per-kernel device times: a second, shorter run with an event pair
        # around every launch (no graphs), for the kernel shares and the roofline
        prof, st = m.run_profiled(min(args.steps, 200), L2_FLUSH)
        if st.code != 0:
            raise SystemExit(f"profiled run failed with code {st.code}")
        m.close()
        stage_ms = allmax(prof.kernel_ms[0] / max(prof.launches[0], 1))
        kernels = {abi.PROFILE_NAMES[k]: {"launches": int(prof.launches[k]),
                                          "avg_us": 1e3 * prof.kernel_ms[k] / prof.launches[k],
                                          "share": prof.kernel_ms[k] / max(sum(prof.kernel_ms), 1e-12)}
                   for k in range(abi.PROFILE_KINDS) if prof.launches[k]}
        return {"t_dev": t_dev, "value": args.gpus * cells * args.steps / t_dev, "stage_ms": stage_ms,
                "kernels": kernels, "launches": launches}

    main = time_form(storage, args.build)
    t_dev, value, kernels, launches = main["t_dev"], main["value"], main["kernels"], main["launches"]
    stage_bytes = STAGE_BYTES_PER_CELL if storage == "native" else STAGE_BYTES_PER_CELL_16
    step_bytes = STEP_BYTES_PER_CELL if storage == "native" else STEP_BYTES_PER_CELL_16
    achieved = stage_bytes * cells / (main["stage_ms"] / 1e3) / 1e9
    peak, peak_kind = peaks()
    # the other forms of the metric on the same workload: the FMA build, and
    # the 16-bit storage forms (their error against Float64 is in the precision
    # study); each with its device time per step and ratio to this line's value
    others = {}
    if storage == "native" and not args.no_forms:
        for name, (stg, bld) in {"fp32_fast_build": ("native", "fast"), "bf16": ("bf16", args.build),
                                 "f16": ("f16", args.build)}.items():
            if bld == args.build and stg == storage:
                continue
            r = time_form(stg, bld)
            others[name] = {"value": r["value"], "ratio_to_value": r["value"] / value,
                            "ms_per_step": 1e3 * r["t_dev"] / args.steps,
                            "bytes_per_cell_step": STEP_BYTES_PER_CELL if stg == "native" else STEP_BYTES_PER_CELL_16,
                            "kernels_us": {k: round(v["avg_us"], 2) for k, v in r["kernels"].items()}}

    # e2e: drop-in call with pinned host buffers (create, upload, run, download)
    from swb200 import time_integration  # noqa: F401
    from swb200.run_model import time_integration as ti
    pinned = [torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy() for a in Prog]
    for dst, src in zip(pinned, Prog):
        dst[...] = src
    import ctypes as C
    lib = abi.load_library(build=args.build)
    cfg = abi.make_config(S, nt=args.steps, storage=storage)
    static = abi.StaticFields(S)
    status = abi.SwStatus()

    def e2e_call(c):
        for dst, src in zip(pinned, Prog):      # the call overwrites its buffers: restore the inputs (untimed)
            dst[...] = src
        barrier()
        t0 = time.perf_counter()
        rc = lib.sw_time_integration(C.byref(c), static.ptr(), *abi.state_ptrs(*pinned), C.byref(status))
        dt = time.perf_counter() - t0
        barrier()
        if rc != 0:
            raise SystemExit(f"sw_time_integration failed: {rc}")
        return dt

    # one untimed call of W steps (first-use costs of the process), then the
    # median of three timed calls of K steps
    e2e_call(abi.make_config(S, nt=max(args.warmup, 1), storage=storage))
    t_e2e = allmax(statistics.median(e2e_call(cfg) for _ in range(3)))
    clk.stop()
    state_bytes = sum(a.nbytes for a in pinned)
    static_bytes = packed_static_bytes(static)
    # the same call's phases, timed through the context API on the same pinned
    # buffers: upload (with the state's ghost points), steps, download
    phases = {}
    with Model(S, storage=storage, build=args.build) as mp:
        for _ in range(2):
            barrier()
            t0 = time.perf_counter()
            mp.set_state(type(Prog)(*pinned))
            t1 = time.perf_counter()
            mp.run(args.steps)
            t2 = time.perf_counter()
            rc = mp.lib.sw_get_state(mp.ctx, *abi.state_ptrs(*pinned))
            t3 = time.perf_counter()
            if rc != 0:
                raise SystemExit(f"sw_get_state failed: {rc}")
        phases = {"set_state_ms": 1e3 * (t1 - t0), "run_ms": 1e3 * (t2 - t1), "get_state_ms": 1e3 * (t3 - t2)}
    e2e = {"value": args.gpus * cells * args.steps / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": (state_bytes + static_bytes) / args.steps,
           "d2h_bytes_per_step": state_bytes / args.steps,
           "call": "sw_time_integration with pinned host buffers: static fields packed and uploaded, state "
                   "uploaded, K steps, state downloaded; the context of the warm-up call is reused "
                   "(median of 3 after 1 warm-up call)",
           "call_ms": 1e3 * t_e2e, "phases_context_api": phases}

    cpu = None
    if rank == 0 and args.gpus == 1 and not args.no_cpu:
        v, n, dt, used = cpu_run(S, Prog, 1, args.cpu_seconds, 200)
        hi = host_info()
        cpu = {"value": v, "unit": UNIT, "cores": used, "kind": "port",
               "sample": f"{n} steps of the {G.nx}x{G.ny} workload, single thread, {dt:.1f} s, on {hi['model']} "
                         f"({hi['nproc']} logical CPUs)"}

    if rank == 0:
        line = dict(base)
        line.update({
            "value": value, "ms_per_step": 1e3 * t_dev / args.steps,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": ncu_traffic(cells) if storage == "native" else None,
                         "kernel": "rk_stage_tma" if storage == "native" else "s16_stage_kernel",
                         "bytes_per_cell": stage_bytes,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s"},
            "step_roofline": {"bytes_per_cell_step": step_bytes,
                              "achieved_gbs": step_bytes * cells * args.steps / t_dev / 1e9 / args.gpus,
                              "frac": step_bytes * cells * args.steps / t_dev / 1e9 / args.gpus / peak},
            "other_forms": others,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        })
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
