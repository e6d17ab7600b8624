"""The precision forms against Float64, on the GPU.

The headline workload is a periodic wind-driven channel, 2048 x 1024 at full
size: RK4, Arakawa-Hsu, Smagorinsky, quadratic drag, tracer every step, flat
H = 500 m.  The wind amplitude Fx0 ~ U(0.08, 0.16) Pa, the eta noise
(sigma = 0.01 m) and the +-1 tracer checkerboard are seeded.  This module runs
it in several forms from the same initial state:

  f64   T = Tprog = Float64 (the reference solution; the GPU Float64 path is
        bit-exact with the Float64 oracle in the parity tests)
  f32   plain Float32
  bf16  Float32 compute, u, v, eta stored as compensated bfloat16 pairs (u, v
        scaled by 2^10), tracer as bfloat16
  f16   the same with IEEE half

and reports, for each form against f64 after the run, the RMSE of eta and u
relative to the standard deviation of the f64 field, the relative difference
of the total energy (FP64 on-device sum) and of the kinetic energy from f64's,
and the device time per step.

Two more workloads run the same comparison:

  c1  the periodic channel at 100 x 50 (Fx0 = 0.12 Pa, tracer every step)
  c2  the double gyre at 512 x 512: nonperiodic free slip (α = 0), double-gyre
      wind Fx0 = 0.12 Pa, a 50 m Gaussian seamount on 500 m, tracer on
      (Uadv = 0.25, a tracer step every nadvstep steps)

both from rest with seeded η noise (σ = 0.01 m) and the ±1 checkerboard.

    python -m swb200.precision --workload c3 --nx 2048 --days 10
    python -m swb200.precision --workload c2 --days 100 --forms f64,f32
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

FORMS = {"f64": (np.float64, "native"), "f32": (np.float32, "native"),
         "bf16": (np.float32, "bf16"), "f16": (np.float32, "f16")}


def channel_params(nx=2048, seed=1234, Ndays=100.0):
    """Parameter keywords of the channel workload and the rng for its state."""
    rng = np.random.default_rng(seed)
    Fx0 = float(rng.uniform(0.08, 0.16))
    kw = dict(nx=nx, L_ratio=2, bc="periodic", wind_forcing_x="channel", Fx0=Fx0, topography="flat", H=500,
              g=10, cfl=1, time_scheme="RK", RKo=4, adv_scheme="ArakawaHsu", diffusion="Smagorinsky",
              bottom_drag="quadratic", tracer_advection=True, Uadv=1000, Ndays=Ndays)
    return kw, rng


def workload_params(workload, nx=2048, days=100.0, seed=1234):
    """Parameter keywords and state rng of a study workload (c1, c2 or c3)."""
    if workload == "c3":
        return channel_params(nx, seed, Ndays=days)
    rng = np.random.default_rng(seed)
    if workload == "c1":
        kw = dict(nx=100, L_ratio=2, bc="periodic", wind_forcing_x="channel", Fx0=0.12, topography="flat", H=500,
                  g=10, cfl=1, time_scheme="RK", RKo=4, adv_scheme="ArakawaHsu", diffusion="Smagorinsky",
                  bottom_drag="quadratic", tracer_advection=True, Uadv=1000, Ndays=days)
    elif workload == "c2":
        kw = dict(nx=512, L_ratio=1, bc="nonperiodic", α=0, wind_forcing_x="double_gyre", Fx0=0.12,
                  topography="seamount", topo_height=50, H=500, g=10, cfl=1, time_scheme="RK", RKo=4,
                  tracer_advection=True, Ndays=days)
    else:
        raise ValueError(f"unknown workload {workload!r}")
    return kw, rng


def kinetic_energy(u, v, S):
    """½ Σ (Ix(u²) + Iy(v²)) over the T-cells of the interior state (float64)."""
    G = S.grid
    uu = np.asarray(u, np.float64) ** 2
    vv = np.asarray(v, np.float64) ** 2
    N, M, ep = G.nx, G.ny, G.ep
    # interiors without halo: u is nux x M, v is N x (M-1); pad the walls with zeros
    ux = np.zeros((M, N + 1))
    ux[:, (1 - ep):(1 - ep) + uu.shape[1]] = uu
    if ep:
        ux[:, N] = uu[:, 0]
    vy = np.zeros((M + 1, N))
    vy[1:M, :] = vv
    return float(0.5 * np.sum(0.5 * (ux[:, :-1] + ux[:, 1:]) + 0.5 * (vy[:-1] + vy[1:])))


def channel_state(S, rng):
    """Seeded eta noise and the +-1 tracer checkerboard of 10 x 10-cell blocks."""
    from . import initial_conditions
    G = S.grid
    eta = rng.normal(0.0, 0.01, (G.ny, G.nx))
    i = np.arange(G.nx)[None, :]
    j = np.arange(G.ny)[:, None]
    sst = np.where(((i // 10) + (j // 10)) % 2 == 0, 1.0, -1.0)
    return initial_conditions(S.parameters.Tprog, S, η0=eta, sst0=sst)


def run_form(form, nx, days, scale=1024.0, workload="c3"):
    """Final interiors (u, v, eta, sst as float64), energies, KE and ms per step."""
    from . import Model, Parameter, model_setup
    from .initial_conditions import remove_halo
    T, storage = FORMS[form]
    kw, rng = workload_params(workload, nx, days)
    P = Parameter(T=T, **kw)
    S = model_setup(P)
    Prog = channel_state(S, rng)
    with Model(S, storage=storage, storage_scale_uv=scale) as m:
        m.set_state(Prog)
        e0 = m.diagnostics().energy
        ms, st = m.run_timed(S.grid.nt)
        e1 = m.diagnostics().energy
        out = [np.asarray(a, np.float64) for a in remove_halo(*m.get_state(), S)]
    ke = kinetic_energy(out[0], out[1], S)
    return out, (e0, e1), ms / max(st.steps_done, 1), st.steps_done, st.code, ke, S


def study(nx=2048, days=10.0, forms=("f64", "f32", "bf16", "f16"), workload="c3"):
    res = {f: run_form(f, nx, days, workload=workload) for f in forms}
    (u64, _, e64, _), (_, E64), _, steps, _, KE64, S = res["f64"]
    G = S.grid
    out = {"workload": f"{workload}: {G.nx}x{G.ny} {S.parameters.bc}, {days} days", "steps": steps,
           "energy_f64": E64, "kinetic_energy_f64": KE64, "forms": {}}
    for f in forms:
        (u, _, e, _), (_, E), ms, n, code, KE, _ = res[f]
        out["forms"][f] = {
            "eta_rmse_rel_std": float(np.sqrt(np.mean((e - e64) ** 2)) / np.std(e64)),
            "u_rmse_rel_std": float(np.sqrt(np.mean((u - u64) ** 2)) / np.std(u64)),
            "energy_rel_to_f64": float((E - E64) / E64),
            "kinetic_energy_rel_to_f64": float((KE - KE64) / KE64),
            "ms_per_step": ms, "steps": n, "status": code}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3"])
    ap.add_argument("--nx", type=int, default=2048, help="grid size of the c3 channel")
    ap.add_argument("--days", type=float, default=10.0)
    ap.add_argument("--forms", default="f64,f32,bf16,f16")
    a = ap.parse_args()
    t0 = time.time()
    r = study(a.nx, a.days, tuple(a.forms.split(",")), workload=a.workload)
    r["wall_s"] = time.time() - t0
    print(json.dumps(r))


if __name__ == "__main__":
    main()
