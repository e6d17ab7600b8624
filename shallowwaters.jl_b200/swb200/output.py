"""NetCDF output and restart of the host side (src/output.jl:1-207,
src/initial_conditions.jl:39-120,144-150).

The time loop runs on the GPU; with ``Parameter.output`` the host runs it in
chunks of ``nout`` steps and writes one frame per chunk, as output_nc! does
every nout steps (src/time_integration.jl:233).  Files, variable names, units,
the run folder numbering (run0000, run0001, ... by get_id_mode) and the frame
contents follow the reference:

* u, v, eta, sst: the state after the step, halo removed, as Float32;
* du, dv, deta: the change over the last step (u_{n+1} - u_n, :100-112);
* q, relvort: potential and relative vorticity at the q-points.  The reference
  writes whatever its work arrays hold at that moment (q of the last RK
  stage's input; dvdx/dudy of that input, or of the pre-diffusion state when
  Smagorinsky diffusion ran); here both are evaluated from the written state,
  with PV!'s formula (src/PV_advection.jl:2-18) and relvort = ζ/|f| (:89-94).

The files are NetCDF classic (scipy's writer; netCDF-4/HDF5 libraries are not
part of this environment), which the reference's NetCDF.jl reads as well.
"""
from __future__ import annotations

import os

import numpy as np
from scipy.io import netcdf_file

from .model_setup import ModelSetup

# output_vars name -> (variable, x grid, y grid, units, long_name)   (src/output.jl:29-37)
VARS = {
    "u": ("u", "x_u", "y_u", "m/s", "zonal velocity"),
    "v": ("v", "x_v", "y_v", "m/s", "meridional velocity"),
    "η": ("eta", "x_T", "y_T", "m", "sea surface height"),
    "sst": ("sst", "x_T", "y_T", "1", "sea surface temperature"),
    "q": ("q", "x_q", "y_q", "1/(ms)", "potential vorticity"),
    "ζ": ("relvort", "x_q", "y_q", "1", "relative vorticity"),
    "du": ("du", "x_u", "y_u", "m^2/s^2", "zonal velocity tendency"),
    "dv": ("dv", "x_v", "y_v", "m^2/s^2", "meridional velocity tendency"),
    "dη": ("deta", "x_T", "y_T", "m^2/s", "sea surface height tendency"),
}


def _run_ids(outpath):
    return [int(d[3:]) for d in os.listdir(outpath) if d.startswith("run") and d[3:].isdigit()]


def get_run_id_path(S: ModelSetup):
    """get_run_id_path (src/output.jl:168-207): create and return the run folder."""
    P = S.parameters
    existing = _run_ids(P.outpath)
    if not existing:
        run_id = 0
    elif P.get_id_mode == "fill":
        run_id = min(set(range(max(existing) + 2)) - set(existing))
    elif P.get_id_mode == "specific":
        run_id = P.run_id
    else:  # continue
        run_id = max(existing) + 1
    runpath = os.path.join(P.outpath, f"run{run_id:04d}")
    if P.get_id_mode == "specific" and os.path.isdir(runpath):
        import shutil
        shutil.rmtree(runpath)
    os.makedirs(runpath)
    return run_id, runpath


def vorticities(u, v, η, S: ModelSetup):
    """q and relvort at the q-points (x_q, y_q) from a state with halo ([j][i])."""
    G, P = S.grid, S.parameters
    T = P.T
    N, M, ep = G.nx, G.ny, G.ep
    nqx, nqy = len(G.x_q), len(G.y_q)
    F = np.arange(nqx)[None, :]
    Gq = np.arange(nqy)[:, None]
    uu = np.asarray(u).astype(T)
    vv = np.asarray(v).astype(T)
    h = (np.asarray(η).astype(T) + np.asarray(S.forcing.H, dtype=T)).astype(T)

    def U(f, b):
        return uu[b + 2, f + 1 + ep]

    def V(a, g):
        return vv[g + 1, a + 2]

    def Hh(a, b):
        return h[b + 1, a + 1]

    q4 = T(0.25)
    dvdx = V(F, Gq) - V(F - 1, Gq)
    dudy = U(F, Gq) - U(F, Gq - 1)
    hq = q4 * (Hh(F - 1, Gq - 1) + Hh(F, Gq - 1)) + q4 * (Hh(F - 1, Gq) + Hh(F, Gq))
    fq = np.asarray(G.f_q, dtype=T)[:nqy, :nqx]
    q = (fq + dvdx - dudy) / hq
    with np.errstate(divide="ignore", invalid="ignore"):
        relvort = (dvdx - dudy) / np.abs(fq)
    return q.astype(np.float32), relvort.astype(np.float32)


class NcFiles:
    """The output files of one run (src/output.jl:1-60)."""

    def __init__(self, S: ModelSetup):
        self.S = S
        P, G = S.parameters, S.grid
        self.run_id, self.runpath = get_run_id_path(S)
        self.files = {}
        self.iout = 0
        for key in P.output_vars:
            if key not in VARS:
                raise ValueError(f"output variable {key!r} unsupported")
            name, xg, yg, unit, long_name = VARS[key]
            nc = netcdf_file(os.path.join(self.runpath, name + ".nc"), "w", version=2)
            x, y = np.asarray(getattr(G, xg), float), np.asarray(getattr(G, yg), float)
            nc.createDimension("t", None)              # the record dimension comes first in classic files
            nc.createDimension("y", len(y))
            nc.createDimension("x", len(x))
            for dim, vals, ln in (("x", x, "zonal coordinate"), ("y", y, "meridional coordinate")):
                cv = nc.createVariable(dim, "f8", (dim,))
                cv[:] = vals
                cv.units, cv.long_name = "m", ln
            tv = nc.createVariable("t", "i4", ("t",))
            tv.units, tv.long_name = "s", "time"
            var = nc.createVariable(name, "f4", ("t", "y", "x"))
            var.units, var.long_name, var.missing_value = unit, long_name, np.float32(-999999.0)
            self.files[key] = (nc, name)

    def write(self, i, new, old, rhs=None):
        """output_nc!(i) (src/output.jl:63-133): ``new`` is the state after step i
        and ``old`` the one before it, both with halo.  ``rhs`` is the (u, v, η)
        the reference's vorticity work arrays were last computed from (the
        input of the step's last right-hand-side evaluation); q and relvort
        come from it, or from ``new`` when it is not given."""
        from .initial_conditions import remove_halo
        S = self.S
        new, old = tuple(new), tuple(old)
        un, vn, en, sn = remove_halo(*new, S)
        uo, vo, eo, _ = remove_halo(*old, S)
        f32 = np.float32
        frames = {"u": un.astype(f32), "v": vn.astype(f32), "η": en.astype(f32), "sst": sn.astype(f32),
                  "du": un.astype(f32) - uo.astype(f32), "dv": vn.astype(f32) - vo.astype(f32),
                  "dη": en.astype(f32) - eo.astype(f32)}
        if "q" in self.files or "ζ" in self.files:
            src = rhs if rhs is not None else new
            frames["q"], frames["ζ"] = vorticities(src[0], src[1], src[2], S)
        k = self.iout
        for key, (nc, name) in self.files.items():
            nc.variables[name][k] = frames[key]
            nc.variables["t"][k] = i * S.grid.dtint
            nc.flush()
        self.iout = k + 1

    def close(self):
        for nc, _ in self.files.values():
            nc.close()
        self.files = {}


# ------------------------------------------------------------------ restart

def _interp2(xo, yo, f, xn, yn):
    """Bilinear interpolation of f (rows y, columns x) from the grid (xo, yo) to
    (xn, yn), flat outside: Interpolations.jl's Gridded(Linear()) with Flat()
    extrapolation as used by the reference."""
    def weights(o, n):
        n = np.clip(n, o[0], o[-1])
        k = np.clip(np.searchsorted(o, n, side="right") - 1, 0, len(o) - 2) if len(o) > 1 else np.zeros(len(n), int)
        w = (n - o[k]) / (o[k + 1] - o[k]) if len(o) > 1 else np.zeros(len(n))
        return k, w
    kx, wx = weights(np.asarray(xo, float), np.asarray(xn, float))
    ky, wy = weights(np.asarray(yo, float), np.asarray(yn, float))
    f = np.asarray(f, float)
    f00 = f[np.ix_(ky, kx)]
    f01 = f[np.ix_(ky, np.minimum(kx + 1, f.shape[1] - 1))]
    f10 = f[np.ix_(np.minimum(ky + 1, f.shape[0] - 1), kx)]
    f11 = f[np.ix_(np.minimum(ky + 1, f.shape[0] - 1), np.minimum(kx + 1, f.shape[1] - 1))]
    wx, wy = wx[None, :], wy[:, None]
    return (1 - wy) * ((1 - wx) * f00 + wx * f01) + wy * ((1 - wx) * f10 + wx * f11)


def read_restart(S: ModelSetup):
    """initial_cond == "ncfile" (src/initial_conditions.jl:39-120,144-150):
    u, v, η (and sst with sst_initial == "restart") from frame init_starti of
    run init_run_id in initpath, interpolated when the grid size differs.
    Returns the interior fields in [j][i] storage (sst None unless restarted)."""
    P, G = S.parameters, S.grid
    path = os.path.join(P.initpath, f"run{P.init_run_id:04d}")

    def frame(name):
        with netcdf_file(os.path.join(path, name + ".nc"), "r", mmap=False) as nc:
            k = nc.variables["t"].shape[0] if P.init_starti == -1 else P.init_starti
            return np.array(nc.variables[name][k - 1], dtype=np.float64)

    u, v, η = frame("u"), frame("v"), frame("eta")
    ny_old, nx_old = η.shape
    if (nx_old, ny_old) != (G.nx, G.ny):
        if not P.init_interpolation:
            raise ValueError(f"Grid size {(G.nx, G.ny)} doesn't match initial conditions on a "
                             f"{(nx_old, ny_old)} grid.")
        dx, dy = nx_old / G.nx, ny_old / G.ny
        x_T, y_T = np.arange(nx_old) + 0.5, np.arange(ny_old) + 0.5
        x_u, y_v = np.arange(nx_old, dtype=float), np.arange(1, ny_old, dtype=float)
        x_Tn, y_Tn = np.arange(G.nx) * dx + dx / 2, np.arange(G.ny) * dy + dy / 2
        x_un, y_vn = np.arange(G.nx) * dx, np.arange(1, G.ny) * dy
        u = _interp2(x_u[:u.shape[1]], y_T, u, x_un[:G.nux], y_Tn)
        v = _interp2(x_T, y_v, v, x_Tn, y_vn)
        η = _interp2(x_T, y_T, η, x_Tn, y_Tn)
    sst = frame("sst") if P.sst_initial == "restart" else None
    return u, v, η, sst
