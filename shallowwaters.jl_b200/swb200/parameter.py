"""Parameter: the model's keyword configuration.

Mirrors ``@with_kw struct Parameter`` of ShallowWaters.jl
(src/default_parameters.jl:1-148): the same field names, defaults and
assertions, so ``Parameter(nx=128, bc="nonperiodic")`` means what it means in
Julia.  Number formats are numpy dtypes (``np.float16``, ``np.float32``,
``np.float64``) in place of Julia's ``Float16/Float32/Float64``.

Integer-valued fields that the reference types as ``Real`` (``Ndays``, ``H``,
``topo_height`` ...) keep the Python type they are given, because the
reference's arithmetic keeps Julia's ``Int``/``Float64`` distinction there
(e.g. ``Ndays*3600*24`` is exact integer arithmetic for ``Ndays=1``).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

_FORMATS = (np.float16, np.float32, np.float64)


def _as_format(t):
    if t is None:
        return None
    t = np.dtype(t).type
    if t not in _FORMATS:
        raise ValueError(f"number format {t} unsupported (Float16, Float32, Float64)")
    return t


@dataclass
class Parameter:
    T: type = np.float32            # number format                      (:3)
    Tprog: Optional[type] = None    # prognostic variables, default T    (:5)
    Tcomm: Optional[type] = None    # ghost-point copies, default Tprog  (:6)

    # DOMAIN RESOLUTION AND RATIO (:9-11)
    nx: int = 100
    Lx: float = 2000e3
    L_ratio: float = 2

    # PHYSICAL CONSTANTS (:14-19)
    g: float = 10.
    H: float = 500.
    ρ: float = 1e3
    ϕ: float = 45.
    ω: float = 2 * np.pi / (24 * 3600)
    R: float = 6.371e6

    # WIND FORCING OPTIONS (:22-29)
    wind_forcing_x: str = "channel"
    wind_forcing_y: str = "constant"
    Fx0: float = 0.12
    Fy0: float = 0.0
    seasonal_wind_x: bool = False
    seasonal_wind_y: bool = False
    ωFx: float = 1.0
    ωFy: float = 1.0

    # BOTTOM TOPOGRAPHY OPTIONS (:32-34)
    topography: str = "ridge"
    topo_height: float = 50.
    topo_width: float = 300e3

    # SURFACE RELAXATION (:37-40)
    surface_relax: bool = False
    t_relax: float = 100.
    η_refh: float = 5.
    η_refw: float = 50e3

    # SURFACE FORCING (:43-47)
    surface_forcing: bool = False
    ωFη: float = 1.0
    A: float = 3e-5
    ϕk: Optional[float] = None      # default ϕ
    wk: float = 10e3

    # TIME STEPPING OPTIONS (:50-58)
    time_scheme: str = "RK"
    RKo: int = 4
    RKs: int = 3
    RKn: int = 2
    cfl: float = 1.0
    Ndays: float = 10.0
    nstep_diff: int = 1
    nstep_advcor: int = 0

    # BOUNDARY CONDITION OPTIONS (:62-63)
    bc: str = "periodic"
    α: float = 2.

    # MOMENTUM ADVECTION OPTIONS (:67-68)
    adv_scheme: str = "ArakawaHsu"
    dynamics: str = "nonlinear"

    # BOTTOM FRICTION OPTIONS (:71-73)
    bottom_drag: str = "quadratic"
    cD: float = 1e-5
    τD: float = 300.

    # DIFFUSION OPTIONS (:76-78)
    diffusion: str = "constant"
    νB: float = 500.0
    cSmag: float = 0.15

    # TRACER ADVECTION (:81-98)
    tracer_advection: bool = True
    tracer_relaxation: bool = False
    tracer_consumption: bool = False
    tracer_pumping: bool = False
    injection_region: str = "west"
    sst_initial: str = "south"
    sst_rect_coords: List[float] = field(default_factory=lambda: [0., 0.15, 0., 1.0])
    Uadv: float = 0.25
    SSTmax: float = 1.
    SSTmin: float = 0.
    τSST: float = 500.
    jSST: float = 365.
    SST_λ0: float = 222e3
    SST_λs: float = 111e3
    SST_γ0: float = 8.35
    SSTw: float = 5e3
    SSTϕ: float = 0.5

    # OUTPUT OPTIONS (:101-104)
    output: bool = False
    output_vars: List[str] = field(default_factory=lambda: ["u", "v", "η", "sst"])
    output_dt: float = 6
    outpath: str = "."

    # INITIAL CONDITIONS (:107-113)
    initial_cond: str = "rest"
    initpath: Optional[str] = None
    init_run_id: int = 0
    init_starti: int = -1
    get_id_mode: str = "continue"
    run_id: int = -1
    init_interpolation: bool = True

    def __post_init__(self):
        self.T = _as_format(self.T)
        self.Tprog = _as_format(self.Tprog) or self.T
        self.Tcomm = _as_format(self.Tcomm) or self.Tprog
        if self.ϕk is None:
            self.ϕk = self.ϕ
        if self.initpath is None:
            self.initpath = self.outpath
        self._check()

    def _check(self):
        """The assertions of src/default_parameters.jl:116-147."""
        def req(cond, msg):
            if not cond:
                raise AssertionError(msg)
        req(all(x > 0. for x in (self.nx, self.Lx, self.L_ratio)), "nx, Lx, L_ratio have to be >0")
        req(all(x > 0. for x in (self.g, self.H, self.ρ, self.ω, self.R)), "g,H,ρ,ω,R have to be >0")
        req(-90.0 <= self.ϕ <= 90.0, f"ϕ has to be in (-90,90), {self.ϕ} given.")
        winds = ["channel", "double_gyre", "shear", "constant", "none"]
        req(self.wind_forcing_x in winds, f"Wind forcing '{self.wind_forcing_x}' unsupported")
        req(self.wind_forcing_y in winds, f"Wind forcing '{self.wind_forcing_y}' unsupported")
        req(self.topography in ["ridge", "seamount", "flat", "ridges"],
            f"Topography '{self.topography}' unsupported")
        req(self.topo_width > 0.0, f"topo_width has to be >0, {self.topo_width} given.")
        req(self.t_relax > 0.0, f"t_relax has to be >0, {self.t_relax} given.")
        req(self.η_refw > 0.0, f"η_refw has to be >0, {self.η_refw} given.")
        req(self.time_scheme in ["RK", "SSPRK2", "SSPRK3", "4SSPRK3"],
            f"Time scheme {self.time_scheme} unsupported.")
        req(self.RKo in [2, 3, 4], f"RKo has to be 2,3 or 4; {self.RKo} given.")
        req(self.RKs > 1, f"RKs has to be >= 2; {self.RKs} given.")
        req(self.Ndays > 0.0, f"Ndays has to be >0, {self.Ndays} given.")
        req(self.nstep_diff > 0, f"nstep_diff has to be >0, {self.nstep_diff} given.")
        req(self.nstep_advcor >= 0, f"nstep_advcor has to be >=0, {self.nstep_advcor} given.")
        req(self.bc in ["periodic", "nonperiodic"], f"boundary condition '{self.bc}' unsupported.")
        req(0.0 <= self.α <= 2.0, f"Tangential boundary condition α has to be in (0,2), {self.α} given.")
        req(self.adv_scheme in ["Sadourny", "ArakawaHsu"], f"Advection scheme '{self.adv_scheme}' unsupported")
        req(self.dynamics in ["linear", "nonlinear"], f"Dynamics '{self.dynamics}' unsupported.")
        req(self.bottom_drag in ["quadratic", "linear", "none"], f"Bottom drag '{self.bottom_drag}' unsupported.")
        req(self.cD >= 0.0, f"Bottom drag coefficient cD has to be >=0, {self.cD} given.")
        req(self.τD >= 0.0, f"Bottom drag coefficient τD has to be >=0, {self.τD} given.")
        req(self.diffusion in ["Smagorinsky", "constant"], f"Diffusion '{self.diffusion}' unsupported.")
        req(self.νB > 0.0, f"Diffusion scaling constant νB has to be >0, {self.νB} given.")
        req(self.cSmag > 0.0, f"Smagorinsky coefficient cSmag has to be >0, {self.cSmag} given.")
        req(self.injection_region in ["west", "south"], f"Injection region '{self.injection_region}' unsupported.")
        req(self.Uadv > 0.0, f"Advection velocity scale Uadv has to be >0, {self.Uadv} given.")
        req(self.output_dt > 0, f"Output time step has to be >0, {self.output_dt} given.")
        req(self.initial_cond in ["rest", "ncfile"], f"Initial conditions '{self.initial_cond}' unsupported.")
        req(self.init_run_id >= 0, f"Initial condition run id, init_run_id, has to be >= 0, {self.init_run_id} given.")
        req(self.init_starti > 0 or self.init_starti == -1,
            f"Start index, init_starti, has to be >0 || -1, {self.init_starti} given.")
        req(self.get_id_mode in ["continue", "fill", "specific"], f"get_id_mode {self.get_id_mode} unsupported.")

    def replace(self, **kwargs) -> "Parameter":
        """A copy with some fields changed (Parameters.jl's reconstruct)."""
        d = {f.name: getattr(self, f.name) for f in dataclasses.fields(self)}
        # re-derive defaults that follow other fields unless given explicitly
        if "T" in kwargs and "Tprog" not in kwargs and self.Tprog == self.T:
            d["Tprog"] = None
        if ("T" in kwargs or "Tprog" in kwargs) and "Tcomm" not in kwargs and self.Tcomm == self.Tprog:
            d["Tcomm"] = None
        d.update(kwargs)
        return Parameter(**d)
