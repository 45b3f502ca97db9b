"""Lattice descriptor on the Python side, converted to ``lbm_desc`` for the C ABI.

The enums mirror the reference's switches (src/LBM/util/flag.py:10-110); the
side table mirrors ``set_BC`` (src/LBM/LBM2D/_io.py:385-402): an ``inlet``
fixes velocity and extrapolates density, an ``outlet`` fixes density and
extrapolates velocity, a ``wall`` fixes velocity to zero.
"""
from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass, field

from . import _native as N

PERIODIC, ZERO_GRADIENT, FIXED_VALUE = N.LBM_BC_PERIODIC, N.LBM_BC_ZEROGRADIENT, N.LBM_BC_FIXEDVALUE
FLOW_RATE = N.LBM_BC_FLOWRATE   # velocity type of side 0 only (flow-rate inlet)

# d'Humieres et al. (2002) rates for D3Q19: e, eps, q, pi, m (viscous rows use 1/tau)
MRT_RATES_3D = {1: 1.19, 2: 1.4, 4: 1.2, 6: 1.2, 8: 1.2, 10: 1.4, 12: 1.4, 16: 1.98, 17: 1.98, 18: 1.98}
# Lallemand & Luo (2000) rates for D2Q9: e, eps, q
MRT_RATES_2D = {1: 1.64, 2: 1.54, 4: 1.9, 6: 1.9}

GAS_CONSTANT = 8.314441  # src/LBM/util/constant.py:17


@dataclass
class SideBC:
    """One domain side.  ``active`` False keeps the side periodic; ``model`` is the
    boundary scheme of an active side: "nee" (non-equilibrium extrapolation), "es"
    (equilibrium populations of the side's state) or "nebb" (Zou-He non-equilibrium
    bounce-back, 2D), the reference's BC_MODEL."""
    active: bool = False
    v_type: int = PERIODIC
    rho_type: int = PERIODIC
    T_type: int = PERIODIC
    v: tuple = (0.0, 0.0, 0.0)
    rho: float = 1.0
    T: float = 0.0
    model: str = "nee"

    def code(self) -> int:
        """lbm_side_desc.active: 0 periodic, 1 NEE, 2 ES, 3 NEBB."""
        if not self.active:
            return 0
        codes = {"nee": 1, "es": 2, "nebb": 3}
        if self.model not in codes:
            raise ValueError(f"side model {self.model!r}: 'nee', 'es' or 'nebb'")
        return codes[self.model]

    @staticmethod
    def inlet(v, T_type=PERIODIC, T=0.0) -> "SideBC":
        return SideBC(True, FIXED_VALUE, ZERO_GRADIENT, T_type, tuple(v), 1.0, T)

    @staticmethod
    def outlet(rho, T_type=PERIODIC, T=0.0) -> "SideBC":
        return SideBC(True, ZERO_GRADIENT, FIXED_VALUE, T_type, (0.0, 0.0, 0.0), rho, T)

    @staticmethod
    def pressure(rho, T_type=PERIODIC, T=0.0) -> "SideBC":
        """Fixed density with extrapolated velocity (an ``outlet`` used as a pressure inlet)."""
        return SideBC.outlet(rho, T_type, T)

    @staticmethod
    def wall(T_type=PERIODIC, T=0.0) -> "SideBC":
        return SideBC(True, FIXED_VALUE, ZERO_GRADIENT, T_type, (0.0, 0.0, 0.0), 1.0, T)

    @staticmethod
    def inlet_flowrate(flowrate, T_type=PERIODIC, T=0.0) -> "SideBC":
        """Flow-rate inlet, side 0 only (the reference's BC_FLOW.inlet_flow,
        src/LBM/LBM2D/_boundary.py:324-333): the inlet velocity is steered each step
        so that the sum of rho*u_x over the side's cells approaches ``flowrate``."""
        return SideBC(True, FLOW_RATE, ZERO_GRADIENT, T_type, (float(flowrate), 0.0, 0.0), 1.0, T)


@dataclass
class LatticeConfig:
    dim: int
    nx: int
    ny: int
    nz: int = 1
    collision: str = "bgk"          # "bgk" | "mrt"
    precision: str = "fp32"         # "fp32" | "fp16" | "fp64"
    eos: str = "ideal_gas"          # "ideal_gas" | "incompressible"
    nu: float = 0.1                 # lattice viscosity; tau = 3 nu/rho + 1/2 (ideal gas)
    force: tuple = (0.0, 0.0, 0.0)  # body acceleration (lattice units)
    half_force_velocity: bool = False
    thermal: str = "none"           # "none" | "conjugate" | "two_field" (reference TF/TS, adiabatic interface)
    tauT_fluid: float = 0.6
    tauT_solid: float = 0.9
    pyro: bool = False
    pyro_A: float = 1e8             # 1/s
    pyro_b: float = 0.0
    pyro_Ea: float = 1.25e5         # J/mol
    pyro_Tmin: float = 0.0          # K
    T_ref: float = 300.0            # K at T = 0
    T_scale: float = 500.0          # K per unit T
    dt_phys: float = 1e-4           # s per lattice step
    heat_norm: float = 0.8          # dH/(c_s T_scale) = 4e5/(1000*500)
    gas_coef: float = 0.75          # (1 - char yield) * rho_s, rho_s = 1 lattice unit
    alpha_flip: float = 0.01
    mrt_rates: dict = field(default_factory=dict)
    rho0: float = 1.0
    T0: float = 0.0
    sides: list = field(default_factory=lambda: [SideBC() for _ in range(6)])
    bulk_form: str = "auto"         # "auto" (cell lists from 65536 cells) | "tile" | "list" | "dense" (3D)
    viscosity: str = "constant"     # "constant" (nu) | "sutherland" (per cell from T; thermal only)
    suth_A: float = 0.0             # Sutherland: nu = suth_A TK^1.5 / (TK + suth_Ts), TK = T_ref + T_scale T
    suth_Ts: float = 0.0            #   (suth_A = As dt/dx^2 in lattice units, suth_Ts in K)
    porous: str = "none"            # porous cells (0 < solid fraction < 1): "none" | "ergun" | "darcy"
                                    #   | "darcy_forchheimer" (the reference's PORO_MODEL)
    # two fields with porous cells: TF and TS exchange heat in porous cells
    Ts_ref: float | None = None     # solid temperature mapping (TS.v_ref / v_scale); None: T_ref / T_scale
    Ts_scale: float | None = None
    cap_fluid: float = 1000.0       # mass heat capacities (J/(kg K)), TF.cm / TS.cm
    cap_solid: float = 1000.0
    dx_phys: float = 1.0            # cell size (m): radiation per volume, a / dx
    radiation: bool = False         # surface radiation of porous cells (RADIATION_MODEL.SURFACE_UNIFORM)
    T_ambient: float = 300.0        # K
    fp16_rounding: str = "stochastic"  # FP16 storage of the temperature populations: "stochastic" | "nearest"
    # temperature-dependent thermal properties (THERMAL_DIFF_MODEL.DERIVED) per phase: None
    # (the constant tauT_fluid / tauT_solid) or a dict made by thermal_props(); tp_rhos is
    # the solid density of the derived solid diffusivity, tp_dt and tp_dx2 the physical dt, dx^2
    tprop_fluid: dict | None = None
    tprop_solid: dict | None = None
    tp_rhos: float = 1.0
    tp_dt: float = 1.0
    tp_dx2: float = 1.0
    # > 0: the fluid's PRANDTL diffusivity, the cell's kinetic viscosity / tp_prandtl
    # (instead of tprop_fluid and tauT_fluid)
    tp_prandtl: float = 0.0

    @property
    def shape(self) -> tuple:
        return (self.nx, self.ny, self.nz)

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def Q(self) -> int:
        return 9 if self.dim == 2 else 19

    @property
    def QT(self) -> int:
        return 5 if self.dim == 2 else 7

    def replace(self, **kw) -> "LatticeConfig":
        c = dataclasses.replace(self, **kw)
        c.sides = [dataclasses.replace(s) for s in (kw.get("sides") or self.sides)]
        return c

    def to_dict(self) -> dict:
        """Plain JSON-able form (checkpoints)."""
        d = dataclasses.asdict(self)
        d["mrt_rates"] = {str(k): v for k, v in self.mrt_rates.items()}
        return d

    @staticmethod
    def from_dict(d: dict) -> "LatticeConfig":
        d = dict(d)
        d["force"] = tuple(d["force"])
        d["mrt_rates"] = {int(k): float(v) for k, v in d.get("mrt_rates", {}).items()}
        d["sides"] = [SideBC(**{**s, "v": tuple(s["v"])}) for s in d["sides"]]
        return LatticeConfig(**d)

    def tau(self, rho: float = 1.0) -> float:
        nu = self.nu / rho if self.eos == "ideal_gas" else self.nu
        return 3.0 * nu + 0.5

    def mrt_s(self) -> list:
        base = MRT_RATES_2D if self.dim == 2 else MRT_RATES_3D
        s = [0.0] * 19
        for r, v in base.items():
            s[r] = v
        for r, v in self.mrt_rates.items():
            s[int(r)] = float(v)
        return s

    def to_desc(self) -> N.lbm_desc:
        d = N.lbm_desc()
        d.struct_size = ctypes.sizeof(N.lbm_desc)
        d.dim, d.nx, d.ny, d.nz = self.dim, self.nx, self.ny, (1 if self.dim == 2 else self.nz)
        d.collision = {"bgk": N.LBM_COLL_BGK, "mrt": N.LBM_COLL_MRT}[self.collision]
        d.precision = {"fp32": N.LBM_PREC_FP32, "fp16": N.LBM_PREC_FP16, "fp64": N.LBM_PREC_FP64}[self.precision]
        d.eos = {"ideal_gas": N.LBM_EOS_IDEAL_GAS, "incompressible": N.LBM_EOS_INCOMPRESSIBLE}[self.eos]
        d.thermal = {"none": N.LBM_THERMAL_NONE, "conjugate": N.LBM_THERMAL_CONJUGATE,
                     "two_field": N.LBM_THERMAL_TWOFIELD}[self.thermal]
        d.pyro = int(self.pyro)
        d.half_force_velocity = int(self.half_force_velocity)
        d.bulk_form = {"auto": 0, "tile": 1, "list": 2, "dense": 3}[self.bulk_form]
        d.nu = self.nu
        for i in range(3):
            d.force[i] = float(self.force[i])
        d.tauT_fluid, d.tauT_solid = self.tauT_fluid, self.tauT_solid
        d.pyro_A, d.pyro_b, d.pyro_Ea, d.pyro_Tmin = self.pyro_A, self.pyro_b, self.pyro_Ea, self.pyro_Tmin
        d.T_ref, d.T_scale, d.dt_phys = self.T_ref, self.T_scale, self.dt_phys
        d.heat_norm, d.gas_coef, d.alpha_flip = self.heat_norm, self.gas_coef, self.alpha_flip
        for r, v in enumerate(self.mrt_s()):
            d.mrt_s[r] = v
        d.rho0, d.T0 = self.rho0, self.T0
        fill_sides(d.side, self.sides)
        d.viscosity = {"constant": N.LBM_VISC_CONSTANT, "sutherland": N.LBM_VISC_SUTHERLAND}[self.viscosity]
        d.suth_A, d.suth_Ts = self.suth_A, self.suth_Ts
        d.porous = {"none": N.LBM_PORO_NONE, "ergun": N.LBM_PORO_ERGUN, "darcy": N.LBM_PORO_DARCY,
                    "darcy_forchheimer": N.LBM_PORO_DARCY_FORCHHEIMER}[self.porous]
        d.Ts_ref = self.T_ref if self.Ts_ref is None else self.Ts_ref
        d.Ts_scale = self.T_scale if self.Ts_scale is None else self.Ts_scale
        d.cap_fluid, d.cap_solid, d.dx_phys = self.cap_fluid, self.cap_solid, self.dx_phys
        d.T_ambient, d.radiation = self.T_ambient, int(self.radiation)
        d.fp16_rounding = {"stochastic": N.LBM_FP16_STOCHASTIC, "nearest": N.LBM_FP16_NEAREST}[self.fp16_rounding]
        d.tprop = 0
        for ph, tp in enumerate((self.tprop_fluid, self.tprop_solid)):
            if tp is None:
                continue
            d.tprop |= 1 << ph
            for i in range(5):
                d.tp_cond[ph][i] = float(tp["cond"][i])
                d.tp_cap_lo[ph][i] = float(tp["cap_lo"][i])
                d.tp_cap_hi[ph][i] = float(tp["cap_hi"][i])
            d.tp_cap_Tmid[ph], d.tp_cap_mul[ph] = float(tp["cap_Tmid"]), float(tp["cap_mul"])
        d.tp_rhos, d.tp_dt, d.tp_dx2 = self.tp_rhos, self.tp_dt, self.tp_dx2
        if self.tp_prandtl > 0:
            if self.tprop_fluid is not None:
                raise ValueError("tp_prandtl and tprop_fluid both set the fluid's diffusivity")
            d.tprop |= 4
            d.tp_prandtl = self.tp_prandtl
        return d

    @property
    def porous_heat(self) -> bool:
        """Porous cells with two temperature fields: a porous cell carries TF and TS."""
        return self.porous != "none" and self.thermal == "two_field"


GAS_CONSTANT = 8.314441   # J/(mol K), src/LBM/util/constant.py:17


def thermal_props(cond=None, cond_poly=None, cap=None, cap_poly=None, nasa7=None, solid=False) -> dict:
    """One phase's temperature-dependent diffusivity inputs (src/LBM/LBM2D/_thermal.py:62-107,
    :167-210): a constant or polynomial conductivity, a constant, polynomial or NASA7
    (Trange, 2 x 7 coefficients) capacity.  The polynomials keep the reference's nested form
    c0 + T (c1 + T (c2 T + T (c3 + T c4))); the solid conductivity uses four coefficients and a
    fluid NASA7 capacity is multiplied by the gas constant (the solid's is not)."""
    def five(v):
        v = [float(x) for x in v]
        return (v + [0.0] * 5)[:5]
    if cond_poly is not None:
        kc = five(cond_poly)
        if solid:
            kc[4] = 0.0
    elif cond is not None:
        kc = [float(cond), 0.0, 0.0, 0.0, 0.0]
    else:
        raise ValueError("a derived diffusivity needs a conductivity")
    mul, Tmid = 1.0, 0.0
    if nasa7 is not None:
        Trange, data = nasa7
        lo, hi, Tmid = five(data[0]), five(data[1]), float(Trange[1])
        mul = 1.0 if solid else GAS_CONSTANT
    elif cap_poly is not None:
        lo = hi = five(cap_poly)
    elif cap is not None:
        lo = hi = [float(cap), 0.0, 0.0, 0.0, 0.0]
    else:
        raise ValueError("a derived diffusivity needs a capacity")
    return dict(cond=kc, cap_lo=lo, cap_hi=hi, cap_Tmid=Tmid, cap_mul=mul)


def fill_sides(arr, sides) -> None:
    for i, s in enumerate(sides):
        arr[i].active = s.code()
        arr[i].v_type, arr[i].rho_type, arr[i].T_type = int(s.v_type), int(s.rho_type), int(s.T_type)
        for k in range(3):
            arr[i].v[k] = float(s.v[k])
        arr[i].rho, arr[i].T = float(s.rho), float(s.T)
