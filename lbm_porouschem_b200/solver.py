"""Reference-shaped solver classes on the CUDA lattice update.

``LBM2DSolver`` / ``LBM3DSolver`` keep the constructor, the setters that the
reference's YAML driver calls (src/LBM/app.py:101-602), ``init_simulation``,
``step``, ``log_info`` and field access (``rho``, ``v``, ``solid``, ``TF.S``,
``TS.S`` with ``to_numpy``/``from_numpy``) of src/LBM/LBM2D/__init__.py:29-70 and
src/LBM/LBM3D/__init__.py:11-62, and run every step through the C ABI.

Supported on the CUDA path: constant or Sutherland viscosity (IDEAL_GAS or
INCOMPRESSIBLE), binary solid masks with halfway bounce-back, porous cells, body force
(Guo), BGK or MRT, the reference's two temperature fields (TF in fluid, TS in solid; with a
binary mask they exchange no heat, so the interface is adiabatic; in porous cells they
exchange heat and radiate), or with pyrolysis the conjugate temperature field (one
distribution over fluid and solid), constant, Prandtl or derived thermal diffusivities (the
latter two per cell, derived from constant, polynomial or NASA7 properties), the
single-step pyrolysis model with solid->fluid flip, and NEE / ES / NEBB boundaries
(inlet / outlet / wall / symmetric / flow-rate inlet, temperature fixedValue / zeroGradient).
Features of the reference outside that set raise NotImplementedError with the
reason instead of silently running something else.
"""
from __future__ import annotations

import logging
import os
from typing import Callable, Optional

import numpy as np

from .config import FIXED_VALUE, FLOW_RATE, PERIODIC, ZERO_GRADIENT, LatticeConfig, SideBC, thermal_props
from .flag import (BC, BC_FLOW, BC_MODEL, FLUID_STATE_EQUATION, FORCE_TERM, PORO_MODEL, RADIATION_MODEL, SOURCE_TERM,
                   VISCOSITY_MODEL)
from .vtk import PVDWriter, write_vts

_BC_CODE = {BC.periodic: PERIODIC, BC.zeroGradient: ZERO_GRADIENT, BC.fixedValue: FIXED_VALUE}
_log = logging.getLogger("LBM 2D logger")


def _as_array(param, shape, ncomp: int = 0):
    """init_field semantics (src/LBM/LBM2D/_io.py:37-57): a number fills the field, a str
    is a text file in Fortran order, an ndarray is used as is."""
    if isinstance(param, (int, float, np.floating, np.integer)):
        return np.full(shape, float(param))
    if isinstance(param, str):
        return np.reshape(np.loadtxt(param), shape, order="F")
    a = np.asarray(param, dtype=np.float64)
    if a.shape != shape:
        a = a.reshape(shape)
    return a


class Field:
    """Host-side stand-in for a Taichi field of the reference solver.

    Before ``init_simulation`` it holds the initial values; afterwards
    ``to_numpy`` returns the current state read back from the GPU."""

    def __init__(self, solver: "_SolverBase", name: str, ncomp: int = 0, init=0.0):
        self._s = solver
        self.name = name
        self.ncomp = ncomp
        shp = solver._shape + ((ncomp,) if ncomp else ())
        self._host = np.full(shp, float(init))

    @property
    def shape(self):
        return self._s._shape

    def from_numpy(self, a) -> None:
        if self._s._lat is not None:
            raise RuntimeError(f"{self.name}: set initial fields before init_simulation()")
        self._host = np.asarray(a, dtype=np.float64).reshape(self._host.shape).copy()

    def to_numpy(self) -> np.ndarray:
        return self._s._read_field(self.name, self._host)

    def fill(self, v) -> None:
        self.from_numpy(np.full(self._host.shape, float(v)))


class ScalarFieldView:
    """TF / TS of the reference (src/LBM/LBM2D/_scalarField.py:5-58): normalisation and
    per-side boundary settings of one temperature field."""

    def __init__(self, solver: "_SolverBase", name: str):
        self.LBM = solver
        self.name = name
        self.S = Field(solver, name)
        self.v_ref = 0.0
        self.v_scale = 1.0
        self.BC = [BC.periodic] * solver._nsides
        self.s_BC = [0.0] * solver._nsides
        self.thermal_diff = 3e-5
        # THERMAL_DIFF_MODEL.DERIVED (src/LBM/LBM2D/_thermal.py:62-107): D = cond / (rho cm),
        # conductivity constant or polynomial, capacity constant, polynomial or NASA7
        self.derived = False
        self.Pr: Optional[float] = None         # THERMAL_DIFF_MODEL.PRANDTL (fluid)
        self.cond: Optional[float] = None
        self.cond_poly: Optional[list] = None
        self.cm: Optional[float] = None
        self.cm_poly: Optional[list] = None
        self.nasa7: Optional[tuple] = None      # (Trange, 2 x 7 coefficients)
        # heat exchange and radiation of porous cells (TS, src/LBM/LBM2D/_thermal.py:110-120):
        # per-cell exchange coefficient and surface, radiating surface and emissivity
        self.exchangeCoef = Field(solver, name + "_exchangeCoef")
        self.exchangeSurface = Field(solver, name + "_exchangeSurface")
        self.radiation_surface = Field(solver, name + "_radiation_surface")
        self.emissivity = Field(solver, name + "_emissivity")
        self.radiation_model = RADIATION_MODEL.NONE
        self.Tambient = 300.0

    def get_physical_value(self, v):
        return v * self.v_scale + self.v_ref

    def get_normalized_value(self, v_phys):
        return (v_phys - self.v_ref) / self.v_scale

    def set_BC(self, i, bc):
        self.BC[i] = bc

    def set_BCs(self, bcs):
        for i, b in enumerate(bcs):
            self.set_BC(i, b)

    def set_s_BC_value(self, i, s):
        self.s_BC[i] = self.get_normalized_value(s)


class _SolverBase:
    DIM = 2

    def __init__(self, X, Y, Z, dx=1, dt=1, name="default_LBM", isThermal=False, isChemical=False,
                 isPoro=False, isRadiation=False):
        self.name = name
        self.X, self.Y, self.Z = X, Y, Z
        self.dx, self.dt = dx, dt
        self.nx = int(X / dx)
        self.ny = int(Y / dx)
        self.nz = int(Z / dx) if self.DIM == 3 else 1
        self._shape = (self.nx, self.ny, self.nz)
        self._nsides = 4 if self.DIM == 2 else 6
        self.t = 0.0
        self.tLattice: int = 0
        self.tol = 1e-6
        self.TEMPERATURE = bool(isThermal)
        self.CHEMISTRY = bool(isChemical)
        self.PORO = bool(isPoro)
        self.RADIATION = bool(isRadiation and isThermal)
        self.viscosity_model = VISCOSITY_MODEL.NONE
        self.visco = 2e-5
        self.sutherland_coef = [1.6e-6, 170.0]   # src/LBM/LBM2D/_core.py:27
        self.source_term_model = SOURCE_TERM.NONE
        self.force_term_model = FORCE_TERM.NONE
        self.boundary_condition_model = BC_MODEL.NEE
        self.EOS = FLUID_STATE_EQUATION.IDEAL_GAS
        self.collision = "bgk"
        self.precision = "fp32"
        self.body_force = (0.0, 0.0, 0.0)
        self.half_force_velocity = False
        # reference behaviour switches (default: the fixed behaviour)
        self.ref_quirk_nee_on_periodic = False
        self.bc = [BC_FLOW.periodic] * self._nsides
        self.bc_v = [BC.periodic] * self._nsides
        self.bc_rho = [BC.periodic] * self._nsides
        self.v_BC = [(0.0, 0.0, 0.0)] * self._nsides
        self.rho_BC = [1.0] * self._nsides
        self.flow_BC = [0.0] * self._nsides
        self.UpdateBCfunc: list[Callable] = []
        self.GetVariableFunc: list[Callable] = []
        self.exportPath = "vtk"
        self.snapshotPath = "snapshot.yaml"
        self.specieName: list = []          # no species transport on the CUDA path
        self.PVD = PVDWriter(self.exportPath, name)
        # node coordinates of the VTK grid (src/LBM/LBM2D/_core.py:38-40)
        self.x = np.linspace(0, X, self.nx)
        self.y = np.linspace(0, Y, self.ny)
        self.z = np.linspace(0, Z, self.nz)
        self.rho = Field(self, "rho", 0, 1.0)
        self.v = Field(self, "v", 3, 0.0)
        self.solid = Field(self, "solid", 0, 0.0)
        self.rhos = Field(self, "rhos", 0, 0.0)
        self.TF = ScalarFieldView(self, "TF")
        self.TS = ScalarFieldView(self, "TS")
        self._pyro: Optional[dict] = None
        self._reactive: Optional[np.ndarray] = None
        self._lat = None
        if self.PORO:
            # src/LBM/LBM2D/_core.py:92-95: SPHERICAL (Ergun from the porosity) until a
            # set_poro_* setter picks another model; per-cell coefficients
            self.poro_model = PORO_MODEL.SPHERICAL
            self.coefDarcy = Field(self, "coefDarcy", 0, 0.0)
            self.coefForchheimer = Field(self, "coefForchheimer", 0, 0.0)

    # ------------------------------------------------------------ reference dunders
    def __repr__(self):
        return self.__str__()

    def __str__(self):
        return self.description()

    def __call__(self):
        print(self)

    def description(self) -> str:
        d = f"{self.name}: {self.nx} x {self.ny} x {self.nz} lattice, dx={self.dx}, dt={self.dt}\n"
        d += f"  collision {self.collision.upper()}, storage {self.precision}, viscosity (LU) {self._nu_lu():.6g}\n"
        d += f"  thermal {self._thermal_mode()}, pyrolysis {'on' if self._pyro else 'off'}\n"
        return d

    # ------------------------------------------------------------ setters (src/LBM/LBM2D/_io.py)
    def set_vtk_path(self, path):
        self.exportPath = path
        self.PVD.exportPath = path

    def init_field(self, field: Field, param):
        field.from_numpy(_as_array(param, self._shape))

    def init_field3(self, field: Field, p1, p2, p3):
        comps = [_as_array(p, self._shape) for p in (p1, p2, p3)]
        field.from_numpy(np.stack(comps, axis=-1))

    def add_solid(self, solid):
        s = self.solid._host + np.asarray(solid, dtype=np.float64).reshape(self._shape)
        self.solid.from_numpy(s)

    def add_rho_solid(self, rhos):
        self.rhos.from_numpy(self.rhos._host + np.asarray(rhos, dtype=np.float64).reshape(self._shape))

    def set_viscosity(self, mu):
        self.visco = mu
        self.viscosity_model = VISCOSITY_MODEL.CONSTANT

    def set_viscosity_sutherland(self, As, Ts):
        """src/LBM/LBM2D/_io.py:144-147: mu = As T^1.5/(T + Ts) at the fluid temperature."""
        self.sutherland_coef = [float(As), float(Ts)]
        self.viscosity_model = VISCOSITY_MODEL.SUTHERLAND

    def set_viscosity_mixture(self):
        raise NotImplementedError("mixture viscosity needs species transport, which is not on the CUDA path")

    def set_fluid_Trange(self, Trange):
        self.TF.v_ref, self.TF.v_scale = Trange[0], Trange[1] - Trange[0]

    def set_solid_Trange(self, Trange):
        self.TS.v_ref, self.TS.v_scale = Trange[0], Trange[1] - Trange[0]

    # each diffusivity setter selects its model (src/LBM/LBM2D/_io.py:174-184, :218-224)
    def set_fluid_thermal_diff(self, diff):
        self.TF.thermal_diff, self.TF.derived, self.TF.Pr = diff, False, None

    def set_solid_thermal_diff(self, diff):
        self.TS.thermal_diff, self.TS.derived = diff, False

    # D = kinetic_viscosity(i) / Pr per cell (the cell's viscosity, constant or Sutherland,
    # over its density for an ideal gas); thermal_diff keeps the value at rho = 1
    def set_fluid_Prandtl(self, Pr):
        self.TF.thermal_diff, self.TF.derived, self.TF.Pr = self.visco / Pr, False, float(Pr)

    # derived diffusivity D = cond(T) / (rho cm(T)) (src/LBM/LBM2D/_io.py:182-251,
    # _thermal.py:62-107, :167-210), evaluated per cell at its temperature by the kernels
    # (lbm_desc.tprop): the fluid divides by the cell's lattice density, the solid by its
    # density from add_rho_solid (uniform over the solid cells).  Each setter replaces the
    # phase's previous conductivity or capacity model, as the reference's do.
    def set_fluid_thermal_diff_derived(self):
        self.TF.derived, self.TF.Pr = True, None

    def set_fluid_conductivity(self, value):
        self.TF.cond, self.TF.cond_poly = float(value), None

    def set_fluid_conductivity_poly(self, poly):
        self.TF.cond, self.TF.cond_poly = None, [float(x) for x in poly]

    def set_fluid_capacity(self, value):
        self.TF.cm, self.TF.cm_poly, self.TF.nasa7 = float(value), None, None

    def set_fluid_capacity_poly(self, poly):
        self.TF.cm, self.TF.cm_poly, self.TF.nasa7 = None, [float(x) for x in poly], None

    def set_fluid_capacity_NASA7(self, Trange, data):
        self.TF.cm, self.TF.cm_poly, self.TF.nasa7 = None, None, (list(Trange), [list(r) for r in data])

    def set_solid_thermal_diff_derived(self):
        self.TS.derived = True

    def set_solid_conductivity(self, value):
        self.TS.cond, self.TS.cond_poly = float(value), None

    def set_solid_conductivity_poly(self, poly):
        self.TS.cond, self.TS.cond_poly = None, [float(x) for x in poly]

    def set_solid_capacity(self, value):
        self.TS.cm, self.TS.cm_poly, self.TS.nasa7 = float(value), None, None

    def set_solid_capacity_poly(self, poly):
        self.TS.cm, self.TS.cm_poly, self.TS.nasa7 = None, [float(x) for x in poly], None

    def set_solid_capacity_NASA7(self, Trange, data):
        self.TS.cm, self.TS.cm_poly, self.TS.nasa7 = None, None, (list(Trange), [list(r) for r in data])

    def _thermal_props(self, view: ScalarFieldView, solid: bool) -> dict:
        if (view.cond is None and view.cond_poly is None) or (view.cm is None and view.cm_poly is None
                                                               and view.nasa7 is None):
            raise ValueError(f"{view.name}: a derived diffusivity needs set_*_conductivity and set_*_capacity")
        return thermal_props(cond=view.cond, cond_poly=view.cond_poly, cap=view.cm, cap_poly=view.cm_poly,
                             nasa7=view.nasa7, solid=solid)

    def _temperature_dependent(self, view: ScalarFieldView) -> bool:
        return view.derived and (view.cond_poly is not None or view.cm_poly is not None or view.nasa7 is not None)

    def _derived_diff(self, view: ScalarFieldView, rho: float) -> float:
        """The phase's derived diffusivity at its reference temperature (T = 0, i.e. v_ref)
        and density rho: the constant tauT the descriptor also carries."""
        tp = self._thermal_props(view, view is self.TS)
        T = view.v_ref
        def nested(c):
            return c[0] + T * (c[1] + T * (c[2] * T + T * (c[3] + T * c[4])))
        cm = (nested(tp["cap_lo"]) if T < tp["cap_Tmid"] else nested(tp["cap_hi"])) * tp["cap_mul"]
        return nested(tp["cond"]) / rho / cm if cm != 0 else 0.0

    def _solid_density(self) -> float:
        s = self.solid._host >= 1
        r = self.rhos._host[s]
        if r.size == 0 or not np.all(r == r.flat[0]) or r.flat[0] <= 0:
            raise NotImplementedError("a derived solid diffusivity needs one positive solid density "
                                      "(add_rho_solid) on every solid cell on the CUDA path")
        return float(r.flat[0])

    def set_BC(self, i, bc):
        """Flow side type (src/LBM/LBM2D/_io.py:385-402)."""
        self.bc[i] = bc
        if bc == BC_FLOW.inlet or bc == BC_FLOW.inlet_flow or bc == BC_FLOW.wall:
            self.bc_v[i], self.bc_rho[i] = BC.fixedValue, BC.zeroGradient
        elif bc == BC_FLOW.outlet:
            self.bc_v[i], self.bc_rho[i] = BC.zeroGradient, BC.fixedValue
        elif bc == BC_FLOW.symmetric:
            self.bc_v[i], self.bc_rho[i] = BC.zeroGradient, BC.zeroGradient
        if bc == BC_FLOW.wall:
            self.v_BC[i] = (0.0, 0.0, 0.0)

    def set_BCs(self, bcs):
        for i, b in enumerate(bcs):
            self.set_BC(i, b)

    def set_v_BC(self, i, bc):
        self.bc_v[i] = bc

    def set_rho_BC(self, i, bc):
        self.bc_rho[i] = bc

    def set_v_BC_value(self, i, v):
        v = tuple(float(x) for x in (v if np.ndim(v) else (v, 0.0, 0.0)))
        self.v_BC[i] = (v + (0.0, 0.0, 0.0))[:3]
        self._push_sides()

    def set_rho_BC_value(self, i, r):
        self.rho_BC[i] = float(r)
        self._push_sides()

    def set_flow_BC_value(self, i, f):
        self.flow_BC[i] = float(f)
        self._push_sides()

    def set_flow_BCs_value(self, fs):
        for i, f in enumerate(fs):
            self.set_flow_BC_value(i, f)

    def set_TF_BC(self, i, bc):
        self.TF.set_BC(i, bc)

    def set_TF_BC_value(self, i, T):
        self.TF.set_s_BC_value(i, T)
        self._push_sides()

    def set_TS_BC(self, i, bc):
        self.TS.set_BC(i, bc)

    def set_TS_BC_value(self, i, T):
        self.TS.set_s_BC_value(i, T)

    def set_heat_exchange_surface(self, surface):
        """Exchange surface of the porous cells (src/LBM/LBM2D/_io.py:133-135)."""
        self.init_field(self.TS.exchangeSurface, surface)

    def set_heat_exchange_coef(self, coef):
        """Exchange coefficient of the porous cells (src/LBM/LBM2D/_io.py:136-138)."""
        self.init_field(self.TS.exchangeCoef, coef)

    def set_poro_Darcy(self, s, coefDarcy):
        """Darcy drag in the porous cells (src/LBM/LBM2D/_io.py:152-164): the coefficient
        (1/length^2) scaled by dx^2 over the zone s."""
        self._need_poro()
        self.poro_model = PORO_MODEL.DARCY
        coefDarcy = coefDarcy * self.dx ** 2
        self.init_field(self.coefDarcy, coefDarcy * np.asarray(s, dtype=np.float64))

    def set_poro_Darcy_Forchheimer(self, s, coefDarcy, coefForchheimer):
        """Darcy-Forchheimer drag (src/LBM/LBM2D/_io.py:165-172): coefficients scaled by dx^2
        and dx over the zone s."""
        self._need_poro()
        self.poro_model = PORO_MODEL.DARCYFORCHHEIMER
        coefDarcy = coefDarcy * self.dx ** 2
        coefForchheimer = coefForchheimer * self.dx
        self.init_field(self.coefDarcy, coefDarcy * np.asarray(s, dtype=np.float64))
        self.init_field(self.coefForchheimer, coefForchheimer * np.asarray(s, dtype=np.float64))

    def _need_poro(self):
        if not self.PORO:
            raise ValueError("porous setters need the solver created with isPoro=True")

    def set_specie(self, *a, **k):
        raise NotImplementedError("species transport is not on the CUDA path; use set_pyrolysis()")

    def set_radiation(self, model, param):
        """Surface radiation of the porous cells to the ambient temperature ``param`` (K)
        (src/LBM/LBM2D/_io.py:259-271, _thermal.py:213-220); needs isRadiation."""
        if model == RADIATION_MODEL.SURFACE_UNIFORM:
            self.TS.radiation_model = model
            self.TS.Tambient = float(param)
        elif model != RADIATION_MODEL.NONE:
            raise NotImplementedError(f"radiation model {model} is not on the CUDA path (SURFACE_UNIFORM is)")

    def add_reaction(self, *a, **k):
        raise NotImplementedError("general reaction networks are not on the CUDA path; use set_pyrolysis()")

    def load_cantera(self, file):
        raise NotImplementedError("Cantera mechanisms are not on the CUDA path; use set_pyrolysis()")

    def load_stl(self, stl_path, scale=(1.0, 1.0, 1.0), translate=(0, 0, 0), rotate=(0, 0, 0), **kwargs):
        """(voxel_array, surface_array) of an STL mesh on this lattice
        (src/LBM/LBM2D/_io.py:489-495), voxelised on the GPU (lbm_porouschem_b200.stl)."""
        from .stl import StlReader
        r = StlReader(self.X, self.Y, self.Z, self.dx, self.DIM, logger=kwargs.get("logger"))
        return r.voxel_stl(stl_path, scale, translate, rotate)

    # ------------------------------------------------------------ new settings of the CUDA path
    def set_body_force(self, g, half_force_velocity: bool = True):
        """Constant body acceleration (lattice units); u includes F/2 by default."""
        self.body_force = tuple(float(x) for x in g) + (0.0,) * (3 - len(g))
        self.half_force_velocity = half_force_velocity
        self.force_term_model = FORCE_TERM.GUO

    def set_collision(self, model: str):
        self.collision = model.lower()

    def set_precision(self, precision: str):
        self.precision = precision.lower()

    def set_pyrolysis(self, A=1e8, Ea=1.25e5, b=0.0, dH=4e5, capacity=1000.0, rho_solid=1.0,
                      char_yield=0.25, alpha_flip=0.01, Tmin=0.0, reactive=None):
        """Single-step pyrolysis of reactive solid cells: rate A (T+1e-6)^b exp(-Ea/(R T)) at the
        cell temperature (K), endothermic dH (J/kg), gas fraction 1 - char_yield released to
        the fluid, the cell turns fluid below reactive fraction ``alpha_flip``.  ``reactive``:
        mask of reactive cells (default: every solid cell)."""
        if not self.TEMPERATURE:
            raise ValueError("pyrolysis needs the temperature field (isThermal=True)")
        self._pyro = dict(A=A, Ea=Ea, b=b, dH=dH, capacity=capacity, rho_solid=rho_solid,
                          char_yield=char_yield, alpha_flip=alpha_flip, Tmin=Tmin)
        if reactive is not None:
            self._reactive = np.asarray(reactive, dtype=bool).reshape(self._shape)

    # ------------------------------------------------------------ configuration
    def _thermal_mode(self) -> str:
        """The reference's TF / TS fields (adiabatic interface), or the conjugate field
        that pyrolysis needs (the reacting solid is heated through the interface)."""
        if not self.TEMPERATURE:
            return "none"
        return "conjugate" if self._pyro else "two_field"

    def _nu_lu(self) -> float:
        return self.visco * self.dt / self.dx ** 2

    def _tau_T(self, diff) -> float:
        D = diff * self.dt / self.dx ** 2
        return (3.0 if self.DIM == 2 else 4.0) * D + 0.5   # _scalarField.py:56-58 (2D/3D)

    def _sides(self) -> list:
        sides = [SideBC() for _ in range(6)]
        for i in range(self._nsides):
            vt, rt, Tt = _BC_CODE[self.bc_v[i]], _BC_CODE[self.bc_rho[i]], _BC_CODE[self.TF.BC[i]]
            if not self.TEMPERATURE:
                Tt = PERIODIC
            if self.boundary_condition_model == BC_MODEL.NONE:
                active = False
            elif self.boundary_condition_model in (BC_MODEL.NEE, BC_MODEL.ES):
                active = self.ref_quirk_nee_on_periodic or (vt, rt, Tt) != (PERIODIC, PERIODIC, PERIODIC)
            elif self.boundary_condition_model == BC_MODEL.NEBB:
                # Boundary_condition_NEBB (src/LBM/LBM2D/_boundary.py:103-226): the flow sides
                # that are walls, inlets or outlets; 2D only (the 3D solver has none) and the
                # scalar NEBB boundary reads the previous step's macro fields
                if self.DIM != 2 or self.TEMPERATURE:
                    raise NotImplementedError("NEBB is on the CUDA path in 2D without the temperature field")
                active = (vt, rt) != (PERIODIC, PERIODIC)
            else:
                raise NotImplementedError(f"{self.boundary_condition_model} is not on the CUDA path")
            v = self.v_BC[i]
            if self.bc[i] == BC_FLOW.inlet_flow and vt == FIXED_VALUE:
                # the reference sets an inlet profile for side 0 only
                # (src/LBM/LBM2D/_initialize.py:67-73, LBM3D/_initialize.py:78-85); the
                # 2D solver steers it each step (LBM2D/_boundary.py:324-333), the 3D one
                # keeps v0 = F/ny/nz (LBM3D/_boundary.py:12-14 only runs user callbacks)
                v = (0.0, 0.0, 0.0)
                if i == 0 and self.DIM == 2:
                    vt, v = FLOW_RATE, (self.flow_BC[0], 0.0, 0.0)
                elif i == 0:
                    v = (self.flow_BC[0] / self.ny / self.nz, 0.0, 0.0)
            model = {BC_MODEL.ES: "es", BC_MODEL.NEBB: "nebb"}.get(self.boundary_condition_model, "nee")
            sides[i] = SideBC(active, vt, rt, Tt, v, self.rho_BC[i], self.TF.s_BC[i], model)
        return sides

    def _config(self) -> LatticeConfig:
        if self.viscosity_model not in (VISCOSITY_MODEL.CONSTANT, VISCOSITY_MODEL.NONE, VISCOSITY_MODEL.SUTHERLAND):
            raise NotImplementedError(f"{self.viscosity_model} is not on the CUDA path")
        cfg = LatticeConfig(
            dim=self.DIM, nx=self.nx, ny=self.ny, nz=self.nz, collision=self.collision, precision=self.precision,
            eos="ideal_gas" if self.EOS == FLUID_STATE_EQUATION.IDEAL_GAS else "incompressible",
            nu=self._nu_lu(), force=self.body_force, half_force_velocity=self.half_force_velocity,
            thermal=self._thermal_mode(), sides=self._sides())
        if self.TEMPERATURE:
            dF = self._derived_diff(self.TF, 1.0) if self.TF.derived else self.TF.thermal_diff
            dS = self._derived_diff(self.TS, self._solid_density()) if self.TS.derived else self.TS.thermal_diff
            cfg.tauT_fluid = self._tau_T(dF)
            cfg.tauT_solid = self._tau_T(dS)
            cfg.T_ref, cfg.T_scale = self.TF.v_ref, self.TF.v_scale
            porous = bool(np.any((self.solid._host > 0) & (self.solid._host < 1)))
            if porous and (self._temperature_dependent(self.TF) or self._temperature_dependent(self.TS)):
                raise NotImplementedError("temperature-dependent conductivity or capacity with porous cells is not "
                                          "on the CUDA path (their heat exchange uses constant capacities)")
            if not porous and self.TF.Pr is not None:
                cfg.tp_prandtl = self.TF.Pr
            if not porous and (self.TF.derived or self.TS.derived):
                # per cell at its temperature and (fluid) density, _thermal.py:62-71, :167-174
                if self.TF.derived:
                    cfg.tprop_fluid = self._thermal_props(self.TF, False)
                if self.TS.derived:
                    cfg.tprop_solid = self._thermal_props(self.TS, True)
                    cfg.tp_rhos = self._solid_density()
                cfg.Ts_ref, cfg.Ts_scale = self.TS.v_ref, self.TS.v_scale
                cfg.tp_dt, cfg.tp_dx2 = self.dt, self.dx ** 2
                # the constant rates are not used where tprop is set; keep them valid
                if cfg.tprop_fluid is not None and not cfg.tauT_fluid > 0.5:
                    cfg.tauT_fluid = 1.0
                if cfg.tprop_solid is not None and not cfg.tauT_solid > 0.5:
                    cfg.tauT_solid = 1.0
        if self.viscosity_model == VISCOSITY_MODEL.SUTHERLAND:
            # src/LBM/LBM2D/_evolution.py:232-234 at GetTF (:304-307): the fluid
            # temperature, or 273.15 K without the temperature field
            As, Ts = self.sutherland_coef
            if self.TEMPERATURE:
                cfg.viscosity, cfg.suth_A, cfg.suth_Ts = "sutherland", As * self.dt / self.dx ** 2, Ts
            else:
                cfg.nu = As * 273.15 ** 1.5 / (273.15 + Ts) * self.dt / self.dx ** 2
        s = self.solid._host
        if np.any((s > 0) & (s < 1)):
            if not self.PORO:
                raise ValueError("cells with a solid fraction between 0 and 1 need isPoro=True")
            model = {PORO_MODEL.SPHERICAL: "ergun", PORO_MODEL.ERGUN: "ergun", PORO_MODEL.DARCY: "darcy",
                     PORO_MODEL.DARCYFORCHHEIMER: "darcy_forchheimer"}.get(self.poro_model)
            if model is None:
                raise NotImplementedError(f"{self.poro_model} is not on the CUDA path")
            if self.TEMPERATURE:
                if self._pyro:
                    raise NotImplementedError("pyrolysis with porous cells is not on the CUDA path")
                # two fields in a porous cell, exchanging heat there and radiating
                # (src/LBM/LBM2D/_evolution.py:186-202)
                cfg.Ts_ref, cfg.Ts_scale = self.TS.v_ref, self.TS.v_scale
                cfg.cap_fluid = 1000.0 if self.TF.cm is None else self.TF.cm   # capacity_m defaults,
                cfg.cap_solid = 1000.0 if self.TS.cm is None else self.TS.cm   # _thermal.py:18, :128
                cfg.dt_phys, cfg.dx_phys = self.dt, self.dx
                if self.RADIATION and self.TS.radiation_model == RADIATION_MODEL.SURFACE_UNIFORM:
                    cfg.radiation, cfg.T_ambient = True, self.TS.Tambient
            cfg.porous = model
        if self._pyro:
            pz = self._pyro
            cfg.pyro = True
            cfg.pyro_A, cfg.pyro_Ea, cfg.pyro_b, cfg.pyro_Tmin = pz["A"], pz["Ea"], pz["b"], pz["Tmin"]
            cfg.dt_phys = self.dt
            cfg.heat_norm = pz["dH"] / (pz["capacity"] * cfg.T_scale)
            cfg.gas_coef = (1.0 - pz["char_yield"]) * pz["rho_solid"]
            cfg.alpha_flip = pz["alpha_flip"]
        return cfg

    # ------------------------------------------------------------ run
    def init_simulation(self, device: str = "cuda"):
        """Equilibrium initialisation (src/LBM/LBM2D/_initialize.py:16-65) on the GPU."""
        from .lattice import Lattice
        s = self.solid._host
        solid = s >= 1
        cfg = self._config()
        reactive = None
        if cfg.pyro:
            reactive = solid if self._reactive is None else (self._reactive & solid)
        self._cfg = cfg
        self._lat = Lattice(cfg, device=device)
        self._lat.set_geometry(solid, reactive)
        if cfg.porous != "none":
            frac = np.where(solid, 0.0, s)
            heat = {}
            if cfg.porous_heat:
                heat = dict(h=self.TS.exchangeCoef._host, a=self.TS.exchangeSurface._host, rho_solid=self.rhos._host,
                            emissivity=self.TS.emissivity._host, radiation_surface=self.TS.radiation_surface._host)
            self._lat.set_porous(frac, self.coefDarcy._host, self.coefForchheimer._host, **heat)
        u = np.moveaxis(self.v._host, -1, 0)
        two = cfg.thermal == "two_field"
        self._lat.init(rho=self.rho._host, u=u, T=self.TF.S._host if self.TEMPERATURE else 0.0,
                       Ts=self.TS.S._host if two else None)
        self._cache = None
        self._cache_step = -1

    def updateBC(self, t):
        for func in self.UpdateBCfunc:
            func(self, t)

    def step(self):
        """One lattice step (src/LBM/LBM2D/_evolution.py:12-15)."""
        if self._lat is None:
            raise RuntimeError("call init_simulation() first")
        self.updateBC(self.t)
        self._lat.step(1)
        self.tLattice += 1
        self.t = self.tLattice * self.dt

    def _push_sides(self):
        if getattr(self, "_lat", None) is not None:
            self._lat.set_sides(self._sides())

    def _state(self) -> dict:
        if self._cache_step != self._lat.nsteps:
            self._cache = self._lat.fields()
            self._cache_step = self._lat.nsteps
        return self._cache

    def _read_field(self, name: str, host: np.ndarray) -> np.ndarray:
        if self._lat is None:
            return host.copy()
        st = self._state()
        if name == "rho":
            out = host.copy()
            fl = ~st["solid"]
            out[fl] = st["rho"][fl]
            return out
        if name == "v":
            out = host.copy()
            fl = ~st["solid"]
            out[fl] = np.moveaxis(st["u"], 0, -1)[fl]
            out[~fl] = 0.0
            return out
        if name == "solid":
            return st["solid"].astype(np.float64)
        if name == "TS" and "Ts" in st:   # porous cells carry a TS of their own
            return np.where(self.solid._host > 0, st["Ts"], st["T"])
        if name in ("TF", "TS"):
            return st["T"].copy()
        return host.copy()

    # ------------------------------------------------------------ output (src/LBM/LBM2D/_io.py:538-598)
    def _diag(self) -> dict:
        if self._lat is None or self._lat.nsteps == 0:
            fl = self.solid._host < 1
            u = np.linalg.norm(self.v._host, axis=-1)
            T = self.TF.S._host
            return {"umax": float(u[fl].max(initial=0.0)), "Tmin": float(T.min()), "Tmax": float(T.max())}
        return self._lat.diagnostics()

    def get_max_v(self):
        return self._diag()["umax"]

    def get_max_T(self):
        return self.TF.get_physical_value(self._diag()["Tmax"]) if self.TEMPERATURE else -1

    def get_min_T(self):
        return self.TF.get_physical_value(self._diag()["Tmin"]) if self.TEMPERATURE else -1

    def log_info(self) -> str:
        d = self._diag()
        p = f"    t(LU)={self.tLattice} : Max velocity magnitude (LU) : {d['umax']:.7f}, "
        if self.TEMPERATURE:
            p += (f"Min temperature: {self.TF.get_physical_value(d['Tmin']):.7f} K, "
                  f"Max temperature : {self.TF.get_physical_value(d['Tmax']):.7f}")
        return p

    def export_snapshot(self, config=None) -> Optional[str]:
        """Checkpoint of the lattice state (Lattice.save_checkpoint) to
        ``<snapshotPath stem>_<tLattice>.npz``; ``load_snapshot`` continues from it bit for
        bit.  The reference reserves this call for a binary dump and leaves it empty
        (src/LBM/LBM2D/_io.py:589-598)."""
        if self._lat is None:
            return None
        stem = os.path.splitext(self.snapshotPath)[0] if self.snapshotPath else self.name
        path = f"{stem}_{self.tLattice}.npz"
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        return self._lat.save_checkpoint(path)

    def load_snapshot(self, path: str, device="cuda") -> None:
        """Continue from a checkpoint written by ``export_snapshot`` (in place of
        init_simulation; no reference counterpart).  The checkpoint's lattice settings
        replace this solver's."""
        from .lattice import Lattice
        if self._lat is not None:
            self._lat.close()
        self._lat = Lattice.load_checkpoint(path, device=device)
        self._cfg = self._lat.cfg
        self.tLattice = self._lat.nsteps
        self.t = self.tLattice * self.dt
        self._cache = None
        self._cache_step = -1

    def check_python(self):
        pass

    def export_VTK_pyvista(self) -> str:
        """``exportPath/name_<tLattice>.vts`` and the ``exportPath/name.pvd`` time series
        (src/LBM/LBM2D/_io.py:621-635), written without pyvista (lbm_porouschem_b200.vtk).
        Point data under the reference's names: solid, rho, velocity and, with the
        temperature field, Tf and Ts in K (one field here: equal arrays); with pyrolysis
        also the reactive fraction alpha."""
        os.makedirs(self.exportPath, exist_ok=True)
        data = {"solid": self.solid.to_numpy(), "rho": self.rho.to_numpy(), "velocity": self.v.to_numpy()}
        if self.TEMPERATURE:
            T = self.TF.get_physical_value(self.TF.S.to_numpy())
            data["Tf"] = T
            data["Ts"] = T
        if self._lat is not None and self._lat.cfg.pyro and self._lat.nsteps > 0:
            data["alpha"] = self._state()["alpha"]
        fn = os.path.join(self.exportPath, f"{self.name}_{self.tLattice}.vts")
        write_vts(fn, data, self._shape, coords=(self.x, self.y, self.z))
        self.PVD.exportPath = self.exportPath
        self.PVD.add(self.tLattice * self.dt, os.path.basename(fn))
        self.PVD.write()
        return fn

    def close(self):
        if self._lat is not None:
            self._lat.close()
            self._lat = None


def _unsupported(name: str, why: str):
    def method(self, *a, **k):
        raise NotImplementedError(f"{name}: {why}")
    method.__name__ = name
    method.__doc__ = f"Reference setter (src/LBM/LBM2D/_io.py) that raises here: {why}."
    return method


_SPECIES = "species transport is not on the CUDA path; use set_pyrolysis()"
for _n, _why in [
    ("set_fluid_conductivity_mixture", _SPECIES), ("set_fluid_capacity_mixture", _SPECIES),
    ("set_solid_conductivity_mixture", _SPECIES), ("set_solid_capacity_mixture", _SPECIES),
    ("set_specie_viscosity", _SPECIES), ("set_specie_viscosity_sutherland", _SPECIES),
    ("set_specie_diff", _SPECIES), ("set_specie_diff_Schmidt", _SPECIES), ("set_specie_capacity", _SPECIES),
    ("set_specie_enthalpy", _SPECIES), ("set_specie_NASA7", _SPECIES), ("set_specie_conductivity", _SPECIES),
    ("set_specie_conductivity_poly", _SPECIES), ("set_specie_BC", _SPECIES), ("set_specie_BC_value", _SPECIES),
    ("set_species_BC", _SPECIES), ("init_specie", _SPECIES),
]:
    setattr(_SolverBase, _n, _unsupported(_n, _why))


class LBM2DSolver(_SolverBase):
    """2D solver (D2Q9 flow + D2Q5 temperature) with the reference constructor
    (src/LBM/LBM2D/__init__.py:65-70)."""
    DIM = 2


class LBM3DSolver(_SolverBase):
    """3D solver (D3Q19 flow + D3Q7 temperature) with the reference constructor
    (src/LBM/LBM3D/__init__.py:11-62)."""
    DIM = 3
