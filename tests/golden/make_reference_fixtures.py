"""Generate golden fixtures by running LBM_porousChem's own solver code on small lattices.

TEST INFRASTRUCTURE ONLY (run by hand in a checkout that has the reference next to it; the
fixtures it writes are committed and the tests read only those):

    python tests/golden/make_reference_fixtures.py /path/to/LBM_porousChem

The reference is Python + Taichi 1.7.4, and Taichi is not installable here, so the script
puts ``tests/golden/standin`` (a sequential NumPy stand-in for the Taichi subset the solver
uses, plus empty ``pyevtk``/``pyvista``/``ruamel.yaml`` modules its I/O file imports) ahead
of ``<reference>/src`` on ``sys.path`` and drives the **unmodified** ``LBM.LBM2D.LBM2DSolver``
/ ``LBM.LBM3D.LBM3DSolver`` through their own setters, exactly as ``src/LBM/app.py:101-677``
does: constructor, ``set_viscosity``, ``set_BC``..., ``init_field``/``init_field3``/
``add_solid``, ``init_simulation()``, then ``step()`` N times.  Real type: float64.

Each case also records the ``LatticeConfig`` that describes the same run to this package
(``meta``), with the mapping rules written next to it:

* ``set_viscosity(mu)`` with dx = dt = 1 -> ``nu = mu`` (``LBM2D/_evolution.py:227-249``);
  IDEAL_GAS, so tau = 3 nu/rho + 1/2 in both.
* thermal diffusivity D -> ``tauT = 3 D + 1/2`` (2D) / ``4 D + 1/2`` (3D),
  ``_scalarField.py:56-58``; the fixture computes tauT with the same expression.
* ``BC_FLOW.inlet`` / ``outlet`` / ``wall`` -> ``SideBC.inlet`` / ``outlet`` / ``wall``
  (``LBM2D/_io.py:385-402``); under ``BC_MODEL.NEE`` every side is extrapolated, so sides the
  case leaves periodic are active with PERIODIC types (``ref_quirk_nee_on_periodic``).
* 3D side 4 (z = 0) "zero-gradient" density assigns the cell to itself
  (``LBM3D/_boundary.py:128``), i.e. keeps the cell's own density: PERIODIC density type.
* two-field temperature on a binary mask: fluid cells carry ``TF``, solid cells ``TS``;
  ``macro`` skips solid cells, so ``TS`` there is never refreshed from the streamed
  populations (``LBM2D/_evolution.py:119``): ``ref_quirk_frozen_solid_T``.

Every input is float32-representable (``init_field`` of a constant goes through float32,
``LBM2D/_io.py:49-51``, and the CUDA path takes float32 initial fields).
"""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from lbm_porouschem_b200.config import (FIXED_VALUE, PERIODIC, ZERO_GRADIENT,  # noqa: E402
                                        LatticeConfig, SideBC, thermal_props)


def _import_reference(ref_root: str):
    sys.path.insert(0, str(HERE / "standin"))
    sys.path.insert(1, os.path.join(ref_root, "src"))
    from LBM.LBM2D import LBM2DSolver
    from LBM.LBM3D import LBM3DSolver
    from LBM.util import flag
    return LBM2DSolver, LBM3DSolver, flag


# --------------------------------------------------------------------------- inputs
def _disks(shape, n, rmin, rmax, margin_x, seed):
    """Binary mask of ``n`` seeded disks (circles in 2D, spheres in 3D) kept ``margin_x`` cells
    away from the x sides (those are the active sides of the channel cases)."""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    m = np.zeros(shape, dtype=bool)
    for _ in range(n):
        r = rng.uniform(rmin, rmax)
        c = [rng.uniform(margin_x + r, shape[0] - 1 - margin_x - r)]
        c += [rng.uniform(0, s) for s in shape[1:]]
        d2 = sum((g - cc) ** 2 for g, cc in zip(grids, c))
        m |= d2 <= r * r
    return m


def _smooth_field(shape, seed, amp):
    """float32-representable smooth random perturbation."""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    out = np.zeros(shape)
    for _ in range(3):
        k = [rng.integers(1, 3) * 2 * np.pi / s for s in shape]
        ph = rng.uniform(0, 2 * np.pi)
        out += np.cos(sum(kk * g for kk, g in zip(k, grids)) + ph)
    return (amp * out / 3).astype(np.float32).astype(np.float64)


# --------------------------------------------------------------------------- cases
def _common_inputs(shape, seed, solid, u_amp=0.02, rho_amp=0.002, T0=None):
    nd = len(shape)
    rho = (1.0 + _smooth_field(shape, seed, rho_amp)).astype(np.float32).astype(np.float64)
    u = np.stack([_smooth_field(shape, seed + 1 + d, u_amp) if d < nd else np.zeros(shape)
                  for d in range(3)])
    u[:, solid] = 0.0
    T = np.zeros(shape) if T0 is None else T0
    return rho, u, T


def case_periodic2d():
    shape = (16, 12, 1)
    solid = _disks(shape[:2], 3, 1.5, 2.5, 0, 1)[..., None]
    rho, u, T = _common_inputs(shape, 11, solid)
    cfg = LatticeConfig(dim=2, nx=16, ny=12, nz=1, collision="bgk", precision="fp64", nu=0.1)
    return dict(name="ref_periodic2d", cfg=cfg, bc_model="NONE", solid=solid, rho=rho, u=u, T=T,
                steps=60, thermal=None, sides=None)


def _channel_sides(flag, dim, u_in, rho_out, thermal):
    """inlet at x = 0, outlet at x = nx-1, walls on the other sides (2D: y; 3D: y and z)."""
    T_in = 1.0
    ref = {0: ("inlet", (u_in, 0.0, 0.0), None), 1: ("outlet", None, rho_out)}
    for s in range(2, 2 * dim):
        ref[s] = ("wall", None, None)
    tbc = {0: ("fixed", T_in), 1: ("zero", None)}
    for s in range(2, 2 * dim):
        tbc[s] = ("zero", None)
    Tt = lambda s: (FIXED_VALUE if tbc[s][0] == "fixed" else ZERO_GRADIENT) if thermal else PERIODIC
    sides = [SideBC() for _ in range(6)]
    sides[0] = SideBC.inlet((u_in, 0.0, 0.0), Tt(0), T_in)
    sides[1] = SideBC.outlet(rho_out, Tt(1), 0.0)
    for s in range(2, 2 * dim):
        sides[s] = SideBC.wall(Tt(s), 0.0)
    if dim == 3:
        sides[4].rho_type = PERIODIC   # LBM3D/_boundary.py:128 self-assignment
    return ref, tbc, sides


def case_channel2d_thermal():
    nx, ny = 20, 12
    shape = (nx, ny, 1)
    solid = np.zeros(shape, dtype=bool)
    solid[:, 2:ny - 2, 0] = _disks((nx, ny - 4), 3, 1.5, 2.2, 3, 2)
    T0 = (_smooth_field(shape, 23, 0.2) + 0.3).astype(np.float32).astype(np.float64)
    rho, u, T = _common_inputs(shape, 21, solid, T0=T0)
    Df, Ds = 1.0 / 30.0, 0.1
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision="bgk", precision="fp64", nu=0.1,
                        thermal="two_field", tauT_fluid=3 * Df + .5, tauT_solid=3 * Ds + .5)
    return dict(name="ref_channel2d_thermal", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u,
                T=T, steps=60, thermal=(Df, Ds), channel=(0.03, 1.0))


def case_channel2d_es():
    d = case_channel2d_thermal()
    d["name"] = "ref_channel2d_es"
    d["bc_model"] = "ES"
    d["steps"] = 40
    return d


def case_nee_periodic2d():
    """NEE model with the y sides left periodic: the reference extrapolates them anyway."""
    nx, ny = 18, 10
    shape = (nx, ny, 1)
    solid = np.zeros(shape, dtype=bool)
    solid[:, 2:ny - 2, 0] = _disks((nx, ny - 4), 2, 1.5, 2.0, 3, 5)
    rho, u, T = _common_inputs(shape, 31, solid)
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision="bgk", precision="fp64", nu=0.12)
    return dict(name="ref_nee_periodic2d", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u, T=T,
                steps=50, thermal=None, channel=(0.02, 1.0), periodic_y=True)


def case_periodic3d():
    shape = (10, 8, 8)
    solid = _disks(shape, 2, 1.5, 2.2, 0, 7)
    rho, u, T = _common_inputs(shape, 41, solid)
    cfg = LatticeConfig(dim=3, nx=10, ny=8, nz=8, collision="bgk", precision="fp64", nu=0.1)
    return dict(name="ref_periodic3d", cfg=cfg, bc_model="NONE", solid=solid, rho=rho, u=u, T=T,
                steps=24, thermal=None)


def case_channel3d_thermal():
    nx, ny, nz = 12, 8, 8
    shape = (nx, ny, nz)
    solid = np.zeros(shape, dtype=bool)
    solid[:, 2:ny - 2, 2:nz - 2] = _disks((nx, ny - 4, nz - 4), 2, 1.2, 1.8, 3, 8)
    T0 = (_smooth_field(shape, 53, 0.2) + 0.3).astype(np.float32).astype(np.float64)
    rho, u, T = _common_inputs(shape, 51, solid, T0=T0)
    Df, Ds = 0.025, 0.1
    cfg = LatticeConfig(dim=3, nx=nx, ny=ny, nz=nz, collision="bgk", precision="fp64", nu=0.1,
                        thermal="two_field", tauT_fluid=4 * Df + .5, tauT_solid=4 * Ds + .5)
    return dict(name="ref_channel3d_thermal", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u,
                T=T, steps=20, thermal=(Df, Ds), channel=(0.03, 1.0))


def case_periodic3d_x32():
    """32 x 8 x 8: a shape the dense (TMA-staged) 3D bulk form runs too."""
    shape = (32, 8, 8)
    solid = _disks(shape, 3, 1.5, 2.2, 0, 9)
    rho, u, T = _common_inputs(shape, 61, solid)
    cfg = LatticeConfig(dim=3, nx=32, ny=8, nz=8, collision="bgk", precision="fp64", nu=0.1)
    return dict(name="ref_periodic3d_x32", cfg=cfg, bc_model="NONE", solid=solid, rho=rho, u=u, T=T,
                steps=16, thermal=None)


def case_channel3d_flow_x32():
    """NEE channel without temperature, 32 x 8 x 8 (dense-form shape)."""
    nx, ny, nz = 32, 8, 8
    shape = (nx, ny, nz)
    solid = np.zeros(shape, dtype=bool)
    solid[:, 2:ny - 2, 2:nz - 2] = _disks((nx, ny - 4, nz - 4), 3, 1.2, 1.8, 3, 10)
    rho, u, T = _common_inputs(shape, 71, solid)
    cfg = LatticeConfig(dim=3, nx=nx, ny=ny, nz=nz, collision="bgk", precision="fp64", nu=0.1)
    return dict(name="ref_channel3d_flow_x32", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u, T=T,
                steps=16, thermal=None, channel=(0.03, 1.0))


def _porous_zone(shape, centre, r):
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    return sum((g - c) ** 2 for g, c in zip(grids, centre)) <= r * r


def case_porous2d_darcy():
    """NEE channel with a porous cylinder (DARCY), like examples/2D/cylinder_poro."""
    nx, ny = 24, 12
    shape = (nx, ny, 1)
    zone = _porous_zone((nx, ny), (10.3, 5.7), 3.6)[..., None]
    solid = np.zeros(shape, dtype=bool)
    rho, u, T = _common_inputs(shape, 81, solid)
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision="bgk", precision="fp64", nu=0.1, porous="darcy")
    return dict(name="ref_porous2d_darcy", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u, T=T, steps=60,
                thermal=None, channel=(0.03, 1.0), porous=dict(model="darcy", zone=zone, eps=0.6, darcy=0.5))


def case_porous2d_ergun():
    """Periodic flow through a porous blob (default SPHERICAL model: Ergun from the
    porosity) next to an impermeable disk."""
    shape = (16, 12, 1)
    zone = _porous_zone((16, 12), (5.2, 6.1), 3.3)[..., None]
    solid = _porous_zone((16, 12), (12.4, 4.0), 2.1)[..., None] & ~zone
    rho, u, T = _common_inputs(shape, 91, solid)
    cfg = LatticeConfig(dim=2, nx=16, ny=12, nz=1, collision="bgk", precision="fp64", nu=0.1, porous="ergun")
    return dict(name="ref_porous2d_ergun", cfg=cfg, bc_model="NONE", solid=solid, rho=rho, u=u, T=T, steps=60,
                thermal=None, porous=dict(model="ergun", zone=zone, eps=0.5))


def case_porous3d_df():
    """3D NEE channel with a porous sphere (DARCYFORCHHEIMER; the 3D drag uses viscosity(i))."""
    nx, ny, nz = 12, 8, 8
    shape = (nx, ny, nz)
    zone = _porous_zone(shape, (5.6, 3.6, 3.6), 1.9)
    solid = np.zeros(shape, dtype=bool)
    rho, u, T = _common_inputs(shape, 101, solid)
    cfg = LatticeConfig(dim=3, nx=nx, ny=ny, nz=nz, collision="bgk", precision="fp64", nu=0.1,
                        porous="darcy_forchheimer")
    return dict(name="ref_porous3d_df", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u, T=T, steps=20,
                thermal=None, channel=(0.03, 1.0),
                porous=dict(model="darcy_forchheimer", zone=zone, eps=0.7, darcy=0.5, forch=0.3))


def _border(zone):
    """Zone cells with a face neighbour outside the zone, weight 1: the surface weights the
    driver takes from the zone's geometry for radiation (src/LBM/app.py:545-566)."""
    b = np.zeros(zone.shape, dtype=bool)
    for ax in range(zone.ndim):
        if zone.shape[ax] == 1:
            continue
        for sh in (1, -1):
            b |= zone & ~np.roll(zone, sh, axis=ax)
    return b.astype(np.float64)


def case_porous2d_heat():
    """NEE channel through a porous cylinder (DARCY) with two temperature fields: TF and TS
    exchange heat in the porous cells (src/LBM/LBM2D/_evolution.py:186-200), whose surface
    also radiates (SURFACE_UNIFORM, :201-202); TS starts apart from TF and has its own
    temperature range and capacity."""
    nx, ny = 24, 12
    shape = (nx, ny, 1)
    zone = _porous_zone((nx, ny), (10.3, 5.7), 3.6)[..., None]
    solid = np.zeros(shape, dtype=bool)
    T0 = (_smooth_field(shape, 113, 0.2) + 0.3).astype(np.float32).astype(np.float64)
    Ts0 = (_smooth_field(shape, 117, 0.15) + 0.45).astype(np.float32).astype(np.float64)
    rho, u, T = _common_inputs(shape, 111, solid, T0=T0)
    Df, Ds = 1.0 / 30.0, 0.1
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision="bgk", precision="fp64", nu=0.1, porous="darcy",
                        thermal="two_field", tauT_fluid=3 * Df + .5, tauT_solid=3 * Ds + .5,
                        T_ref=300.0, T_scale=500.0, Ts_ref=250.0, Ts_scale=600.0, cap_fluid=1200.0,
                        cap_solid=800.0, dt_phys=1.0, dx_phys=1.0, radiation=True, T_ambient=350.0)
    return dict(name="ref_porous2d_heat", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u, T=T, steps=60,
                thermal=(Df, Ds), channel=(0.03, 1.0), porous=dict(model="darcy", zone=zone, eps=0.6, darcy=0.5),
                heat=dict(h=3.0, a=1.0, rhos=2.0, emis=0.8, Ts0=Ts0))


def case_porous3d_heat():
    """3D NEE channel through a porous sphere (SPHERICAL: Ergun from the porosity) with two
    temperature fields exchanging heat in it (LBM3D/_evolution.py:179-193), no radiation."""
    nx, ny, nz = 12, 8, 8
    shape = (nx, ny, nz)
    zone = _porous_zone(shape, (5.4, 3.7, 3.4), 2.1)
    solid = np.zeros(shape, dtype=bool)
    T0 = (_smooth_field(shape, 123, 0.2) + 0.3).astype(np.float32).astype(np.float64)
    Ts0 = (_smooth_field(shape, 127, 0.1) + 0.6).astype(np.float32).astype(np.float64)
    rho, u, T = _common_inputs(shape, 121, solid, T0=T0)
    Df, Ds = 0.025, 0.1
    cfg = LatticeConfig(dim=3, nx=nx, ny=ny, nz=nz, collision="bgk", precision="fp64", nu=0.1, porous="ergun",
                        thermal="two_field", tauT_fluid=4 * Df + .5, tauT_solid=4 * Ds + .5,
                        T_ref=300.0, T_scale=500.0, Ts_ref=280.0, Ts_scale=450.0, cap_fluid=1000.0,
                        cap_solid=700.0, dt_phys=1.0, dx_phys=1.0)
    return dict(name="ref_porous3d_heat", cfg=cfg, bc_model="NEE", solid=solid, rho=rho, u=u, T=T, steps=20,
                thermal=(Df, Ds), channel=(0.03, 1.0), porous=dict(model="ergun", zone=zone, eps=0.55),
                heat=dict(h=2.0, a=1.5, rhos=1.5, emis=0.0, Ts0=Ts0))


def _nebb_case(name, kinds, seed, steps, quirks):
    """BC_MODEL.NEBB channel: ``kinds`` maps a side to ("wall" | "inlet" | "outlet", value)."""
    nx, ny = 24, 12
    shape = (nx, ny, 1)
    solid = np.zeros(shape, dtype=bool)
    solid[:, 2:ny - 2, 0] = _disks((nx, ny - 4), 2, 1.4, 2.0, 4, seed)
    rho, u, T = _common_inputs(shape, seed + 130, solid, u_amp=0.01)
    sides = [SideBC() for _ in range(6)]
    for s, (kind, val) in kinds.items():
        sides[s] = {"wall": lambda: SideBC.wall(), "inlet": lambda: SideBC.inlet(val),
                    "outlet": lambda: SideBC.outlet(val)}[kind]()
        sides[s].model = "nebb"
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision="bgk", precision="fp64", nu=0.1, sides=sides)
    return dict(name=name, cfg=cfg, bc_model="NEBB", solid=solid, rho=rho, u=u, T=T, steps=steps, thermal=None,
                nebb=kinds, quirk_dependent=quirks)


def case_nebb_channel2d():
    """Zou-He channel: velocity inlet west, pressure outlet east, walls south and north (the
    branches the reference writes as Zou and He do)."""
    return _nebb_case("ref_nebb_channel2d", {0: ("inlet", (0.03, 0.0, 0.0)), 1: ("outlet", 1.0),
                                            2: ("wall", None), 3: ("wall", None)}, 141, 60, False)


def case_nebb_quirks2d():
    """The reference's other NEBB branches: pressure outlet west (velocity sign flipped), wall
    east (rebuilds the west populations), inlet south and outlet north (no change)."""
    return _nebb_case("ref_nebb_quirks2d", {0: ("outlet", 1.002), 1: ("wall", None),
                                           2: ("inlet", (0.0, 0.01, 0.0)), 3: ("outlet", 1.0)}, 151, 40, True)


# temperature-dependent properties (THERMAL_DIFF_MODEL.DERIVED): coefficients of the
# reference's nested polynomials, c0 + c1 T + (c2 + c3) T^3 + c4 T^4, chosen so that the
# lattice diffusivities stay between 0.03 and 0.1 over 300-800 K, with the NASA7 switch
# at 550 K inside the range the channel reaches
TP_FLUID = dict(cond_poly=[0.2, 4e-4, 2e-10, 1e-10, -1e-13],
                nasa7=([200.0, 550.0, 3500.0], [[1.0, 4e-4, 1e-10, -5e-11, 2e-14, 0.0, 0.0],
                                                [1.2, 2e-4, 5e-11, 0.0, 0.0, 0.0, 0.0]]))
TP_SOLID = dict(cond_poly=[1.0, 1e-3, 1e-9, 1e-9], cap_poly=[2.0, 5e-3, 1e-10, 0.0, 0.0])
TP_RHOS = 5.0


def _tprop_case(base, name, steps):
    d = base()
    d["cfg"] = d["cfg"].replace(
        T_ref=300.0, T_scale=500.0, Ts_ref=300.0, Ts_scale=500.0, tp_rhos=TP_RHOS, tp_dt=1.0, tp_dx2=1.0,
        tprop_fluid=thermal_props(cond_poly=TP_FLUID["cond_poly"], nasa7=TP_FLUID["nasa7"]),
        tprop_solid=thermal_props(cond_poly=TP_SOLID["cond_poly"], cap_poly=TP_SOLID["cap_poly"], solid=True))
    d.update(name=name, steps=steps, tprop=(TP_FLUID, TP_SOLID, TP_RHOS))
    return d


def case_tprop2d():
    return _tprop_case(case_channel2d_thermal, "ref_tprop2d", 60)


def case_tprop3d():
    return _tprop_case(case_channel3d_thermal, "ref_tprop3d", 20)


def case_prandtl2d():
    """THERMAL_DIFF_MODEL.PRANDTL with the Sutherland viscosity: the fluid's diffusivity is
    the cell's kinetic viscosity over Pr, both following its temperature and density."""
    d = case_channel2d_thermal()
    As, Ts, Pr = 0.008, 110.0, 0.71          # nu 0.10-0.20 over 300-800 K (dt = dx = 1)
    d["cfg"] = d["cfg"].replace(T_ref=300.0, T_scale=500.0, viscosity="sutherland", suth_A=As, suth_Ts=Ts,
                                tp_prandtl=Pr)
    d.update(name="ref_prandtl2d", steps=60, sutherland=(As, Ts), prandtl=Pr)
    return d


CASES = [case_periodic2d, case_channel2d_thermal, case_channel2d_es, case_nee_periodic2d,
         case_periodic3d, case_channel3d_thermal, case_periodic3d_x32, case_channel3d_flow_x32,
         case_porous2d_darcy, case_porous2d_ergun, case_porous3d_df, case_porous2d_heat, case_porous3d_heat,
         case_nebb_channel2d, case_nebb_quirks2d, case_tprop2d, case_tprop3d, case_prandtl2d]


# --------------------------------------------------------------------------- driver
def run_reference(case, Solver2D, Solver3D, flag):
    cfg = case["cfg"]
    dim = cfg.dim
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    thermal = case.get("thermal")
    Solver = Solver2D if dim == 2 else Solver3D
    poro = case.get("porous")
    heat = case.get("heat")
    lb = Solver(nx, ny, nz, 1, 1, case["name"], thermal is not None, False, poro is not None, bool(cfg.radiation))
    lb.source_term_model = flag.SOURCE_TERM.MICRO       # app.py:103-104
    lb.force_term_model = flag.FORCE_TERM.GUO
    lb.set_viscosity(cfg.nu)
    lb.boundary_condition_model = getattr(flag.BC_MODEL, case["bc_model"])
    sides = [SideBC() for _ in range(6)]
    if "channel" in case:
        u_in, rho_out = case["channel"]
        ref, tbc, sides = _channel_sides(flag, dim, u_in, rho_out, thermal is not None)
        if case.get("periodic_y"):
            ref = {s: v for s, v in ref.items() if s < 2}
            for s in (2, 3):
                sides[s] = SideBC(True, PERIODIC, PERIODIC, PERIODIC)
        for s, (kind, v, r) in ref.items():
            lb.set_BC(s, getattr(flag.BC_FLOW, kind))
            if v is not None:
                lb.set_v_BC_value(s, list(v))
            if r is not None:
                lb.set_rho_BC_value(s, r)
        if thermal is not None:
            for s, (kind, val) in tbc.items():
                bc = flag.BC.fixedValue if kind == "fixed" else flag.BC.zeroGradient
                lb.set_TF_BC(s, bc)
                lb.set_TS_BC(s, bc)
                if val is not None:
                    lb.set_TF_BC_value(s, val)
                    lb.set_TS_BC_value(s, val)
    if "nebb" in case:
        for s, (kind, val) in case["nebb"].items():
            lb.set_BC(s, getattr(flag.BC_FLOW, kind))
            if kind == "inlet":
                lb.set_v_BC_value(s, list(val))
            elif kind == "outlet":
                lb.set_rho_BC_value(s, val)
        sides = case["cfg"].sides
    if case["bc_model"] == "NEE":
        for s in range(2 * dim):
            if not sides[s].active:
                sides[s] = SideBC(True, PERIODIC, PERIODIC, PERIODIC)
    if case["bc_model"] == "ES":
        for s in range(2 * dim):
            sides[s].model = "es"
    cfg.sides = sides
    if thermal is not None:
        Df, Ds = thermal
        lb.set_fluid_thermal_diff(Df)
        lb.set_solid_thermal_diff(Ds)
        lb.init_field(lb.TF.S, case["T"].copy())
        lb.init_field(lb.TS.S, (case["T"] if heat is None else heat["Ts0"]).copy())
    if "sutherland" in case:
        # src/LBM/LBM2D/_io.py:144-147; GetTF needs the fluid's temperature range
        lb.set_fluid_Trange([cfg.T_ref, cfg.T_ref + cfg.T_scale])
        lb.set_viscosity_sutherland(*case["sutherland"])
    if "prandtl" in case:
        lb.set_fluid_Prandtl(case["prandtl"])
    if "tprop" in case:
        # src/LBM/app.py:143-175 with thermalDiff "derived" and polynomial / NASA7 properties
        fl, so, rhos = case["tprop"]
        lb.set_fluid_Trange([cfg.T_ref, cfg.T_ref + cfg.T_scale])
        lb.set_solid_Trange([cfg.Ts_ref, cfg.Ts_ref + cfg.Ts_scale])
        lb.set_fluid_thermal_diff_derived()
        lb.set_fluid_conductivity_poly(list(fl["cond_poly"]))
        lb.set_fluid_capacity_NASA7(*fl["nasa7"])
        lb.set_solid_thermal_diff_derived()
        lb.set_solid_conductivity_poly(list(so["cond_poly"]))
        lb.set_solid_capacity_poly(list(so["cap_poly"]))
        lb.add_rho_solid(case["solid"].astype(np.float64) * rhos)
    if heat is not None:
        # app.py:537-566 for a porous zone: rhos, exchange surface and coefficient over it,
        # radiation surface and emissivity on its border; TS range and capacities
        lb.set_fluid_Trange([cfg.T_ref, cfg.T_ref + cfg.T_scale])
        lb.set_solid_Trange([cfg.Ts_ref, cfg.Ts_ref + cfg.Ts_scale])
        lb.set_fluid_capacity(cfg.cap_fluid)
        lb.set_solid_capacity(cfg.cap_solid)
        zs = poro["zone"].astype(np.float64)
        lb.add_rho_solid(heat["rhos"] * zs)
        lb.set_heat_exchange_surface(heat["a"] * zs)
        lb.set_heat_exchange_coef(heat["h"] * zs)
        case["xh"], case["xa"], case["rhos"] = heat["h"] * zs, heat["a"] * zs, heat["rhos"] * zs
        case["Ts0"] = heat["Ts0"]
        if cfg.radiation:
            lb.set_radiation(flag.RADIATION_MODEL.SURFACE_UNIFORM, cfg.T_ambient)
            border = _border(poro["zone"])
            lb.init_field(lb.TS.radiation_surface, border.copy())
            lb.init_field(lb.TS.emissivity, border * heat["emis"])
            case["emis"], case["rsurf"] = border * heat["emis"], border
    lb.init_field(lb.rho, case["rho"].copy())
    lb.init_field3(lb.v, case["u"][0].copy(), case["u"][1].copy(), case["u"][2].copy())
    lb.add_solid(case["solid"].astype(np.float64))
    if poro is not None:
        # app.py:537-573: solid fraction (1 - porosity) over the zone, coefficients over it
        zs = poro["zone"].astype(np.float64)
        frac = (1.0 - poro["eps"]) * zs
        lb.add_solid(frac)
        case["sfrac"] = case["solid"].astype(np.float64) + frac
        case["darcy"] = np.zeros(zs.shape)
        case["forch"] = np.zeros(zs.shape)
        if poro["model"] == "darcy":
            lb.set_poro_Darcy(zs, poro["darcy"])
            case["darcy"] = poro["darcy"] * zs
        elif poro["model"] == "darcy_forchheimer":
            lb.set_poro_Darcy_Forchheimer(zs, poro["darcy"], poro["forch"])
            case["darcy"] = poro["darcy"] * zs
            case["forch"] = poro["forch"] * zs
    lb.init_simulation()
    t0 = time.time()
    for _ in range(case["steps"]):
        lb.step()
    out = dict(rho=lb.rho.to_numpy(), u=np.moveaxis(lb.v.to_numpy(), -1, 0),
               f=np.moveaxis(lb.f.to_numpy(), -1, 0))
    if thermal is not None:
        tf, ts = lb.TF.S.to_numpy(), lb.TS.S.to_numpy()
        out["T"] = np.where(case["solid"], ts, tf)
        out["g"] = np.moveaxis(np.where(case["solid"][..., None], lb.TS.g.to_numpy(), lb.TF.g.to_numpy()), -1, 0)
        if heat is not None:
            out["Ts"] = ts
            out["gs"] = np.moveaxis(lb.TS.g.to_numpy(), -1, 0)
    return out, time.time() - t0


def main(argv):
    if len(argv) < 2:
        print(__doc__)
        return 2
    Solver2D, Solver3D, flag = _import_reference(argv[1])
    only = set(argv[2:])
    for mk in CASES:
        case = mk()
        if only and case["name"] not in only:
            continue
        out, dt = run_reference(case, Solver2D, Solver3D, flag)
        meta = dict(cfg=case["cfg"].to_dict(), steps=case["steps"], bc_model=case["bc_model"],
                    ref_quirk_frozen_solid_T=case["cfg"].thermal == "two_field",
                    ref_quirk_nebb="nebb" in case, quirk_dependent=case.get("quirk_dependent", False),
                    generator="tests/golden/make_reference_fixtures.py")
        path = HERE / f"{case['name']}.npz"
        extra = {k: case[k] for k in ("sfrac", "darcy", "forch", "xh", "xa", "rhos", "emis", "rsurf", "Ts0")
                 if k in case}
        np.savez_compressed(path, meta=json.dumps(meta), solid=case["solid"], rho0=case["rho"],
                            u0=case["u"], T0=case["T"], **extra, **{k + "_ref": v for k, v in out.items()})
        print(f"{case['name']}: {case['steps']} steps in {dt:.1f} s -> {path.name} "
              f"({path.stat().st_size} B)")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
