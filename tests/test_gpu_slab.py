"""Slab decomposition on the GPU: the slabs of one lattice (``SlabSet``: every slab on this device,
exchanged by device copies after every step) against the undivided lattice, both in the tile form.

Bit for bit in FP32, FP16 and FP64, through solid -> fluid flips next to the slab edges, with
the pyrolysis packing (conjugate heat, MRT) and with porous cells carrying two temperature
fields; and the FP64 slabs against the oracle at 1e-10.  The exchange between processes
(``DistExchange``) is tested on the CPU with two gloo ranks (tests/test_slab.py).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("rho", "u", "T", "alpha", "solid")


def _pyro(precision, nz=20):
    from lbm_porouschem_b200 import workloads
    w = workloads.pyro3d(32, seed=4, ny=16, nz=nz, collision="mrt", precision=precision)
    cfg = w.cfg.replace(pyro_A=2e11, heat_norm=0.02, gas_coef=0.05, bulk_form="tile")
    return cfg, w.solid.reshape(cfg.shape), w.reactive.reshape(cfg.shape), dict(w.init, T=1.0)


def _whole(cfg, solid, reactive, init, steps):
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(cfg)
    lat.set_geometry(solid, reactive)
    lat.init(**init)
    lat.step(steps)
    out = lat.fields()
    lat.close()
    return out


def _slabs(cfg, solid, reactive, init, steps, nslabs):
    from lbm_porouschem_b200.slab import SlabSet
    s = SlabSet(cfg, nslabs)
    s.set_geometry(solid, reactive)
    s.init(**init)
    s.step(steps)
    out = s.fields()
    s.close()
    return out


@pytest.mark.parametrize("nslabs", [1, 2, 3])
@pytest.mark.parametrize("precision", ["fp32", "fp16", "fp64"])
def test_slabs_equal_the_whole_lattice(precision, nslabs):
    cfg, solid, reactive, init = _pyro(precision)
    steps = 60
    ref = _whole(cfg, solid, reactive, init, steps)
    got = _slabs(cfg, solid, reactive, init, steps, nslabs)
    assert (solid & ~ref["solid"]).sum() >= 3
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k


def test_fp64_slabs_match_the_oracle(oracle_mod):
    cfg, solid, reactive, init = _pyro("fp64")
    steps = 60
    got = _slabs(cfg, solid, reactive, init, steps, 3)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(solid, reactive, **init)
    o.step(steps)
    r = o.fields()
    fl = ~r["solid"]
    assert np.array_equal(got["solid"], r["solid"])
    for k in ("rho", "T", "alpha"):
        assert float(np.linalg.norm(got[k][fl] - r[k][fl]) / np.linalg.norm(r[k][fl])) < 1e-10, k
    assert float(np.linalg.norm(got["u"][:, fl] - r["u"][:, fl]) / np.linalg.norm(r["u"][:, fl])) < 1e-10


def test_porous_heat_slabs_equal_the_whole_lattice():
    """Porous cells with TF and TS: the porous TS populations are exchanged too."""
    from lbm_porouschem_b200.config import FIXED_VALUE, ZERO_GRADIENT, LatticeConfig, SideBC
    from lbm_porouschem_b200.lattice import Lattice
    from lbm_porouschem_b200.slab import SlabSet
    shape = (32, 12, 12)
    g = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    zone = sum((gi - ci) ** 2 for gi, ci in zip(g, (12.3, 6.1, 10.9))) <= 4.3 ** 2   # crosses z = 0
    solid = (sum((gi - ci) ** 2 for gi, ci in zip(g, (22.0, 5.5, 5.0))) <= 2.2 ** 2) & ~zone
    sides = [SideBC.inlet((0.02, 0, 0), FIXED_VALUE, 1.0), SideBC.outlet(1.0, ZERO_GRADIENT, 0.0)] + [SideBC()] * 4
    cfg = LatticeConfig(dim=3, nx=32, ny=12, nz=12, collision="bgk", precision="fp32", nu=0.08, porous="darcy",
                        sides=sides, thermal="two_field", tauT_fluid=0.66, tauT_solid=0.86, Ts_ref=260.0,
                        Ts_scale=580.0, cap_solid=750.0, dt_phys=1.0, dx_phys=1.0, radiation=True,
                        T_ambient=320.0, bulk_form="tile")
    zf = zone.astype(np.float64)
    heat = dict(h=2.5 * zf, a=zf, rho_solid=1.5 * zf + (1 - zf), emissivity=0.7 * zf, radiation_surface=zf)
    init = dict(rho=1.0, u=(0.0, 0.0, 0.0), T=0.2, Ts=0.6)
    lat = Lattice(cfg)
    lat.set_geometry(solid)
    lat.set_porous(0.45 * zf, 0.05 * zf, **heat)
    lat.init(**init)
    lat.step(50)
    ref = lat.fields()
    lat.close()
    s = SlabSet(cfg, 2)
    s.set_geometry(solid)
    s.set_porous(0.45 * zf, 0.05 * zf, **heat)
    s.init(**init)
    s.step(50)
    got = s.fields()
    s.close()
    for k in ("rho", "u", "T", "Ts"):
        assert np.array_equal(got[k], ref[k]), k


@pytest.mark.parametrize("mode", ["derived", "prandtl"])
def test_temperature_dependent_slabs_equal_the_whole_lattice(mode):
    """Per-cell thermal diffusivities (derived from polynomial / NASA7 properties of both
    phases, or the fluid's Prandtl model over the Sutherland viscosity) through pyrolysis flips:
    the rates depend on the cell's own state only, so the slabs stay bit for bit equal."""
    from lbm_porouschem_b200.config import thermal_props
    cfg, solid, reactive, init = _pyro("fp32")
    if mode == "derived":
        cfg = cfg.replace(
            Ts_ref=cfg.T_ref, Ts_scale=cfg.T_scale, tp_rhos=5.0,
            tprop_fluid=thermal_props(cond_poly=[0.2, 4e-4, 2e-10, 1e-10, -1e-13],
                                      nasa7=([200.0, 550.0, 3500.0], [[1.0, 4e-4, 1e-10, -5e-11, 2e-14, 0, 0],
                                                                      [1.2, 2e-4, 5e-11, 0, 0, 0, 0]])),
            tprop_solid=thermal_props(cond_poly=[1.0, 1e-3, 1e-9, 1e-9], cap_poly=[2.0, 5e-3, 1e-10, 0, 0],
                                      solid=True))
    else:
        cfg = cfg.replace(viscosity="sutherland", suth_A=0.005, suth_Ts=170.0, tp_prandtl=0.71)
    ref = _whole(cfg, solid, reactive, init, 60)
    got = _slabs(cfg, solid, reactive, init, 60, 2)
    assert (solid & ~ref["solid"]).sum() >= 3
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k
