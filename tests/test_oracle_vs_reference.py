"""The FP64 oracle against outputs of the reference's own solver code (golden fixtures).

The fixtures under ``tests/golden/ref_*.npz`` were written by
``tests/golden/make_reference_fixtures.py``, which runs the unmodified reference modules
``src/LBM/LBM2D`` / ``src/LBM/LBM3D`` (``step`` = ``_evolution.py:12-25`` with
``collision_source_streaming``, ``macro`` and the NEE / ES boundaries) on a sequential NumPy
stand-in for Taichi, in float64, from float32-representable inputs.  Each case records the
``LatticeConfig`` describing the same run here.

The bar is 1e-12 relative L2 (the restatement follows the reference's arithmetic order, so
in practice the fields agree bit for bit); fluid and porous cells are compared for rho, u and
the flow populations, every cell for temperature.  The porous cases run the reference with
``isPoro``: cells of solid fraction between 0 and 1, the eps-equilibrium, the Darcy /
Darcy-Forchheimer / Ergun drag in the Guo term and the macro velocity correction.  The
porous heat cases add two temperature fields: a porous cell carries both TF and TS, which
exchange heat there, and its surface radiates (``_evolution.py:186-202``); TS of the porous
cells (temperature and populations) is compared too.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("ref_*.npz"))
TOL = 1e-12


def load_case(name):
    from lbm_porouschem_b200.config import LatticeConfig
    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    cfg = LatticeConfig.from_dict(meta["cfg"])
    return z, meta, cfg


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def planar(a, Q):
    """(Q, nx, ny, nz) -> (Q, N) in the package's cell order (x fastest)."""
    return np.stack([a[k].ravel(order="F") for k in range(Q)])


def test_fixtures_present():
    assert len(CASES) >= 6, CASES


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(oracle_mod, name):
    z, meta, cfg = load_case(name)
    o = oracle_mod.Oracle(cfg, real="f64", ref_quirk_frozen_solid_T=meta["ref_quirk_frozen_solid_T"],
                          ref_quirk_nebb=meta.get("ref_quirk_nebb", False))
    if "sfrac" in z:   # porous cells: solid fraction and drag coefficients
        o.set_porous(z["sfrac"], z["darcy"], z["forch"])
    if "xh" in z:      # two fields with porous cells: exchange and radiation inputs
        o.set_porous_heat(z["xh"], z["xa"], z["rhos"], z["emis"] if "emis" in z else None,
                          z["rsurf"] if "rsurf" in z else None)
    o.init(z["solid"], None, rho=z["rho0"], u=z["u0"], T=z["T0"], Ts=z["Ts0"] if "Ts0" in z else None)
    o.step(meta["steps"])
    r = o.fields()
    fl = ~z["solid"]
    assert np.array_equal(r["solid"], z["solid"])
    assert rel(r["rho"][fl], z["rho_ref"][fl]) <= TOL
    assert rel(r["u"][:, fl], z["u_ref"][:, fl]) <= TOL
    f, g = o.dist()
    flf = fl.ravel(order="F")
    assert rel(f[:, flf], planar(z["f_ref"], cfg.Q)[:, flf]) <= TOL
    if cfg.thermal != "none":
        assert rel(r["T"], z["T_ref"]) <= TOL
        assert rel(g, planar(z["g_ref"], cfg.QT)) <= TOL
    if "Ts_ref" in z:
        pc = z["xh"] > 0
        assert rel(r["Ts"][pc], z["Ts_ref"][pc]) <= TOL
        gs = o.dist_solid()
        pf = pc.ravel(order="F")
        assert rel(gs[:, pf], planar(z["gs_ref"], cfg.QT)[:, pf]) <= TOL


def test_nebb_quirks_matter(oracle_mod):
    """The channel case uses only the NEBB branches the reference writes as Zou and He do:
    with or without the quirk switch the oracle gives the same answer; the quirk case needs
    the switch."""
    for name, differs in (("ref_nebb_channel2d", False), ("ref_nebb_quirks2d", True)):
        z, meta, cfg = load_case(name)
        o = oracle_mod.Oracle(cfg, real="f64", ref_quirk_nebb=False)
        o.init(z["solid"], None, rho=z["rho0"], u=z["u0"], T=z["T0"])
        o.step(meta["steps"])
        fl = ~z["solid"]
        e = rel(o.fields()["u"][:, fl], z["u_ref"][:, fl])
        assert (e > 1e-6) == differs, (name, e)


def test_porous_heat_exchange_matters(oracle_mod):
    """The porous heat case moves heat between the fields: without the exchange and radiation
    inputs the porous cells' temperatures differ from the reference's."""
    z, meta, cfg = load_case("ref_porous2d_heat")
    o = oracle_mod.Oracle(cfg, real="f64")
    o.set_porous(z["sfrac"], z["darcy"], z["forch"])
    o.init(z["solid"], None, rho=z["rho0"], u=z["u0"], T=z["T0"], Ts=z["Ts0"])
    o.set_porous_heat(None, None, z["rhos"], None, None)
    o.step(meta["steps"])
    pc = z["xh"] > 0
    r = o.fields()
    assert rel(r["Ts"][pc], z["Ts_ref"][pc]) > 1e-3
    assert rel(r["T"][pc], z["T_ref"][pc]) > 1e-4


def test_frozen_solid_quirk_matters(oracle_mod):
    """Without the quirk switch the oracle diffuses heat through the solid, which the
    reference does not: the solid temperature then differs while the fluid stays equal
    (the interface is adiabatic in the two-field model)."""
    z, meta, cfg = load_case("ref_channel2d_thermal")
    o = oracle_mod.Oracle(cfg, real="f64", ref_quirk_frozen_solid_T=False)
    o.init(z["solid"], None, rho=z["rho0"], u=z["u0"], T=z["T0"])
    o.step(meta["steps"])
    T = o.fields()["T"]
    s = z["solid"]
    assert rel(T[~s], z["T_ref"][~s]) <= TOL
    assert rel(T[s], z["T_ref"][s]) > 1e-3


@pytest.mark.parametrize("name", ["ref_tprop2d", "ref_tprop3d"])
def test_temperature_dependent_properties_matter(oracle_mod, name):
    """The derived fluid diffusivity matters: with the constant relaxation times the case also
    carries, the fluid temperatures differ from the reference's.  The solid's properties
    leave no trace in these outputs: the reference's pure-solid cells keep their initial
    temperature and equilibrium populations w T (macro skips them), whatever their relaxation
    time, so only the kernels' evolving solid (against this oracle) exercises that path."""
    z, meta, cfg = load_case(name)
    fl = ~z["solid"]
    errs = []
    for c in (cfg.replace(tprop_fluid=None, tprop_solid=None), cfg.replace(tprop_solid=None)):
        o = oracle_mod.Oracle(c, real="f64", ref_quirk_frozen_solid_T=True)
        o.init(z["solid"], None, rho=z["rho0"], u=z["u0"], T=z["T0"])
        o.step(meta["steps"])
        errs.append(rel(o.fields()["T"][fl], z["T_ref"][fl]))
    assert errs[0] > 1e-3 and errs[1] <= TOL, errs


def test_prandtl_and_sutherland_matter(oracle_mod):
    """The Prandtl case's fluid temperature depends on the per-cell diffusivity
    kinetic_viscosity / Pr and its velocity on the Sutherland viscosity: replacing either by
    its constant counterpart moves the result away from the reference's."""
    z, meta, cfg = load_case("ref_prandtl2d")
    fl = ~z["solid"]
    for c, key, bound in ((cfg.replace(tp_prandtl=0.0), "T", 1e-4),
                          (cfg.replace(viscosity="constant"), "u", 1e-3)):
        o = oracle_mod.Oracle(c, real="f64", ref_quirk_frozen_solid_T=True)
        o.init(z["solid"], None, rho=z["rho0"], u=z["u0"], T=z["T0"])
        o.step(meta["steps"])
        r = o.fields()
        got = r[key][..., fl] if key == "u" else r[key][fl]
        ref = z[key + "_ref"][..., fl] if key == "u" else z[key + "_ref"][fl]
        assert rel(got, ref) > bound, (key, rel(got, ref))
