"""The CUDA lattice update (through the C ABI) against outputs of the reference's own solver.

Fixtures: ``tests/golden/ref_*.npz``, written by ``tests/golden/make_reference_fixtures.py``
from the unmodified reference modules (``src/LBM/LBM2D``, ``src/LBM/LBM3D``) in float64.

Tolerances (relative L2 over the compared cells):
  - FP64 kernels, tile and cell-list forms: 1e-10 for rho, u and temperature.  The kernels
    use a pull scheme with mirror stores and fused multiply-adds, so they agree with the
    reference's push-scheme arithmetic to rounding, not bit for bit.
  - FP32 kernels: 1e-5 for rho and temperature, and for u measured against the velocity
    scale (RMS error / max |u|): the velocity is a small difference of O(1) populations.
Cells compared: fluid cells for rho and u; for temperature every fluid cell, and the solid
cells only where the reference's solid temperature evolves (in its two-field model the
pure-solid cells keep their initial temperature, ``src/LBM/LBM2D/_evolution.py:119``, while
these kernels diffuse heat through the solid; the fluid side is unaffected because the
interface is adiabatic in that model).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("ref_*.npz"))


def _load(name):
    from lbm_porouschem_b200.config import LatticeConfig
    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    return z, meta, LatticeConfig.from_dict(meta["cfg"])


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _run(cfg, z, steps):
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(cfg)
    lat.set_geometry(z["solid"])
    lat.init(rho=z["rho0"], u=z["u0"], T=z["T0"])
    lat.step(steps)
    out = lat.fields()
    lat.close()
    return out


@pytest.mark.parametrize("form", ["tile", "list"])
@pytest.mark.parametrize("name", CASES)
def test_fp64_kernels_match_reference(name, form):
    z, meta, cfg = _load(name)
    g = _run(cfg.replace(precision="fp64", bulk_form=form), z, meta["steps"])
    fl = ~z["solid"]
    assert np.array_equal(g["solid"], z["solid"])
    assert _rel(g["rho"][fl], z["rho_ref"][fl]) < 1e-10
    assert _rel(g["u"][:, fl], z["u_ref"][:, fl]) < 1e-10
    if cfg.thermal != "none":
        cells = fl if meta["ref_quirk_frozen_solid_T"] else np.ones_like(fl)
        assert _rel(g["T"][cells], z["T_ref"][cells]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_fp32_kernels_match_reference(name):
    z, meta, cfg = _load(name)
    g = _run(cfg.replace(precision="fp32"), z, meta["steps"])
    fl = ~z["solid"]
    assert _rel(g["rho"][fl], z["rho_ref"][fl]) < 1e-5
    du = g["u"][:, fl] - z["u_ref"][:, fl]
    e_u = np.sqrt(np.mean(du ** 2)) / np.abs(z["u_ref"][:, fl]).max()
    assert e_u < 1e-5, e_u
    if cfg.thermal != "none":
        assert _rel(g["T"][fl], z["T_ref"][fl]) < 1e-5
