"""NEBB (Zou-He non-equilibrium bounce-back, the reference's BC_MODEL.NEBB, 2D) in the CUDA
boundary kernel, through the C ABI, against the oracle.

tests/test_gpu_reference.py checks the kernels against the reference's own NEBB channel
(velocity inlet west, pressure outlet east, walls); here every side kind on every side in the
Zou-He form (the oracle without its ref_quirk_nebb switch), with disks in the channel:
FP64 tile and list forms at 1e-10 on rho and u, FP32 rho within 1e-5 of the FP32 oracle.
"""
import numpy as np
import pytest

from lbm_porouschem_b200.config import LatticeConfig, SideBC

pytestmark = pytest.mark.gpu


def _case(kinds, precision="fp64", collision="bgk"):
    nx, ny = 96, 40
    g = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    solid = np.zeros((nx, ny), dtype=bool)
    for cx, cy, r in ((30.2, 19.7, 5.3), (58.6, 12.4, 4.1), (71.3, 27.8, 4.6)):
        solid |= (g[0] - cx) ** 2 + (g[1] - cy) ** 2 <= r * r
    sides = [SideBC() for _ in range(6)]
    for s, (kind, val) in kinds.items():
        sides[s] = {"wall": SideBC.wall, "inlet": lambda: SideBC.inlet(val),
                    "outlet": lambda: SideBC.outlet(val)}[kind]() if kind != "wall" else SideBC.wall()
        sides[s].model = "nebb"
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision=collision, precision=precision, nu=0.08, sides=sides)
    return cfg, solid.reshape(nx, ny, 1)


CASES = {
    "channel": {0: ("inlet", (0.03, 0.0, 0.0)), 1: ("outlet", 1.0), 2: ("wall", None), 3: ("wall", None)},
    "reversed": {0: ("outlet", 1.0), 1: ("inlet", (-0.02, 0.005, 0.0)), 2: ("wall", None),
                 3: ("inlet", (0.01, 0.0, 0.0))},
    "cross": {0: ("wall", None), 1: ("outlet", 0.999), 2: ("inlet", (0.0, 0.02, 0.0)), 3: ("outlet", 1.0)},
    "x_only": {0: ("inlet", (0.02, 0.0, 0.0)), 1: ("outlet", 1.0)},   # y periodic: rows 0 and ny-1 untreated
}


def _gpu(cfg, solid, steps, form):
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(cfg.replace(bulk_form=form))
    lat.set_geometry(solid)
    lat.init(rho=1.0, u=(0.0, 0.0, 0.0))
    lat.step(steps)
    out = lat.fields()
    lat.close()
    return out


def _oracle(oracle_mod, cfg, solid, steps, real):
    o = oracle_mod.Oracle(cfg, real=real)
    o.init(solid, None, rho=1.0, u=(0.0, 0.0, 0.0))
    o.step(steps)
    return o.fields()


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("form", ["tile", "list"])
@pytest.mark.parametrize("collision", ["bgk", "mrt"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_nebb_matches_oracle(oracle_mod, name, collision, form):
    cfg, solid = _case(CASES[name], collision=collision)
    g = _gpu(cfg, solid, 300, form)
    r = _oracle(oracle_mod, cfg, solid, 300, "f64")
    fl = ~solid
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-10
    assert _rel(g["u"][:, fl], r["u"][:, fl]) < 1e-10
    assert np.abs(r["u"]).max() > 1e-3          # the sides drive a flow


def test_fp32_nebb(oracle_mod):
    cfg, solid = _case(CASES["channel"], precision="fp32")
    g = _gpu(cfg, solid, 300, "list")
    r = _oracle(oracle_mod, cfg, solid, 300, "f32")
    fl = ~solid
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-5
    assert _rel(g["u"][:, fl], r["u"][:, fl]) < 1e-3
