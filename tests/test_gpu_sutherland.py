"""Sutherland viscosity (LBM_VISC_SUTHERLAND, the reference's VISCOSITY_MODEL.SUTHERLAND,
src/LBM/LBM2D/_evolution.py:228-249) on the CUDA path, called through the C ABI,
against the C oracle.

The cases have a temperature gradient (hot inlet at 800 K into a packing at 400 K), so
the lattice viscosity ranges over 0.07-0.12 across the domain.  Tolerances as in the
other parity cases: FP64 vs the FP64 oracle 1e-10 relative L2 for rho, u, T (and
identical masks through pyrolysis flips); FP32 vs the FP32 oracle 1e-5 for rho and T,
u against the FP64 oracle within 2x the FP32 oracle's own error (plus 1e-9).  A batch
of Sutherland lattices equals the lattices stepped one by one, bit for bit."""
import numpy as np
import pytest

from lbm_porouschem_b200.config import FIXED_VALUE, ZERO_GRADIENT, LatticeConfig, SideBC
from lbm_porouschem_b200.geometry import packing

pytestmark = pytest.mark.gpu


def _rel(a, b, mask):
    a, b = np.asarray(a, np.float64)[..., mask], np.asarray(b, np.float64)[..., mask]
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


class _Case:
    pass


def _case(dim, coll="bgk", thermal="conjugate", precision="fp64", pyro=False, seed=0):
    shape = (44, 24) if dim == 2 else (26, 16, 12)
    solid = packing(shape, 1.5, 3.0, 0.7, seed=11 + dim + seed)
    keep = np.zeros(shape, dtype=bool)
    keep[(slice(3, shape[0] - 3),) + tuple(slice(None) for _ in shape[1:])] = True
    solid &= keep
    sides = [SideBC.pressure(1.002, FIXED_VALUE, 1.0), SideBC.outlet(1.0, ZERO_GRADIENT)] + [SideBC()] * 4
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=1 if dim == 2 else shape[2], collision=coll,
                        nu=0.1, precision=precision, sides=sides, thermal=thermal, T_ref=300.0, T_scale=500.0,
                        viscosity="sutherland", suth_A=0.005, suth_Ts=170.0)
    if pyro:
        cfg = cfg.replace(pyro=True, pyro_A=1e13, heat_norm=0.02, gas_coef=0.05)   # flips within ~10 steps at 700 K
    c = _Case()
    c.cfg, c.solid, c.reactive = cfg, solid, (solid if pyro else None)
    c.init = {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 0.8 if pyro else 0.2}
    return c


def _gpu(c, n, bulk=None, monkeypatch=None, cfg=None):
    from lbm_porouschem_b200.lattice import Lattice
    if bulk:
        monkeypatch.setenv("LBM_BULK", bulk)
    lat = Lattice(cfg or c.cfg)
    lat.set_geometry(c.solid, c.reactive)
    lat.init(**c.init)
    lat.step(n)
    out = lat.fields()
    lat.close()
    return out


def _oracle(oracle_mod, c, n, real):
    o = oracle_mod.Oracle(c.cfg, real=real)
    o.init(c.solid, c.reactive, **c.init)
    o.step(n)
    out = o.fields()
    o.close()
    return out


@pytest.mark.parametrize("dim,coll,thermal,pyro,bulk", [(2, "bgk", "conjugate", False, "list"),
                                                        (2, "mrt", "two_field", False, "tile"),
                                                        (2, "mrt", "conjugate", True, "list"),
                                                        (3, "bgk", "conjugate", False, "tile"),
                                                        (3, "mrt", "conjugate", True, "list")])
def test_sutherland_fp64(oracle_mod, monkeypatch, dim, coll, thermal, pyro, bulk):
    c = _case(dim, coll, thermal, pyro=pyro)
    n = 200 if dim == 2 else 100
    g, r = _gpu(c, n, bulk, monkeypatch), _oracle(oracle_mod, c, n, "f64")
    assert np.array_equal(g["solid"], r["solid"])
    if pyro:
        assert (c.solid.reshape(r["solid"].shape) & ~r["solid"]).any()   # cells turned fluid (flip_cells)
    fl = ~r["solid"]
    assert _rel(g["rho"], r["rho"], fl) < 1e-10
    assert _rel(g["u"], r["u"], fl) < 1e-10
    assert _rel(g["T"], r["T"], np.ones_like(fl)) < 1e-10
    # the law matters here: a constant viscosity at the mean temperature differs
    flat = _gpu(c, n, cfg=c.cfg.replace(viscosity="constant", nu=0.09))
    assert _rel(flat["u"], g["u"], fl) > 1e-3


def test_sutherland_fp32(oracle_mod):
    c = _case(2, "mrt", precision="fp32")
    n = 200
    g = _gpu(c, n)
    r32, r64 = _oracle(oracle_mod, c, n, "f32"), _oracle(oracle_mod, c, n, "f64")
    fl = ~r64["solid"]
    assert _rel(g["rho"], r32["rho"], fl) < 1e-5
    assert _rel(g["T"], r32["T"], np.ones_like(fl)) < 1e-5
    assert _rel(g["u"], r64["u"], fl) <= 2 * _rel(r32["u"], r64["u"], fl) + 1e-9


def test_sutherland_batch_equals_single_lattices():
    from lbm_porouschem_b200.lattice import Lattice, LatticeBatch
    cases = [_case(2, "bgk", precision="fp32", pyro=True, seed=s) for s in range(3)]
    ref = [_gpu(c, 60, cfg=c.cfg.replace(bulk_form="list")) for c in cases]
    lats = []
    for c in cases:
        lat = Lattice(c.cfg.replace(bulk_form="list"))
        lat.set_geometry(c.solid, c.reactive)
        lat.init(**c.init)
        lats.append(lat)
    batch = LatticeBatch(lats)
    batch.step(60)
    batch.synchronize()
    for lat, r in zip(lats, ref):
        assert lat.nsteps == 60
        got = lat.fields()
        for k in ("rho", "u", "T", "solid"):
            assert np.array_equal(got[k], r[k]), k
    batch.close()
    for lat in lats:
        lat.close()


def test_sutherland_needs_the_temperature_field():
    from lbm_porouschem_b200 import _native as N
    from lbm_porouschem_b200.lattice import Lattice
    c = _case(2)
    with pytest.raises(N.LBMNativeError, match="Sutherland"):
        Lattice(c.cfg.replace(thermal="none"))
