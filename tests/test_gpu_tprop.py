"""Temperature-dependent thermal properties (lbm_desc.tprop: THERMAL_DIFF_MODEL.DERIVED with
polynomial conductivity and polynomial / NASA7 capacity, src/LBM/LBM2D/_thermal.py:62-107,
:167-210) on the CUDA path, called through the C ABI, against the C oracle.

The cases heat a packing at 400 K from an 800 K inlet (conjugate field: heat crosses into the
solid, so both phases' diffusivities follow an evolving temperature, and the fluid's NASA7
capacity switches range at 550 K inside the domain).  Tolerances as in the other parity
cases: FP64 vs the FP64 oracle 1e-10 relative L2 for rho, u, T (identical masks through
pyrolysis flips); FP32 vs the FP32 oracle 1e-5 for rho and T.  The fixtures
``ref_tprop2d`` / ``ref_tprop3d`` (the reference's own solver) are checked by
test_gpu_reference.py like every other fixture."""
import numpy as np
import pytest

from lbm_porouschem_b200.config import FIXED_VALUE, ZERO_GRADIENT, LatticeConfig, SideBC, thermal_props
from lbm_porouschem_b200.geometry import packing

pytestmark = pytest.mark.gpu

# lattice-unit coefficients (tp_dt = tp_dx2 = 1): diffusivities 0.03-0.1 over 300-800 K
TP_FLUID = thermal_props(cond_poly=[0.2, 4e-4, 2e-10, 1e-10, -1e-13],
                         nasa7=([200.0, 550.0, 3500.0], [[1.0, 4e-4, 1e-10, -5e-11, 2e-14, 0.0, 0.0],
                                                         [1.2, 2e-4, 5e-11, 0.0, 0.0, 0.0, 0.0]]))
TP_SOLID = thermal_props(cond_poly=[1.0, 1e-3, 1e-9, 1e-9], cap_poly=[2.0, 5e-3, 1e-10, 0.0, 0.0], solid=True)


def _rel(a, b, mask=None):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[..., mask], b[..., mask]
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


class _Case:
    pass


def _case(dim, coll="bgk", thermal="conjugate", precision="fp64", pyro=False, suth=False, shape=None):
    shape = shape or ((44, 24) if dim == 2 else (26, 16, 12))
    solid = packing(shape, 1.5, 3.0, 0.7, seed=21 + dim)
    keep = np.zeros(shape, dtype=bool)
    keep[(slice(3, shape[0] - 3),) + tuple(slice(None) for _ in shape[1:])] = True
    solid &= keep
    sides = [SideBC.pressure(1.002, FIXED_VALUE, 1.0), SideBC.outlet(1.0, ZERO_GRADIENT)] + [SideBC()] * 4
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=1 if dim == 2 else shape[2], collision=coll,
                        nu=0.1, precision=precision, sides=sides, thermal=thermal, T_ref=300.0, T_scale=500.0,
                        Ts_ref=300.0, Ts_scale=500.0, tprop_fluid=TP_FLUID, tprop_solid=TP_SOLID, tp_rhos=5.0)
    if suth:
        cfg = cfg.replace(viscosity="sutherland", suth_A=0.005, suth_Ts=170.0)
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


def _oracle(oracle_mod, c, n, real, cfg=None):
    o = oracle_mod.Oracle(cfg or c.cfg, real=real)
    o.init(c.solid, c.reactive, **c.init)
    o.step(n)
    out = o.fields()
    o.close()
    return out


@pytest.mark.parametrize("dim,coll,thermal,pyro,suth,bulk", [(2, "bgk", "conjugate", False, False, "list"),
                                                             (2, "mrt", "two_field", False, False, "tile"),
                                                             (2, "mrt", "conjugate", True, False, "list"),
                                                             (2, "bgk", "conjugate", False, True, "tile"),
                                                             (3, "bgk", "conjugate", False, False, "tile"),
                                                             (3, "mrt", "two_field", False, False, "list"),
                                                             (3, "mrt", "conjugate", True, True, "list")])
def test_tprop_fp64(oracle_mod, monkeypatch, dim, coll, thermal, pyro, suth, bulk):
    c = _case(dim, coll, thermal, pyro=pyro, suth=suth)
    if thermal == "two_field":
        c.init["T"] = np.where(c.solid, 0.6, 0.2)   # the solid's own (adiabatic) range
    n = 150 if dim == 2 else 60
    g, r = _gpu(c, n, bulk, monkeypatch), _oracle(oracle_mod, c, n, "f64")
    assert np.array_equal(g["solid"], r["solid"])
    fl = ~r["solid"]
    assert _rel(g["rho"], r["rho"], fl) < 1e-10
    assert _rel(g["u"], r["u"], fl) < 1e-10
    assert _rel(g["T"], r["T"]) < 1e-10
    if pyro:
        assert (c.solid & fl.reshape(c.solid.shape)).any(), "the case should convert some cells"
    Tk = 300.0 + 500.0 * r["T"][fl]
    if not pyro:
        assert Tk.min() < 550.0 < Tk.max(), "the fluid should cross the NASA7 switch temperature"


def test_tprop_dense_fp64(oracle_mod):
    """The TMA-staged dense form (3D, conjugate field) with both phases' derived diffusivity."""
    c = _case(3, "mrt", shape=(32, 16, 12))
    cfg = c.cfg.replace(bulk_form="dense")
    g, r = _gpu(c, 60, cfg=cfg), _oracle(oracle_mod, c, 60, "f64")
    fl = ~r["solid"]
    assert _rel(g["rho"], r["rho"], fl) < 1e-10
    assert _rel(g["u"], r["u"], fl) < 1e-10
    assert _rel(g["T"], r["T"]) < 1e-10


def test_tprop_fp32(oracle_mod):
    c = _case(2, "mrt", precision="fp32")
    g, r = _gpu(c, 150), _oracle(oracle_mod, c, 150, "f32")
    fl = ~r["solid"]
    assert _rel(g["rho"], r["rho"], fl) < 1e-5
    assert _rel(g["T"], r["T"]) < 1e-5


def test_tprop_changes_the_temperature(oracle_mod):
    """The derived diffusivities are not the constant ones the descriptor also carries: the
    same case with tprop off ends at a different temperature, on the GPU and in the oracle."""
    c = _case(2, "bgk")
    off = c.cfg.replace(tprop_fluid=None, tprop_solid=None)
    g_on, g_off = _gpu(c, 150), _gpu(c, 150, cfg=off)
    assert _rel(g_on["T"], g_off["T"]) > 1e-3
    r_off = _oracle(oracle_mod, c, 150, "f64", cfg=off)
    assert _rel(g_off["T"], r_off["T"]) < 1e-10


def test_tprop_batch_equals_single_lattices():
    """A batch of lattices with derived diffusivities (each its own solid density) equals the
    lattices stepped one by one, bit for bit."""
    from lbm_porouschem_b200.lattice import Lattice, LatticeBatch
    cases = [_case(2, "bgk", precision="fp32"), _case(2, "bgk", precision="fp32")]
    cases[1].cfg = cases[1].cfg.replace(tp_rhos=3.0)
    ref = [_gpu(c, 40, cfg=c.cfg.replace(bulk_form="list")) for c in cases]
    lats = []
    for c in cases:
        lat = Lattice(c.cfg.replace(bulk_form="list"))
        lat.set_geometry(c.solid, c.reactive)
        lat.init(**c.init)
        lats.append(lat)
    batch = LatticeBatch(lats)
    batch.step(40)
    batch.synchronize()
    for lat, r in zip(lats, ref):
        got = lat.fields()
        for k in ("rho", "u", "T"):
            assert np.array_equal(got[k], r[k]), k
    assert not np.array_equal(ref[0]["T"], ref[1]["T"])
    batch.close()
    for lat in lats:
        lat.close()


@pytest.mark.parametrize("dim,thermal,suth,form", [(2, "conjugate", True, "list"), (2, "two_field", False, "tile"),
                                                   (3, "conjugate", True, "dense"), (3, "two_field", True, "list")])
def test_prandtl_fp64(oracle_mod, dim, thermal, suth, form):
    """THERMAL_DIFF_MODEL.PRANDTL: the fluid's diffusivity is the cell's kinetic viscosity
    (constant or Sutherland, over its density) / Pr; FP64 vs the FP64 oracle, 1e-10."""
    c = _case(dim, "mrt", thermal, suth=suth, shape=(32, 16, 12) if form == "dense" else None)
    c.cfg = c.cfg.replace(tprop_fluid=None, tp_prandtl=0.71)
    if thermal == "two_field":
        c.init["T"] = np.where(c.solid, 0.6, 0.2)
    n = 150 if dim == 2 else 60
    g, r = _gpu(c, n, cfg=c.cfg.replace(bulk_form=form)), _oracle(oracle_mod, c, n, "f64")
    fl = ~r["solid"]
    assert _rel(g["rho"], r["rho"], fl) < 1e-10
    assert _rel(g["u"], r["u"], fl) < 1e-10
    assert _rel(g["T"], r["T"]) < 1e-10
