"""Flow-rate inlet (LBM_BC_FLOWRATE, the reference's BC_FLOW.inlet_flow with its
per-step controller, src/LBM/LBM2D/_boundary.py:324-333) on the CUDA path, called
through the C ABI, against the C oracle.

Tolerances: FP64 storage vs the FP64 oracle 1e-10 relative L2 for rho, u and T, as in
the other FP64 parity cases (the kernels sum the inlet flux in a different order, in
FP64, so the controller's coefficient differs in the last bits only).  FP32 vs the
FP32 oracle: 1e-5 for rho; u against the FP64 oracle within 2x the FP32 oracle's own
error (plus 1e-9).  A resumed checkpoint and CUDA-graph replays give the fields of the
plain run bit for bit."""
import numpy as np
import pytest
import torch

from lbm_porouschem_b200.config import FIXED_VALUE, LatticeConfig, SideBC
from lbm_porouschem_b200.geometry import packing

pytestmark = pytest.mark.gpu


def _rel(a, b, mask):
    a, b = np.asarray(a, np.float64)[..., mask], np.asarray(b, np.float64)[..., mask]
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


class _Case:
    pass


def _case(dim, coll="bgk", thermal=False, precision="fp64", F=0.1):
    """Channel with walls at y = 0 / ny-1 (corner cells), a disk or sphere packing in the
    middle, flow-rate inlet at x = 0, pressure outlet at x = nx-1; periodic in z."""
    shape = (48, 22) if dim == 2 else (28, 14, 10)
    solid = packing(shape, 1.5, 3.0, 0.75, seed=5 + dim)
    keep = np.zeros(shape, dtype=bool)
    keep[(slice(3, shape[0] - 3), slice(3, shape[1] - 3)) + ((slice(None),) if dim == 3 else ())] = True
    solid &= keep
    T_in = FIXED_VALUE if thermal else 0
    sides = [SideBC.inlet_flowrate(F, T_in, 1.0), SideBC.outlet(1.0), SideBC.wall(), SideBC.wall(),
             SideBC(), SideBC()]
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=1 if dim == 2 else shape[2], collision=coll,
                        nu=0.08, precision=precision, sides=sides,
                        thermal="conjugate" if thermal else "none")
    c = _Case()
    c.cfg, c.solid = cfg, solid
    c.init = {"rho": 1.0, "u": (0.0, 0.0, 0.0)}
    if thermal:
        c.init["T"] = 0.2
    return c


def _gpu(c, n, bulk=None, monkeypatch=None):
    from lbm_porouschem_b200.lattice import Lattice
    if bulk:
        monkeypatch.setenv("LBM_BULK", bulk)
    lat = Lattice(c.cfg)
    lat.set_geometry(c.solid)
    lat.init(**c.init)
    lat.step(n)
    out = lat.fields()
    lat.close()
    return out


def _oracle(oracle_mod, c, n, real):
    o = oracle_mod.Oracle(c.cfg, real=real)
    o.init(c.solid, **c.init)
    o.step(n)
    out = o.fields()
    o.close()
    return out


@pytest.mark.parametrize("dim,coll,thermal,bulk", [(2, "bgk", False, "list"), (2, "mrt", True, "tile"),
                                                   (2, "bgk", True, "list"), (3, "bgk", False, "list"),
                                                   (3, "mrt", True, "tile")])
def test_flowrate_inlet_fp64(oracle_mod, monkeypatch, dim, coll, thermal, bulk):
    c = _case(dim, coll, thermal)
    n = 240 if dim == 2 else 120
    g, r = _gpu(c, n, bulk, monkeypatch), _oracle(oracle_mod, c, n, "f64")
    fl = ~r["solid"]
    assert np.array_equal(g["solid"], r["solid"])
    assert _rel(g["rho"], r["rho"], fl) < 1e-10
    assert _rel(g["u"], r["u"], fl) < 1e-10
    if thermal:
        assert _rel(g["T"], r["T"], np.ones_like(fl)) < 1e-10
    # the inlet is steered: its velocity follows the controller, not the initial v0
    v0 = c.cfg.sides[0].v[0] / c.cfg.ny / c.cfg.nz
    assert not np.allclose(g["u"][0][0], v0)


def test_flowrate_inlet_fp32(oracle_mod):
    c = _case(2, "mrt", True, precision="fp32")
    n = 240
    g = _gpu(c, n)
    r32, r64 = _oracle(oracle_mod, c, n, "f32"), _oracle(oracle_mod, c, n, "f64")
    fl = ~r64["solid"]
    assert _rel(g["rho"], r32["rho"], fl) < 1e-5
    assert _rel(g["T"], r32["T"], np.ones_like(fl)) < 1e-5
    assert _rel(g["u"], r64["u"], fl) <= 2 * _rel(r32["u"], r64["u"], fl) + 1e-9


def test_flowrate_inlet_resume_and_graph(tmp_path):
    """Saved after an odd step and resumed (LBM_FIELD_INLET travels with the state), and
    stepped by replays of a captured graph (the coefficient kernel is inside it): both
    equal the plain run."""
    from lbm_porouschem_b200.lattice import Lattice
    c = _case(2, "mrt", True)
    ref = _gpu(c, 151)

    lat = Lattice(c.cfg)
    lat.set_geometry(c.solid)
    lat.init(**c.init)
    lat.step(71)
    path = lat.save_checkpoint(tmp_path / "fr.npz")
    lat.close()
    back = Lattice.load_checkpoint(path)
    back.step(80)
    got = back.fields()
    back.close()
    for k in ("rho", "u", "T"):
        assert np.array_equal(got[k], ref[k]), k

    lat = Lattice(c.cfg, stream=torch.cuda.Stream())
    lat.set_geometry(c.solid)
    lat.init(**c.init)
    with torch.cuda.stream(lat.stream):
        lat.step(31)
    lat.capture(40)
    for _ in range(3):
        lat.replay()
    assert lat.nsteps == 151
    got = lat.fields()
    lat.close()
    for k in ("rho", "u", "T"):
        assert np.array_equal(got[k], ref[k]), k


def test_flowrate_rejected_off_side_0_and_in_batches():
    from lbm_porouschem_b200 import _native as N
    from lbm_porouschem_b200.lattice import Lattice, LatticeBatch
    c = _case(2)
    bad = c.cfg.replace(sides=[SideBC.outlet(1.0), SideBC.inlet_flowrate(0.1)] + c.cfg.sides[2:])
    with pytest.raises(N.LBMNativeError, match="side 0"):
        Lattice(bad)
    lat = Lattice(c.cfg.replace(bulk_form="list"))
    lat.set_geometry(c.solid)
    lat.init(**c.init)
    with pytest.raises(N.LBMNativeError, match="flow-rate"):
        LatticeBatch([lat])
    lat.close()
