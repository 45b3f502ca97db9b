"""The dense TMA-staged bulk kernel (bulk_form="dense", 3D) against the tile kernel and
the oracle, and its bounded-wait failure path.

The dense kernel runs the same per-cell arithmetic as the tile and cell-list kernels
(cell_update), fed from shared-memory boxes instead of global loads, so every field must
agree with the tile form bit for bit: through solid->fluid flips, on tiles that touch a
periodic edge (global pulls) and on tiles next to active sides (boxes partly out of
bounds), in every storage precision.  The diagnostics are FP64 sums in another block
order: equal to 1e-12.  Against the FP64 oracle: 1e-10 relative L2.
"""
import numpy as np
import pytest

from lbm_porouschem_b200 import workloads
from lbm_porouschem_b200.config import FIXED_VALUE, ZERO_GRADIENT, LatticeConfig, SideBC

pytestmark = pytest.mark.gpu


def _fast_pyro(w, A=1.2e11):
    w.cfg.pyro_A = A
    w.cfg.heat_norm = 0.02
    w.cfg.gas_coef = 0.05
    w.init["T"] = 1.0
    return w


def _run(w, steps, form, diag=False, cfg=None):
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice((cfg or w.cfg).replace(bulk_form=form))
    assert lat.bulk_kernel == form
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(steps, diag=diag)
    out = lat.fields()
    d = lat.read_diag() if diag else None
    peek = lat.diagnostics()
    lat.close()
    return out, d, peek


def _same(a, b, keys=("rho", "u", "T", "alpha", "solid")):
    for k in keys:
        if k in a:
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("precision", ["fp32", "fp16", "fp64"])
@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_dense_equals_tile_pyro3d_with_flips(precision, coll):
    # x: pressure inlet / outlet (active sides), y and z periodic (edge tiles)
    w = _fast_pyro(workloads.pyro3d(64, seed=11, ny=24, nz=20, precision=precision, collision=coll))
    a, da, pa = _run(w, 80, "dense", diag=True)
    b, db, pb = _run(w, 80, "tile", diag=True)
    assert (w.solid & ~a["solid"]).any()          # cells turned fluid on the way
    _same(a, b)
    for k in ("mass", "energy", "solid_alpha", "nfluid"):
        assert da[k] == pytest.approx(db[k], rel=1e-12), k
        assert pa[k] == pytest.approx(pb[k], rel=1e-12), k
    for k in ("umax", "Tmin", "Tmax"):
        assert da[k] == db[k] and pa[k] == pb[k], k


def test_dense_equals_tile_all_periodic_flow():
    """No active side: every tile on the lattice's faces wraps (x too)."""
    w = workloads.pyro3d(64, seed=3, ny=16, nz=12)
    cfg = w.cfg.replace(thermal="none", pyro=False, sides=[SideBC() for _ in range(6)], force=(1e-5, 0, 0))
    w = workloads.Workload(w.name, cfg, w.solid, None, {"rho": 1.0, "u": (0.0, 0.0, 0.0)})
    a, _, _ = _run(w, 60, "dense")
    b, _, _ = _run(w, 60, "tile")
    _same(a, b, ("rho", "u", "solid"))


def test_dense_equals_tile_walls_and_heat():
    """Walls on y and z (active sides on every face): boxes reach out of the domain,
    tiles never wrap."""
    w = workloads.pyro3d(64, seed=4, ny=16, nz=12)
    sides = list(w.cfg.sides)
    for s in (2, 3, 4, 5):
        sides[s] = SideBC.wall(T_type=ZERO_GRADIENT)
    cfg = w.cfg.replace(pyro=False, sides=sides)
    solid = w.solid.copy()
    solid[:, :2], solid[:, -2:], solid[:, :, :2], solid[:, :, -2:] = False, False, False, False
    w = workloads.Workload(w.name, cfg, solid, None, {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 0.25})
    a, _, _ = _run(w, 60, "dense")
    b, _, _ = _run(w, 60, "tile")
    _same(a, b, ("rho", "u", "T", "solid"))


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_dense_fp64_vs_oracle_with_flips(oracle_mod, coll):
    from lbm_porouschem_b200.lattice import Lattice
    w = _fast_pyro(workloads.pyro3d(64, seed=5, ny=12, nz=10, collision=coll, precision="fp64"))
    lat = Lattice(w.cfg.replace(bulk_form="dense"))
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(120)
    g = lat.fields()
    lat.close()
    o = oracle_mod.Oracle(w.cfg, real="f64")
    o.init(w.solid, w.reactive, **w.init)
    o.step(120)
    r = o.fields()
    assert np.array_equal(g["solid"], r["solid"])
    assert (w.solid & ~r["solid"]).any()
    fl = ~r["solid"]

    def rel(x, y):
        return np.linalg.norm(x - y) / np.linalg.norm(y)

    assert rel(g["rho"][fl], r["rho"][fl]) < 1e-10
    assert rel(g["u"][:, fl], r["u"][:, fl]) < 1e-10
    assert rel(g["T"], r["T"]) < 1e-10


def test_dense_rejects_unsupported_shapes():
    from lbm_porouschem_b200._native import LBMNativeError
    from lbm_porouschem_b200.lattice import Lattice
    cfg = LatticeConfig(dim=3, nx=40, ny=16, nz=8, bulk_form="dense")   # nx % 32 != 0
    with pytest.raises(LBMNativeError):
        Lattice(cfg)
    cfg = LatticeConfig(dim=3, nx=32, ny=16, nz=8, thermal="two_field", bulk_form="dense")
    with pytest.raises(LBMNativeError):
        Lattice(cfg)


def test_dense_wait_timeout_is_reported_and_device_stays_usable():
    """A staged-load wait that gives up at once (wait limit 0): the kernel records the
    timeout, lets its copies land and ends; lbm_read_diag reports LBM_ERR_TIMEOUT; the
    context is still usable (a fresh lattice steps normally)."""
    from lbm_porouschem_b200 import _native as N
    from lbm_porouschem_b200.lattice import Lattice
    w = workloads.pyro3d(64, seed=6, ny=16, nz=8)
    lat = Lattice(w.cfg.replace(bulk_form="dense"))
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.set_wait_limit(0)
    lat.step(2, diag=True)
    with pytest.raises(N.LBMNativeError) as e:
        lat.read_diag()
    assert e.value.code == N.LBM_ERR_TIMEOUT
    with pytest.raises(N.LBMNativeError) as e:      # the asynchronous read reports it too
        lat.read_diag_async().result()
    assert e.value.code == N.LBM_ERR_TIMEOUT
    lat.close()
    b = Lattice(w.cfg.replace(bulk_form="dense"))
    b.set_geometry(w.solid, w.reactive)
    b.init(**w.init)
    b.step(4, diag=True)
    d = b.read_diag()
    assert d["nonfinite"] == 0 and d["step"] == 4
    b.close()
