"""The cell-list bulk kernel (LBM_BULK=list; the default from 65536 cells) against the
tile kernel (LBM_BULK=tile).

Both forms run the same per-cell arithmetic, so every field must agree bit for bit,
through solid->fluid flips (which append list entries and clear neighbour bits),
on lattices with and without interior cells, in every storage precision.  The
diagnostics are FP64 sums over a different block order: equal to 1e-12."""
import numpy as np
import pytest

from lbm_porouschem_b200 import workloads
from lbm_porouschem_b200.config import FIXED_VALUE, PERIODIC, ZERO_GRADIENT, LatticeConfig, SideBC

pytestmark = pytest.mark.gpu


def _fast_pyro(w, A):
    w.cfg.pyro_A = A
    w.cfg.heat_norm = 0.02
    w.cfg.gas_coef = 0.05
    w.init["T"] = 1.0
    return w


def _run(w, steps, kind, monkeypatch, diag=False):
    from lbm_porouschem_b200.lattice import Lattice
    monkeypatch.setenv("LBM_BULK", kind)   # lattices below 65536 cells default to the tile form
    lat = Lattice(w.cfg)
    assert lat.bulk_kernel == kind
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
def test_list_equals_tile_pyro3d_with_flips(precision, coll, monkeypatch):
    w = _fast_pyro(workloads.pyro3d(40, seed=11, ny=24, nz=20, precision=precision, collision=coll), A=1.2e11)
    a, da, pa = _run(w, 80, "list", monkeypatch, diag=True)
    b, db, pb = _run(w, 80, "tile", monkeypatch, diag=True)
    assert (w.solid & ~a["solid"]).any()          # cells turned fluid on the way
    _same(a, b)
    for k in ("mass", "energy", "solid_alpha", "nfluid"):
        assert da[k] == pytest.approx(db[k], rel=1e-12), k
        assert pa[k] == pytest.approx(pb[k], rel=1e-12), k
    for k in ("umax", "Tmin", "Tmax"):
        assert da[k] == db[k] and pa[k] == pb[k], k


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_list_equals_tile_pyro2d_with_flips(coll, monkeypatch):
    w = _fast_pyro(workloads.pyro2d(160, 80, seed=12, collision=coll), A=4.5e10)
    n = 150 if coll == "bgk" else 300              # BGK: a cell turns fluid on the last pass
    a, _, pa = _run(w, n, "list", monkeypatch)
    b, _, pb = _run(w, n, "tile", monkeypatch)
    assert (w.solid.reshape(a["solid"].shape) & ~a["solid"]).any()
    _same(a, b)
    assert pa["mass"] == pytest.approx(pb["mass"], rel=1e-12)


def test_list_equals_tile_flow2d_periodic(monkeypatch):
    w = workloads.flow2d(96, 64, seed=13)
    w.cfg.force = (1e-5, 0.0, 0.0)
    a, _, _ = _run(w, 200, "list", monkeypatch)
    b, _, _ = _run(w, 200, "tile", monkeypatch)
    _same(a, b, ("rho", "u", "solid"))


def test_list_equals_tile_mostly_wrapping_cells(monkeypatch):
    """24 x 3 x 3: all cells but one x row wrap in y or z, so nearly every entry is in a
    general segment."""
    rng = np.random.default_rng(14)
    solid = rng.random((24, 3, 3)) < 0.3
    solid[:2] = solid[-2:] = False          # NEE sides and their inner neighbours are fluid
    cfg = LatticeConfig(dim=3, nx=24, ny=3, nz=3, collision="mrt", nu=0.05, thermal="conjugate", pyro=True,
                        pyro_A=1.2e11, heat_norm=0.02, gas_coef=0.05,
                        sides=[SideBC.pressure(1.001), SideBC.outlet(1.0)] + [SideBC() for _ in range(4)])

    class W:
        pass

    w = W()
    w.cfg, w.solid, w.reactive = cfg, solid, solid
    w.init = {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 1.0}
    a, _, _ = _run(w, 60, "list", monkeypatch)
    b, _, _ = _run(w, 60, "tile", monkeypatch)
    assert (solid & ~a["solid"]).any()
    assert np.isfinite(a["T"]).all()
    for n in (59, 60, 61):   # a peek right after passes with and without flips
        a, _, _ = _run(w, n, "list", monkeypatch)
        b, _, _ = _run(w, n, "tile", monkeypatch)
        _same(a, b)


class _W:
    pass


@pytest.mark.parametrize("dim", [2, 3])
def test_list_equals_tile_with_corner_cells(dim, monkeypatch):
    """Every side active in 2D (x, y and z in 3D, odd sizes): corner cells take two or
    three NEE passes, some with a side's own state (PERIODIC types keep it), some
    without."""
    rng = np.random.default_rng(15 + dim)
    shape = (45, 37) if dim == 2 else (21, 19, 13)
    solid = rng.random(shape) < 0.25
    keep = np.zeros(shape, dtype=bool)
    keep[tuple(slice(2, n - 2) for n in shape)] = True
    solid &= keep                           # sides and their inner neighbours fluid
    sides = [SideBC.inlet((0.02, 0.0, 0.0), FIXED_VALUE, 1.0),
             SideBC.outlet(1.0),                                   # T keeps the cell's own
             SideBC.wall(FIXED_VALUE, 0.5),
             SideBC(True, PERIODIC, FIXED_VALUE, ZERO_GRADIENT)]  # v keeps the cell's own
    sides += ([SideBC.wall(ZERO_GRADIENT), SideBC(True, ZERO_GRADIENT, PERIODIC, FIXED_VALUE, T=0.2)]
              if dim == 3 else [SideBC(), SideBC()])
    nz = shape[2] if dim == 3 else 1
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=nz, collision="mrt", nu=0.05, thermal="conjugate",
                        pyro=True, pyro_A=1.2e11, heat_norm=0.02, gas_coef=0.05, sides=sides)
    w = _W()
    w.cfg, w.solid, w.reactive = cfg, solid, solid
    w.init = {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 1.0}
    a, da, pa = _run(w, 70, "list", monkeypatch, diag=True)
    b, db, pb = _run(w, 70, "tile", monkeypatch, diag=True)
    assert np.isfinite(a["u"]).all()
    _same(a, b)
    for k in ("mass", "energy", "solid_alpha", "nfluid"):
        assert da[k] == pytest.approx(db[k], rel=1e-12), k
        assert pa[k] == pytest.approx(pb[k], rel=1e-12), k
    for k in ("umax", "Tmin", "Tmax"):
        assert da[k] == db[k] and pa[k] == pb[k], k


@pytest.mark.parametrize("x", [0, 1, 30, 31])
def test_solid_cell_on_or_next_to_an_active_side_is_rejected(x):
    """NEE overwrites every population of a side cell from its inner neighbour's, so both
    must be fluid."""
    from lbm_porouschem_b200._native import LBMNativeError
    from lbm_porouschem_b200.lattice import Lattice
    cfg = LatticeConfig(dim=2, nx=32, ny=16, nz=1, sides=[SideBC.pressure(1.001), SideBC.outlet(1.0)]
                        + [SideBC() for _ in range(4)])
    solid = np.zeros((32, 16), dtype=bool)
    solid[x, 5] = True
    lat = Lattice(cfg)
    lat.set_geometry(solid)
    with pytest.raises(LBMNativeError, match="active"):
        lat.init()
    lat.close()
