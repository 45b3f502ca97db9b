"""lbm_diag_noalloc: diagnostics for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc: a plug-in whose host
application owns every device allocation through its own memory pool, or a
monitoring hook inside a latency-critical time loop where an allocation (which
may synchronise the whole device) is not allowed.  lbm_diag_noalloc gives them
the diagnostics of the current lattice state using a static device array as
scratch.  These tests call it through the C ABI and check it against the
allocating path (lbm_compute_macro + lbm_read_diag) on two calls in a row, and
check that a lattice too large for the static array is refused.
"""
import ctypes

import numpy as np
import pytest

from lbm_porouschem_b200 import _native as N
from lbm_porouschem_b200 import workloads

pytestmark = pytest.mark.gpu

KEYS = ("mass", "energy", "solid_alpha", "umax", "Tmin", "Tmax", "nfluid", "nonfinite")


def _noalloc(lat):
    d = N.lbm_diag()
    N.check(lat.lib.lbm_diag_noalloc(lat._h, ctypes.byref(d), lat._s()))
    return {k: getattr(d, k) for k, _ in N.lbm_diag._fields_}


def _allocating(lat):
    return lat.diagnostics()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_allocating_path_twice(precision):
    from lbm_porouschem_b200.lattice import Lattice
    w = workloads.pyro2d(64, 40, seed=11, precision=precision)
    w.cfg.pyro_A = 4.5e10
    w.cfg.heat_norm = 0.02
    w.cfg.gas_coef = 0.05
    w.init["T"] = 1.0
    lat = Lattice(w.cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    rtol = 1e-12 if precision == "fp64" else 1e-6
    for nsteps in (37, 180):            # the second call follows further steps (cells convert)
        lat.step(nsteps)
        a = _noalloc(lat)
        b = _allocating(lat)
        assert a["step"] == b["step"] == lat.nsteps
        for k in KEYS:
            assert a[k] == pytest.approx(b[k], rel=rtol, abs=1e-12), k
    assert a["nfluid"] > 0 and np.isfinite(a["mass"])
    lat.close()


@pytest.mark.parametrize("form", ["list", "dense"])
@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_noalloc_matches_allocating_path_3d_lists(precision, form):
    """The forms lattices from 65536 cells run: cell lists (kept in the lattice's own SCRATCH
    buffer) or dense tiles, with the boundary kernel on its side stream (pressure inlet and
    outlet on x), in 3D; two calls separated by steps in which reactive cells turn fluid."""
    from lbm_porouschem_b200.lattice import Lattice
    w = workloads.pyro3d(64, seed=13, ny=40, nz=32, precision=precision)   # 81920 cells
    w.cfg.pyro_A = 1.2e11
    w.cfg.heat_norm = 0.02
    w.cfg.gas_coef = 0.05
    w.init["T"] = 1.0
    lat = Lattice(w.cfg.replace(bulk_form=form))
    assert lat.bulk_kernel == form
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    for nsteps in (23, 60):
        lat.step(nsteps)
        a = _noalloc(lat)
        b = _allocating(lat)
        assert a["step"] == b["step"] == lat.nsteps
        for k in KEYS:
            assert a[k] == pytest.approx(b[k], rel=1e-6, abs=1e-12), k
    assert (w.solid & ~lat.fields()["solid"]).any()     # cells converted between the calls
    lat.close()


def test_noalloc_rejects_lattice_beyond_static_scratch(monkeypatch):
    from lbm_porouschem_b200.config import LatticeConfig
    from lbm_porouschem_b200.lattice import Lattice
    # 32 x 200 x 200 with the tile form of the bulk update: one 32-wide block per
    # (y, z) row -> 40000 partial rows > 32768 (the cell-list form needs a few hundred)
    monkeypatch.setenv("LBM_BULK", "tile")
    cfg = LatticeConfig(dim=3, nx=32, ny=200, nz=200, nu=0.1)
    lat = Lattice(cfg)
    assert lat.bulk_kernel == "tile"
    lat.set_geometry(np.zeros(cfg.shape, dtype=bool))
    lat.init()
    lat.step(1)
    d = N.lbm_diag()
    rc = lat.lib.lbm_diag_noalloc(lat._h, ctypes.byref(d), lat._s())
    assert rc == N.LBM_ERR_SIZE
    assert b"LBM_NOALLOC_MAX_ROWS" in lat.lib.lbm_last_error()
    lat.close()
