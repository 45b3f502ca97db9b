"""Seeded packings: deterministic, hit the porosity target, respect margins; the
flat device order round-trips."""
import numpy as np

from lbm_porouschem_b200.geometry import fortran_flat, from_flat, mask_bytes, packing
from lbm_porouschem_b200 import workloads


def test_packing_deterministic_and_porosity():
    a = packing((128, 64), 4, 8, 0.65, seed=7, allow_overlap=False)
    b = packing((128, 64), 4, 8, 0.65, seed=7, allow_overlap=False)
    assert np.array_equal(a, b)
    phi = 1 - a.mean()
    assert 0.55 < phi <= 0.65


def test_packing_margin_keeps_boundary_fluid():
    m = packing((96, 48), 5, 9, 0.45, seed=2, periodic=(False, False), margin=3)
    assert not m[:3].any() and not m[-3:].any()
    assert not m[:, :3].any() and not m[:, -3:].any()


def test_sphere_packing_overlap_reaches_target():
    m = packing((48, 40, 40), 3, 6, 0.40, seed=1, periodic=(False, True, True), margin=3, max_attempts=500)
    assert 0.3 < 1 - m.mean() <= 0.40
    assert not m[:3].any() and not m[-3:].any()


def test_flat_round_trip():
    rng = np.random.default_rng(0)
    a = rng.random((5, 4, 3))
    v = fortran_flat(a)
    assert v[1 + 5 * (2 + 4 * 1)] == a[1, 2, 1]
    assert np.array_equal(from_flat(v, a.shape), a)
    s = rng.random((6, 3)) > 0.5
    m = mask_bytes(s, s)
    assert set(np.unique(m)) <= {0, 5}


def test_workload_builders_small():
    w = workloads.flow2d(64, 32, seed=0)
    assert w.cfg.dim == 2 and w.solid.shape == (64, 32)
    w = workloads.pyro2d(64, 32, seed=0)
    assert w.cfg.pyro and w.reactive is not None
    w = workloads.pyro3d(24, seed=0)
    assert w.solid.shape == (24, 24, 24)
    b = workloads.algorithmic_bytes_per_step(w.cfg, w.solid)
    assert b > 0
