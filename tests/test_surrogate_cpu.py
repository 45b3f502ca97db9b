"""Host-side parts of the learned warm start that need no GPU."""
import numpy as np


def _div(vx, vy):
    """The discrete divergence project_solenoidal zeroes: minus the adjoint of forward
    differences (no flux through the x walls, periodic in y)."""
    d = np.zeros_like(vx)
    d[:-1] += vx[:-1]
    d[1:] -= vx[:-1]
    d += vy - np.roll(vy, 1, axis=1)
    return d


def test_projection_is_divergence_free_and_keeps_solenoidal_fields():
    from lbm_porouschem_b200.surrogate import project_solenoidal
    S = 24
    rng = np.random.default_rng(1)
    ux, uy = rng.normal(size=(S, S)), rng.normal(size=(S, S))
    vx, vy = project_solenoidal(ux, uy, np.zeros((S, S), dtype=bool))
    assert np.abs(_div(ux, uy)).max() > 1.0
    assert np.abs(_div(vx, vy)).max() < 1e-6
    # a uniform flow along the periodic direction has no divergence: kept as it is
    wx, wy = project_solenoidal(np.zeros((S, S)), np.full((S, S), 0.3), np.zeros((S, S), dtype=bool))
    assert np.allclose(wy, 0.3, atol=1e-6) and np.allclose(wx, 0.0, atol=1e-6)


def test_projection_zeroes_the_solid():
    from lbm_porouschem_b200.surrogate import project_solenoidal
    S = 20
    solid = np.zeros((S, S), dtype=bool)
    solid[8:12, 5:9] = True
    vx, vy = project_solenoidal(np.ones((S, S)), np.ones((S, S)), solid)
    assert np.all(vx[solid] == 0) and np.all(vy[solid] == 0)
