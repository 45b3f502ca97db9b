"""A single lattice stepped by replays of a captured CUDA graph (Lattice.capture / replay,
lbm_advance) equals the same lattice stepped by lbm_step calls, bit for bit, through
solid->fluid flips, in both bulk forms."""
import numpy as np
import pytest
import torch

from lbm_porouschem_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bulk", ["list", "tile"])
def test_graph_replay_equals_eager_steps(bulk, monkeypatch):
    from lbm_porouschem_b200.lattice import Lattice
    monkeypatch.setenv("LBM_BULK", bulk)
    w = workloads.pyro2d(96, 64, seed=7)
    w.cfg.pyro_A, w.cfg.heat_norm, w.cfg.gas_coef = 4.5e10, 0.02, 0.05
    w.init["T"] = 1.0
    out = []
    for graph in (False, True):
        lat = Lattice(w.cfg, stream=torch.cuda.Stream())
        lat.set_geometry(w.solid, w.reactive)
        lat.init(**w.init)
        with torch.cuda.stream(lat.stream):
            lat.step(10)
        if graph:
            lat.capture(40)
            for _ in range(4):
                lat.replay()
        else:
            lat.step(160)
        assert lat.nsteps == 170
        out.append(lat.fields())
        lat.close()
    a, b = out
    assert (w.solid & ~a["solid"].reshape(w.solid.shape)).any()      # flips happened
    for k in ("rho", "u", "T", "alpha", "solid"):
        assert np.array_equal(a[k], b[k]), k
