"""Batches: many lattices of uneven sizes stepped together must give the same bits as
stepping each one alone, also when the steps are replayed from a CUDA graph."""
import numpy as np
import pytest

from lbm_porouschem_b200 import workloads

pytestmark = pytest.mark.gpu

SIZES = ((64, 32), (96, 48), (128, 64), (160, 48))


def _fast(ws):
    for w in ws:
        w.cfg.pyro_A = 2.0e11      # hot start, fast rate: cells turn fluid within ~40 steps
        w.cfg.heat_norm = 0.02
        w.cfg.gas_coef = 0.05
        w.init["T"] = 1.0
    return ws


def _make(ws):
    from lbm_porouschem_b200.lattice import Lattice
    lats = []
    for w in ws:
        lat = Lattice(w.cfg)
        lat.set_geometry(w.solid, w.reactive)
        lat.init(**w.init)
        lats.append(lat)
    return lats


def _same(a, b):
    fa, fb = a.fields(), b.fields()
    for k in ("rho", "u", "T", "alpha", "solid"):
        assert np.array_equal(fa[k], fb[k]), k


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_batch_equals_single_steps(precision):
    from lbm_porouschem_b200.lattice import LatticeBatch
    ws = _fast(workloads.sweep2d(6, seed0=3, precision=precision, sizes=SIZES))
    single, batched = _make(ws), _make(ws)
    batch = LatticeBatch(batched)
    assert all(lat.bulk_kernel == "list" for lat in batched)
    batch.step(120)
    batch.synchronize()
    for lat in single:
        lat.step(120)
    flipped = 0
    for w, a, b in zip(ws, single, batched):
        assert a.nsteps == b.nsteps == 120
        _same(a, b)
        flipped += int((w.solid.reshape(a.cfg.shape) & ~b.fields()["solid"]).sum())
    assert flipped > 0
    batch.close()


def test_batch_graph_replay():
    from lbm_porouschem_b200.lattice import LatticeBatch
    ws = _fast(workloads.sweep2d(4, seed0=7, sizes=SIZES))
    single, batched = _make(ws), _make(ws)
    batch = LatticeBatch(batched)
    batch.step(2)
    batch.capture(10)
    for _ in range(3):
        batch.replay()
    batch.step(2)                      # ordinary steps after replays keep the parity
    batch.synchronize()
    for lat in single:
        lat.step(34)
    for a, b in zip(single, batched):
        assert b.nsteps == 34
        _same(a, b)
    batch.close()


def test_batch_members_are_checked():
    from lbm_porouschem_b200._native import LBMNativeError
    from lbm_porouschem_b200.lattice import LatticeBatch
    ws = workloads.sweep2d(2, seed0=1, sizes=SIZES)
    ws[1].cfg.bulk_form = "tile"
    with pytest.raises(LBMNativeError, match="cell lists"):
        LatticeBatch(_make(ws))
    ws = workloads.sweep2d(2, seed0=1, sizes=SIZES)
    ws[1].cfg.precision = "fp64"
    with pytest.raises(LBMNativeError, match="share"):
        LatticeBatch(_make(ws))


def test_batch_tune_steps_are_real_steps():
    from lbm_porouschem_b200.lattice import LatticeBatch
    ws = _fast(workloads.sweep2d(3, seed0=11, sizes=SIZES))
    single, batched = _make(ws), _make(ws)
    batch = LatticeBatch(batched)
    times = batch.tune(steps=2, candidates=(2, 4))
    assert set(times) == {2, 4} and batch.blocks_per_sm in (2, 4)
    batch.step(6)
    batch.synchronize()
    n = batched[0].nsteps
    assert n == 2 * (2 + 2) + 6
    for lat in single:
        lat.step(n)
    for a, b in zip(single, batched):
        _same(a, b)
    batch.close()
