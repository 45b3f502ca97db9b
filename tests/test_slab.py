"""Slab decomposition of one 3D lattice along z (``lbm_porouschem_b200.slab``): host logic on the CPU.

The per-rank stepper here is the oracle, whose per-cell state is exposed as arrays (test
infrastructure); the partition, the ghost-plane mapping and the exchange are the package's:
``exchange_local`` for slabs in one process and ``DistExchange`` between two gloo ranks (the
transport torchrun gives the GPU ranks, with NCCL there).  The decomposed run must equal the
undivided run bit for bit, through solid -> fluid flips next to the slab edges, since every
cell's update reads only its own state and that of cells at most two planes away.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
STEPS = 40
# the oracle's state in exchange order: the mask bytes last (the packed buffer stays aligned)
ORDER = ("f", "g", "rho", "u", "T", "dS", "alpha", "rel", "gs", "Ts", "dSs", "mask")


def _case(nz=16):
    from lbm_porouschem_b200 import workloads
    w = workloads.pyro3d(24, seed=4, ny=12, nz=nz, collision="mrt", precision="fp64")
    cfg = w.cfg.replace(pyro_A=2e11, heat_norm=0.02, gas_coef=0.05)   # cells convert within the run
    init = dict(w.init, T=1.0)
    return cfg, w.solid.reshape(cfg.shape), w.reactive.reshape(cfg.shape), init


class OracleSlabs:
    """One oracle per slab of `plan` (ranks `ranks`), initialised from the global inputs."""

    def __init__(self, oracle_mod, cfg, plan, solid, reactive, init, ranks):
        from lbm_porouschem_b200.slab import local_config, local_slice
        self.plan, self.ranks = plan, list(ranks)
        self.orcs = []
        for r in self.ranks:
            o = oracle_mod.Oracle(local_config(cfg, plan, r), real="f64")
            loc = lambda a: local_slice(a, plan, r, cfg.shape)    # noqa: E731
            o.init(loc(solid), loc(reactive), **{k: loc(v) for k, v in init.items()})
            self.orcs.append(o)

    def views(self, i):
        st = self.orcs[i].state_arrays()
        v = [st[k] for k in ORDER if k in st]
        return v, [0] * len(v)

    def interior(self, i):
        f = self.orcs[i].fields()
        return {k: v[..., self.plan.interior(self.ranks[i])] for k, v in f.items()}


def test_plan_partition():
    from lbm_porouschem_b200.slab import SlabPlan
    p = SlabPlan(nz=10, nranks=3, halo=2)
    assert p.counts == [4, 3, 3] and p.starts == [0, 4, 7]
    assert list(p.planes(0)) == [8, 9, 0, 1, 2, 3, 4, 5]
    assert list(p.planes(2)) == [5, 6, 7, 8, 9, 0, 1]
    assert p.interior(1) == slice(2, 5) and p.below(0) == 2 and p.above(2) == 0
    with pytest.raises(ValueError):
        SlabPlan(nz=5, nranks=3, halo=2)


def test_local_config_limits():
    from lbm_porouschem_b200.config import SideBC
    from lbm_porouschem_b200.slab import SlabPlan, local_config
    cfg, *_ = _case()
    plan = SlabPlan(cfg.nz, 2)
    lc = local_config(cfg, plan, 1)
    assert lc.nz == plan.local_nz(1) and lc.bulk_form == "tile"
    walled = cfg.replace(sides=[*cfg.sides[:4], SideBC.wall(), SideBC.wall()])
    with pytest.raises(ValueError, match="periodic"):
        local_config(walled, plan, 0)


@pytest.mark.parametrize("nslabs", [1, 3])
def test_slabs_in_one_process_equal_the_whole_lattice(oracle_mod, nslabs):
    from lbm_porouschem_b200.slab import SlabPlan, exchange_local
    cfg, solid, reactive, init = _case()
    whole = oracle_mod.Oracle(cfg, real="f64")
    whole.init(solid, reactive, **init)
    whole.step(STEPS)
    ref = whole.fields()
    plan = SlabPlan(cfg.nz, nslabs)
    slabs = OracleSlabs(oracle_mod, cfg, plan, solid, reactive, init, range(nslabs))
    for _ in range(STEPS):
        for o in slabs.orcs:
            o.step(1)
        views = [slabs.views(i) for i in range(nslabs)]
        exchange_local([v for v, _ in views], views[0][1], plan)
    parts = [slabs.interior(i) for i in range(nslabs)]
    got = {k: np.concatenate([p[k] for p in parts], axis=-1) for k in ref}
    assert (solid & ~ref["solid"]).sum() >= 3          # cells turned fluid during the run
    for k in ("rho", "u", "T", "alpha", "solid"):
        assert np.array_equal(got[k], ref[k]), k


def test_ghost_planes_matter(oracle_mod):
    """Without the exchange the slabs drift from the whole lattice (the test can fail)."""
    from lbm_porouschem_b200.slab import SlabPlan
    cfg, solid, reactive, init = _case()
    whole = oracle_mod.Oracle(cfg, real="f64")
    whole.init(solid, reactive, **init)
    whole.step(STEPS)
    plan = SlabPlan(cfg.nz, 2)
    slabs = OracleSlabs(oracle_mod, cfg, plan, solid, reactive, init, range(2))
    for o in slabs.orcs:
        o.step(STEPS)
    got = np.concatenate([slabs.interior(i)["rho"] for i in range(2)], axis=-1)
    assert not np.array_equal(got, whole.fields()["rho"])


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as oracle_mod
    from lbm_porouschem_b200.slab import DistExchange, SlabPlan
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, solid, reactive, init = _case()
        plan = SlabPlan(cfg.nz, world)
        slabs = OracleSlabs(oracle_mod, cfg, plan, solid, reactive, init, [rank])
        ex = DistExchange(plan, rank)
        for _ in range(STEPS):
            slabs.orcs[0].step(1)
            ex(*slabs.views(0))
        mine = slabs.interior(0)
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        if rank == 0:
            q.put({k: np.concatenate([p[k] for p in parts], axis=-1) for k in mine})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_the_whole_lattice(oracle_mod):
    cfg, solid, reactive, init = _case()
    whole = oracle_mod.Oracle(cfg, real="f64")
    whole.init(solid, reactive, **init)
    whole.step(STEPS)
    ref = whole.fields()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for k in ("rho", "u", "T", "alpha", "solid"):
        assert np.array_equal(got[k], ref[k]), k
