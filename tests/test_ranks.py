"""Multi-rank host logic of the benchmark on CPU: two gloo ranks, as torchrun would start them.

The lattice update does not shard (each GPU runs an independent replica); what ranks share is the
barrier, the max-over-ranks time and the whole-job throughput, tested here with the same helpers
``bench.py`` uses."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        bench.rank_barrier(world)
        ms = [12.5, 20.0][rank]                       # rank 1 is the slow replica
        ms_max = bench.max_over_ranks(ms, world, "cpu")
        val = bench.job_mlups(1_000_000, 100, world, ms_max)
        from lbm_porouschem_b200 import workloads
        w = workloads.flow2d(64, 32, seed=bench.rank_seed(0, rank))
        q.put((rank, ms_max, val, int(w.solid.sum()), w.solid.tobytes()))
        bench.rank_barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_rank_replica_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, ms_max, val, nsolid, geo = q.get(timeout=120)
        out[r] = (ms_max, val, nsolid, geo)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 20.0               # both ranks report the slowest time
    assert out[0][1] == out[1][1] == pytest.approx(2 * 1e6 * 100 / 0.020 / 1e6)
    assert out[0][3] != out[1][3]                       # one geometry per replica
    assert out[0][2] > 0 and out[1][2] > 0


def test_launch_count_per_step():
    sys.path.insert(0, str(ROOT))
    import bench
    from lbm_porouschem_b200 import workloads
    assert bench.launches_per_step(workloads.flow2d(64, 32).cfg) == 1           # periodic, no pyrolysis
    assert bench.launches_per_step(workloads.pyro2d(64, 32).cfg) == 3           # bulk + sides + flip
    assert bench.launches_per_step(workloads.pyro3d(24).cfg) == 3


def test_reference_arm_nonzero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
