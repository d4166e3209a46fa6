"""The N-GPU path of bench.py on CPU: two gloo ranks.  Each rank runs an
independent replica (its own seeded photons and queries, no exchange on the
data path); the only collective is the max over ranks of the timed region's
device time, and rank 0 alone prints."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.rank_max([10.0 * (rank + 1), 5.0 - rank])
        q.put((rank, got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_rank_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1] == [20.0, 5.0]


def test_rank_max_without_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.rank_max([3.0, 1.5]) == [3.0, 1.5]


def test_replicas_have_their_own_inputs():
    sys.path.insert(0, str(ROOT))
    import bench
    cfg = bench.workload_config("small")
    (p0, q0), (p1, q1) = bench.make_inputs(cfg, 0), bench.make_inputs(cfg, 1)
    assert p0.pos.shape == p1.pos.shape and q0.pos.shape == q1.pos.shape
    assert not np.array_equal(p0.pos, p1.pos) and not np.array_equal(q0.pos, q1.pos)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "small"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
