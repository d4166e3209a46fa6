"""The N-GPU path of bench.py on CPU: two gloo ranks.  The plain workload
divides one map's queries into contiguous ranges (every rank builds the same
map, no exchange on the data path); --division replicas gives every rank its
own seeded photons and queries.  The only collective of the timed region is
the max over ranks of its device time, and rank 0 alone prints."""
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


def test_replica_division_gives_ranks_their_own_inputs():
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


# ---------------------------------------------------------------- sharding --

def test_lpt_assign_covers_every_map_once_and_is_balanced():
    import itertools
    from mnrt_b200.shard import lpt_assign, map_costs
    rng = np.random.default_rng(5)
    for trial in range(40):
        m, world = int(rng.integers(0, 9)), int(rng.integers(1, 5))
        costs = map_costs(rng.integers(0, 2_000_000, m), rng.integers(0, 1_000_000, m))
        parts = lpt_assign(costs, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(m))
        assert all(p == sorted(p) for p in parts)
        if m == 0:
            continue
        span = max(costs[p].sum() if p else 0.0 for p in parts)
        best = min(max(sum(costs[i] for i in range(m) if a[i] == r) for r in range(world))
                   for a in itertools.product(range(world), repeat=m)) if world ** m <= 50_000 else None
        if best is not None:
            assert span <= (4 / 3 - 1 / (3 * world)) * best + 1e-6
    assert lpt_assign([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]   # ties: lower index first, to the lower rank
    with pytest.raises(ValueError):
        lpt_assign([1.0, -1.0], 2)


def test_query_range_partitions_contiguously():
    from mnrt_b200.shard import query_range
    for nq in (0, 1, 7, 1000, 2_073_600):
        for world in (1, 2, 3, 8):
            r = [query_range(nq, i, world) for i in range(world)]
            assert r[0][0] == 0 and r[-1][1] == nq
            assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1


def _forward_worker(rank, world, port, q):
    """Each rank: the oracle's exact kNN and FP64 estimate over its own query
    range of one map, then an all-gather of the per-range answers."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    from mnrt_b200.shard import query_range
    from oracle import oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = bench.workload_config("small")
        ph, qs = bench.make_inputs(cfg, 0)          # every rank: the same map and query set
        a, b = query_range(qs.n, rank, world)
        idx, _d2, cnt, r2 = oracle.KdTree(ph.pos).knn(qs.pos[a:b], cfg["k"], cfg["r_max"])
        rad = oracle.radiance_fp64(ph.pos, ph.pow, qs.pos[a:b], qs.nrm[a:b], idx, cnt, cfg["k"], cfg["r_max"],
                                   cfg["filter"])
        mine = [torch.from_numpy(idx.view(np.int32).copy()), torch.from_numpy(cnt.view(np.int32).copy()),
                torch.from_numpy(r2.copy()), torch.from_numpy(rad.copy())]
        # ranges differ by at most one query: pad to the largest, gather, trim
        size = max(query_range(qs.n, i, world)[1] - query_range(qs.n, i, world)[0] for i in range(world))
        parts = []
        for t in mine:
            pad = torch.zeros((size,) + tuple(t.shape[1:]), dtype=t.dtype)
            pad[:t.shape[0]] = t
            got = [torch.empty_like(pad) for _ in range(world)]
            dist.all_gather(got, pad)
            parts.append(torch.cat([g[:query_range(qs.n, i, world)[1] - query_range(qs.n, i, world)[0]]
                                    for i, g in enumerate(got)]).numpy())
        q.put((rank, parts))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_query_divided_forward_assembles_the_undivided_answer():
    """One map, queries divided over two gloo ranks: the per-range answers,
    gathered in rank order, are the undivided answer bit for bit."""
    sys.path.insert(0, str(ROOT))
    import bench
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    world = 2
    procs = [ctx.Process(target=_forward_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfg = bench.workload_config("small")
    ph, qs = bench.make_inputs(cfg, 0)
    idx, _d2, cnt, r2 = oracle.KdTree(ph.pos).knn(qs.pos, cfg["k"], cfg["r_max"])
    rad = oracle.radiance_fp64(ph.pos, ph.pow, qs.pos, qs.nrm, idx, cnt, cfg["k"], cfg["r_max"], cfg["filter"])
    for rank in range(world):
        g_idx, g_cnt, g_r2, g_rad = out[rank]
        assert np.array_equal(g_idx.view(np.uint32), idx)
        assert np.array_equal(g_cnt.view(np.uint32), cnt)
        assert np.array_equal(g_r2.view(np.uint32), r2.view(np.uint32))
        assert np.array_equal(g_rad.view(np.uint64), rad.view(np.uint64))


def _adjoint_worker(rank, world, port, q):
    """Each rank: the FP64 host adjoint over its own query range, rounded to
    float32 like the engine's output, then the gradient all-reduce."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from mnrt_b200 import gen
    from mnrt_b200.shard import allreduce_gradients, allreduce_scalars, query_range
    from oracle import oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n, nq, k, r = 3000, 900, 16, 0.1
        ph, qs = gen.photons(n, seed=77, caustic_frac=0.2), gen.queries(nq, seed=78)
        a, b = query_range(nq, rank, world)
        idx, _d2, cnt, _r2 = oracle.KdTree(ph.pos).knn(qs.pos[a:b], k, r)
        g = np.random.default_rng(79).standard_normal((nq, 3))[a:b]
        hp, hx = oracle.backward_fp64(ph.pos, ph.pow, qs.pos[a:b], qs.nrm[a:b], idx, cnt, k, r, g, "cone", 1.0, 0)
        gp = torch.zeros((n, 4), dtype=torch.float32)
        gx = torch.zeros((n, 4), dtype=torch.float32)
        gp[:, :3] = torch.from_numpy(hp).float()
        gx[:, :3] = torch.from_numpy(hx).float()
        part = max(float(np.abs(hp).max()), 0.0), max(float(np.abs(hx).max()), 0.0)
        allreduce_gradients(gp, None, gx)
        tot = allreduce_scalars([float(b - a), 1.0])
        q.put((rank, gp.numpy().copy(), gx.numpy().copy(), part, tot))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_query_divided_adjoint_all_reduce_matches_single_rank():
    """The one exchange step: per-rank partial gradients over a query range,
    summed by the all-reduce, against the FP64 adjoint over all queries."""
    from mnrt_b200 import gen
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    world = 2
    procs = [ctx.Process(target=_adjoint_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, gp, gx, part, tot = q.get(timeout=300)
        out[rank] = (gp, gx, part, tot)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n, nq, k, r = 3000, 900, 16, 0.1
    ph, qs = gen.photons(n, seed=77, caustic_frac=0.2), gen.queries(nq, seed=78)
    idx, _d2, cnt, _r2 = oracle.KdTree(ph.pos).knn(qs.pos, k, r)
    g = np.random.default_rng(79).standard_normal((nq, 3))
    hp, hx = oracle.backward_fp64(ph.pos, ph.pow, qs.pos, qs.nrm, idx, cnt, k, r, g, "cone", 1.0, 0)
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])   # every rank the same
    assert out[0][3] == [float(nq), float(world)]
    bp = world * 2.0 ** -24 * max(out[0][2][0], out[1][2][0]) + np.abs(hp) * 2.0 ** -24
    bx = world * 2.0 ** -24 * max(out[0][2][1], out[1][2][1]) + np.abs(hx) * 2.0 ** -24
    assert (np.abs(out[0][0][:, :3] - hp) <= bp).all()
    assert (np.abs(out[0][1][:, :3] - hx) <= bx).all()
    assert np.abs(hp).max() > 0 and np.abs(hx).max() > 0


def test_bench_reads_the_committed_profiles():
    """bench.py's roofline object takes the DRAM and L2 bytes per launch from
    the committed ncu summaries; both are present and plausible."""
    sys.path.insert(0, str(ROOT))
    import bench
    dram = bench.profiled_traffic("k_knn_group", "plain")
    l2 = bench.profiled_traffic("k_knn_group", "plain", "l2_bytes_per_launch")
    assert dram is not None and 1e8 < dram < 1e10
    assert l2 is not None and l2 > dram
    assert bench.profiled_traffic("k_knn_group", "no_such_workload") is None
    peak, kind = bench.measured_peaks()
    assert peak > 1000 and kind in ("measured", "fallback")
