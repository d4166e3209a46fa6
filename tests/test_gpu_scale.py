"""Oracle parity at the benchmark workloads' full sizes.

Each test runs one named workload through the C ABI with neighbour lists and
compares every query with the CPU oracle (multithreaded kd-tree kNN plus the
FP64 estimate over the oracle's own neighbour sets):

  plain         1,048,576 photons (80 % walls, 20 % caustic), 2,073,600 wall
                queries, k = 100, R = 0.05, cone filter -- device buffers
                (pm_query) and pinned host buffers (pm_build_query_host, the
                bench's end-to-end call, radiance only)
  final gather  4,194,304 photons, 8,388,608 queries (half in 64 clusters,
                random order), k = 64, R = 0.05, cone filter, queries
                Hilbert-sorted by the engine and taken as given
  batch         64 maps (photons log-uniform in [1e4, 2e6], queries in
                [1e3, 1e6], k from {16, 32, 64, 128}, seed 777), one batched
                build + query, every map against the oracle on its own
  diff          1,048,576 photons, 1,048,576 wall queries, k = 64,
                Epanechnikov filter (the forward of the adjoint workload)

Bars: neighbour lists, their order, counts and r^2 bit-exact; radiance
within 1e-5 relative of FP64 for every nonzero value (no floor), exactly 0
where FP64 gives 0.  Each test prints its error summary (run with -s to see
the per-workload table).
"""
import numpy as np
import pytest
import torch

from mnrt_b200 import gen
from mnrt_b200.batch import PhotonMapBatch
from mnrt_b200.photon_map import PhotonMap
from tests.test_gpu_parity import RTOL, check_against_oracle, format_errors, radiance_errors, to_dev

pytestmark = pytest.mark.gpu


def workload(name, pseed, qseed):
    c = gen.CONFIGS[name]
    ph = gen.photons(c["n"], seed=pseed, caustic_frac=c.get("caustic_frac", 0.2), power_mean=c.get("power_mean"))
    q = gen.queries(c["nq"], seed=qseed, cluster_frac=c.get("cluster_frac", 0.0))
    return c, ph, q


def engine_query(pm, q, dev, c, sorted_queries=True):
    out = pm.query(to_dev(q.pos, dev), to_dev(q.nrm, dev), want_nbr=True, k=c["k"], r_max=c["r_max"],
                   filter=c["filter"], sorted_queries=sorted_queries)
    torch.cuda.synchronize()
    res = {kk: v.cpu().numpy() for kk, v in out.items()}
    del out
    return res


def test_plain_workload_parity(cuda, oracle_mod):
    c, ph, q = workload("plain", 1000, 2000)
    pm = PhotonMap(c["n"], global_q_radius_max=c["r_max"], knn_target_count=c["k"])
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    res = engine_query(pm, q, cuda, c)
    assert pm.info().device_errors == 0
    knn = oracle_mod.KdTree(ph.pos, threads=0).knn(q.pos, c["k"], c["r_max"], threads=0)
    e = check_against_oracle(oracle_mod, ph, q, res, c["k"], c["r_max"], c["filter"], oracle_knn=knn)
    print(f"\nplain (1,048,576 x 2,073,600, k=100, cone), pm_query: {format_errors(e)}")
    # the end-to-end call the bench times: pinned host buffers in, host radiance out
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_rad = torch.empty((q.n, 4), dtype=torch.float32).pin_memory()
    pm.build_query_host(pin(ph.pos), pin(ph.pow), pin(q.pos), pin(q.nrm), out=h_rad, k=c["k"], r_max=c["r_max"],
                        filter=c["filter"])
    torch.cuda.synchronize()
    assert np.array_equal(h_rad.numpy().view(np.uint32), res["rad"].view(np.uint32)), "host path differs"
    pm.close()


@pytest.mark.parametrize("order", ["sorted", "as_given"])
def test_final_gather_workload_parity(cuda, oracle_mod, order):
    c, ph, q = workload("final_gather", 1000, 2000)
    pm = PhotonMap(c["n"], global_q_radius_max=c["r_max"], knn_target_count=c["k"])
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    res = engine_query(pm, q, cuda, c, sorted_queries=order == "sorted")
    assert pm.info().device_errors == 0
    pm.close()
    knn = oracle_mod.KdTree(ph.pos, threads=0).knn(q.pos, c["k"], c["r_max"], threads=0)
    e = check_against_oracle(oracle_mod, ph, q, res, c["k"], c["r_max"], c["filter"], oracle_knn=knn)
    print(f"\nfinal gather (4,194,304 x 8,388,608, k=64, cone, {order}): {format_errors(e)}")


def test_batch_workload_parity(cuda, oracle_mod):
    spec = gen.batch_spec(64, seed=777)
    phs = [gen.photons(n, seed=s, caustic_frac=0.2) for n, s in zip(spec.n, spec.seeds)]
    qs = [gen.queries(nq, seed=s + 500) for nq, s in zip(spec.nq, spec.seeds)]
    descs = [dict(k=k, r_max=0.05, filter="cone") for k in spec.k]
    poff = np.concatenate([[0], np.cumsum(spec.n)]).astype(np.uint32)
    qoff = np.concatenate([[0], np.cumsum(spec.nq)]).astype(np.uint32)
    cat = lambda xs: to_dev(np.concatenate(xs), cuda)
    b = PhotonMapBatch()
    b.build(cat([p.pos for p in phs]), cat([p.pow for p in phs]), poff)
    out = b.query(descs, cat([q.pos for q in qs]), cat([q.nrm for q in qs]), qoff, want_nbr=True)
    torch.cuda.synchronize()
    assert b.info().device_errors == 0
    rad, r2, cnt, nbr = (out[key].cpu().numpy() for key in ("rad", "r2", "count", "nbr"))
    b.close()
    noff, worst, stats = 0, 0.0, []
    for i, (ph, q, d) in enumerate(zip(phs, qs, descs)):
        a, z, k = int(qoff[i]), int(qoff[i + 1]), d["k"]
        rows = nbr[noff:noff + (z - a) * k].reshape(z - a, k)
        noff += (z - a) * k
        res = {"rad": rad[a:z], "r2": r2[a:z], "count": cnt[a:z], "nbr": rows}   # rows hold per-map indices
        e = check_against_oracle(oracle_mod, ph, q, res, k, 0.05, "cone", threads=0)
        worst = max(worst, e["max"])
        stats.append(e)
    tot = sum(s["values"] for s in stats)
    mean = sum(s["mean"] * s["values"] for s in stats) / tot
    print(f"\nbatch (64 maps, {int(poff[-1]):,} photons, {int(qoff[-1]):,} queries, k in {{16,32,64,128}}, cone): "
          f"max rel err {worst:.2e}, mean {mean:.2e} over {tot:,} values "
          f"({sum(s['zero'] for s in stats):,} exact zeros; "
          f"{sum(s['below_floor'] for s in stats):,} below 1e-6 of their map's mean)")
    assert worst <= RTOL


def test_diff_workload_forward_parity(cuda, oracle_mod):
    c, ph, q = workload("diff", 4000, 4001)
    pm = PhotonMap(c["n"], global_q_radius_max=c["r_max"], knn_target_count=c["k"])
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    res = engine_query(pm, q, cuda, c)
    assert pm.info().device_errors == 0
    pm.close()
    e = check_against_oracle(oracle_mod, ph, q, res, c["k"], c["r_max"], c["filter"], threads=0)
    print(f"\ndiff forward (1,048,576 x 1,048,576, k=64, Epanechnikov): {format_errors(e)}")
