"""Randomized parity sweeps.  Query path: seeded random configurations (photon count,
caustic share, duplicated positions, query count and clustering, k, R,
filter, leaf size, k-buffer layout, queries per warp, rounds per chunk)
against the oracle, with the bars of test_gpu_parity (neighbour lists,
counts and r^2 bit-exact; radiance within 1e-5 of FP64).  Such a sweep found
a channel whose flux sat on the k-th neighbour; the case is pinned in
test_gpu_parity.test_channel_imbalanced_flux_small_k."""
import numpy as np
import pytest

from mnrt_b200 import gen
from tests.test_gpu_parity import check_against_oracle, format_errors, radiance_errors, run

pytestmark = pytest.mark.gpu


def draw(seed):
    rng = np.random.default_rng(seed)
    c = dict(n=int(rng.choice([1, 17, 500, 4000, 30000, 120000])), nq=int(rng.choice([1, 31, 1000, 5000])),
             k=int(rng.choice([1, 2, 7, 32, 64, 100, 128])), r=float(rng.choice([0.003, 0.02, 0.05, 0.2, 1.5])),
             filt=str(rng.choice(["box", "cone", "epanechnikov"])), leaf=int(rng.choice([1, 4, 8, 16, 24, 32])),
             layout=int(rng.choice([0, 1, 2, 2])), caustic=float(rng.choice([0.0, 0.2, 0.9])),
             dup=bool(rng.random() < 0.25), cluster=float(rng.choice([0.0, 0.5])),
             rounds=int(rng.choice([1, 8, 32, 100])), pseed=int(rng.integers(1 << 30)), qseed=int(rng.integers(1 << 30)))
    c["qpw"] = int(rng.choice([1, 2, 4, 8])) if c["layout"] == 1 else 1
    return c


@pytest.mark.parametrize("seed", range(24))
def test_random_configuration(cuda, oracle_mod, seed):
    c = draw(1000 + seed)
    ph = gen.photons(c["n"], seed=c["pseed"], caustic_frac=c["caustic"])
    if c["dup"] and c["n"] > 4:   # duplicated positions: ties broken by the caller index
        half = c["n"] // 2
        ph.pos[half:, :3] = ph.pos[: c["n"] - half, :3]
    q = gen.queries(c["nq"], seed=c["qseed"], cluster_frac=c["cluster"])
    res = run(ph, q, cuda, c["k"], c["r"], c["filt"], leaf=c["leaf"],
              tuning=dict(kbuf_layout=c["layout"], queries_per_warp=c["qpw"], rounds_per_chunk=c["rounds"]))
    assert res["info"].device_errors == 0, c
    check_against_oracle(oracle_mod, ph, q, res, c["k"], c["r"], c["filt"])


@pytest.mark.parametrize("seed", range(8))
def test_random_adjoint(cuda, oracle_mod, seed):
    """The adjoint against the oracle's FP64 host gradient on random
    configurations (bars of test_gpu_backward)."""
    from tests.test_gpu_backward import RTOL_HOST, engine_grads, rel_err, setup_problem
    rng = np.random.default_rng(2000 + seed)
    n, nq = int(rng.choice([500, 8000, 40000])), int(rng.choice([300, 5000]))
    k, r = int(rng.choice([1, 3, 16, 64, 128])), float(rng.choice([0.01, 0.05, 0.3]))
    filt = str(rng.choice(["box", "cone", "epanechnikov"]))
    mf = int(rng.choice([0, 8]))
    ph, q, t, idx, cnt = setup_problem(oracle_mod, n, nq, k, r, filt, seed=int(rng.integers(1 << 20)), min_found=mf)
    res = engine_grads(cuda, ph, q, t, k, r, filt, min_found=mf)
    assert np.array_equal(res["nbr"], idx) and np.array_equal(res["count"], cnt)
    hp, hx = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, res["g"][:, :3].astype(np.float64),
                                      filt, 1.0, mf)
    assert rel_err(res["gpow"][:, :3], hp, 1e-6).max() <= RTOL_HOST
    assert rel_err(res["gpos"][:, :3], hx, 1e-6).max() <= RTOL_HOST


def empty_set():
    return gen.PhotonSet(np.zeros((0, 4), np.float32), np.zeros((0, 4), np.float32), np.zeros((0, 3), np.float32),
                         "packed")


@pytest.mark.parametrize("seed", range(8))
def test_random_batch(cuda, seed):
    """A batch of 1-23 random maps (empty maps, maps without queries, mixed k,
    R, filters and min_found; random leaf size, rounds per chunk and tree
    width) against one pm_build + pm_query per map: radiance and neighbour
    rows bit-identical."""
    import torch
    from mnrt_b200.batch import PhotonMapBatch
    from mnrt_b200.photon_map import PhotonMap
    from tests.test_gpu_batch import to_dev
    rng = np.random.default_rng(3000 + seed)
    phs, qs, descs = [], [], []
    for _ in range(int(rng.integers(1, 24))):
        n, nq = int(rng.choice([0, 1, 5, 33, 700, 9000, 40000])), int(rng.choice([0, 1, 50, 900]))
        phs.append(gen.photons(n, seed=int(rng.integers(1 << 30)), caustic_frac=float(rng.choice([0, 0.2, 0.9])))
                   if n else empty_set())
        qs.append(gen.queries(nq, seed=int(rng.integers(1 << 30))))
        descs.append(dict(k=int(rng.choice([1, 4, 16, 64, 128])), r_max=float(rng.choice([0.01, 0.05, 0.3])),
                          filter=str(rng.choice(["box", "cone", "epanechnikov"])), min_found=int(rng.choice([0, 8]))))
    poff = np.concatenate([[0], np.cumsum([p.n for p in phs])]).astype(np.uint32)
    qoff = np.concatenate([[0], np.cumsum([q.n for q in qs])]).astype(np.uint32)
    cat = lambda xs: np.concatenate(xs).astype(np.float32)
    b = PhotonMapBatch()
    b.set_tuning(leaf_size=int(rng.choice([4, 16, 32, 48, 64])), warps_per_block=4, rounds_per_chunk=int(rng.choice([1, 8, 32])),
                 wide=bool(rng.random() < 0.7))
    b.build(to_dev(cat([p.pos for p in phs]), cuda), to_dev(cat([p.pow for p in phs]), cuda), poff)
    if qoff[-1]:
        out = b.query(descs, to_dev(cat([q.pos for q in qs]), cuda), to_dev(cat([q.nrm for q in qs]), cuda), qoff,
                      want_nbr=True)
        torch.cuda.synchronize()
        rad, nbr = out["rad"].cpu().numpy(), out["nbr"].cpu().numpy()
        noff = 0
        for i, (ph, q, d) in enumerate(zip(phs, qs, descs)):
            if not q.n:
                continue
            pm = PhotonMap(max(ph.n, 1), global_q_radius_max=d["r_max"])
            pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
            o = pm.query(to_dev(q.pos, cuda), to_dev(q.nrm, cuda), want_nbr=True, **d)
            torch.cuda.synchronize()
            a = int(qoff[i])
            assert np.array_equal(rad[a:a + q.n], o["rad"].cpu().numpy()), (i, d)
            assert np.array_equal(nbr[noff:noff + q.n * d["k"]].reshape(q.n, d["k"]), o["nbr"].cpu().numpy()), (i, d)
            noff += q.n * d["k"]
            pm.close()
    assert b.info().device_errors == 0
    b.close()


@pytest.mark.parametrize("seed", range(8))
def test_random_compat(cuda, oracle_mod, seed):
    """PM_MODE_ZHOU_COMPAT on random configurations against the oracle's
    restatement of the radius pipeline (bars of test_gpu_compat)."""
    import torch
    from mnrt_b200 import _lib as L
    from mnrt_b200.photon_map import PhotonMap
    from tests.test_gpu_batch import to_dev
    rng = np.random.default_rng(4000 + seed)
    n, nq = int(rng.choice([300, 3000, 30000, 100000])), int(rng.choice([10, 500, 3000]))
    k, r = int(rng.choice([1, 8, 20, 50, 100])), float(rng.choice([0.01, 0.05, 0.2]))
    iters, filt = int(rng.choice([0, 1, 2, 3])), str(rng.choice(["box", "cone", "epanechnikov"]))
    ph = gen.photons(n, seed=int(rng.integers(1 << 30)), caustic_frac=0.2)
    q = gen.queries(nq, seed=int(rng.integers(1 << 30)))
    pm = PhotonMap(n, global_q_radius_max=r, knn_target_count=k)
    pm.set_tuning(leaf_size=int(rng.choice([4, 16, 32, 48, 64])))
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    out = pm.query(to_dev(q.pos, cuda), to_dev(q.nrm, cuda), mode=L.PM_MODE_ZHOU_COMPAT, refine_iters=iters,
                   filter=filt, min_found=8, k=k)
    radii = pm.compute_query_radii(to_dev(q.pos, cuda), refine_iters=iters, k=k)
    torch.cuda.synchronize()
    nodes, tpos, tpow = pm.export_tree()
    o_radius, o_count, o_r2, o_rad = oracle_mod.compat(nodes, tpos, tpow, q.pos, q.nrm, k, r, iters, filt, 1.0, 8)
    assert np.array_equal(radii.cpu().numpy(), o_radius)
    assert np.array_equal(out["count"].cpu().numpy().view(np.uint32), o_count)
    assert np.array_equal(out["r2"].cpu().numpy(), o_r2)
    e = radiance_errors(out["rad"].cpu().numpy()[:, :3], o_rad)
    assert e["max"] <= 1e-5, format_errors(e)
    assert pm.info().device_errors == 0
    pm.close()


@pytest.mark.parametrize("nq", [1, 97, 20000])
def test_chunk_schedules_give_identical_bits(cuda, nq):
    """Warps take query chunks by guided self-scheduling (long chunks first,
    rounds_per_chunk rounds last).  The schedule only decides which warp
    answers which query and which radius bound a query starts from, so every
    layout, warp count and chunk size must give the same bits."""
    ph = gen.photons(50000, seed=3100, caustic_frac=0.2)
    q = gen.queries(nq, seed=3101, cluster_frac=0.5)
    ref = None
    for layout, qpw, wpb, rounds in [(2, 1, 4, 8), (2, 1, 1, 1), (2, 1, 8, 4096), (1, 4, 2, 3), (1, 1, 4, 4096),
                                     (0, 1, 4, 1), (0, 1, 2, 4096)]:
        res = run(ph, q, cuda, 48, 0.08, "cone", leaf=24,
                  tuning=dict(kbuf_layout=layout, queries_per_warp=qpw, warps_per_block=wpb, rounds_per_chunk=rounds))
        assert res["info"].device_errors == 0
        got = {key: res[key] for key in ("rad", "r2", "count", "nbr")}
        if ref is None:
            ref = got
            continue
        for key in ref:
            assert np.array_equal(got[key], ref[key]), (layout, qpw, wpb, rounds, key)
