"""GPU adjoint (pm_query_backward) through the C ABI.

Bars:
  * against the oracle's FP64 host gradient on the same neighbour sets:
    relative error <= 1e-5 (floor 1e-6 of the largest magnitude); the engine
    evaluates in FP64 and rounds the result to FP32;
  * against FP64 central finite differences of the loss (h = 1e-4 and h/2,
    Richardson-combined): relative error <= 1e-3 (floor 1e-3 of the largest
    magnitude), samples whose neighbour set changes within +-h excluded and
    counted;
  * bitwise: two runs, reuse vs recompute of the kNN, and any chunking give
    the same bits.
"""
import numpy as np
import pytest
import torch

from mnrt_b200 import gen
from mnrt_b200.photon_map import PhotonMap
from tests.fd import LossFD

pytestmark = pytest.mark.gpu

RTOL_HOST = 1e-5
RTOL_FD = 1e-3


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def rel_err(a, b, floor_frac):
    floor = floor_frac * max(np.abs(b).max(), 1e-300)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def setup_problem(oracle_mod, n, nq, k, r, filt, seed, min_found=0):
    ph = gen.photons(n, seed=seed, caustic_frac=0.2)
    q = gen.queries(nq, seed=seed + 1)
    rng = np.random.default_rng(seed + 2)
    tpow = ph.pow.copy()
    tpow[:, :3] *= rng.uniform(0.5, 1.5, size=(n, 3)).astype(np.float32)
    idx, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
    t = oracle_mod.radiance_fp64(ph.pos, tpow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, min_found)
    return ph, q, t, idx, cnt


def engine_grads(dev, ph, q, t, k, r, filt, min_found=0, reuse=True, chunk=0):
    pm = PhotonMap(ph.n, global_q_radius_max=r, knn_target_count=k)
    pm.build(to_dev(ph.pos, dev), to_dev(ph.pow, dev))
    qp, qn = to_dev(q.pos, dev), to_dev(q.nrm, dev)
    kw = dict(k=k, r_max=r, filter=filt, min_found=min_found)
    out = pm.query(qp, qn, want_nbr=True, **kw)
    g = torch.zeros((q.n, 4), dtype=torch.float32, device=dev)
    g[:, :3] = 2.0 * (out["rad"][:, :3].double() - torch.from_numpy(t).to(dev)).float()
    if chunk:
        pm.set_backward_chunk(chunk)
    gp, gx = pm.query_backward(qp, qn, g, nbr=out["nbr"] if reuse else None, count=out["count"] if reuse else None,
                               **kw)
    torch.cuda.synchronize()
    res = dict(gpow=gp.cpu().numpy(), gpos=gx.cpu().numpy(), g=g.cpu().numpy(),
               nbr=out["nbr"].cpu().numpy().view(np.uint32), count=out["count"].cpu().numpy().view(np.uint32))
    assert pm.info().device_errors == 0
    pm.close()
    return res


@pytest.mark.parametrize("filt", ["epanechnikov", "cone", "box"])
def test_backward_matches_host_gradient_and_fd(cuda, oracle_mod, filt):
    k, r = 32, 0.05
    ph, q, t, idx, cnt = setup_problem(oracle_mod, 40000, 20000, k, r, filt, seed=70)
    res = engine_grads(cuda, ph, q, t, k, r, filt)
    assert np.array_equal(res["nbr"], idx) and np.array_equal(res["count"], cnt)
    hp, hx = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, res["g"][:, :3].astype(np.float64),
                                      filt)
    assert rel_err(res["gpow"][:, :3], hp, 1e-6).max() <= RTOL_HOST
    assert rel_err(res["gpos"][:, :3], hx, 1e-6).max() <= RTOL_HOST
    assert (res["gpow"][:, 3] == 0).all() and (res["gpos"][:, 3] == 0).all()
    # finite differences of the loss the gradient belongs to: L = sum (E - T)^2,
    # evaluated by the oracle in FP64 (dL/dE = 2 (E64 - T))
    e64 = oracle_mod.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt)
    hp64, hx64 = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, 2.0 * (e64 - t), filt)
    fd = LossFD(oracle_mod, ph.pos, ph.pow, q.pos, q.nrm, t, k, r, filt)
    rng = np.random.default_rng(9)
    kth = np.unique(idx[cnt == k, k - 1])
    sample = np.concatenate([rng.choice(ph.n, 48, replace=False), rng.choice(kth, 16, replace=False)])
    f = fd.position(sample)
    ok = ~f.excluded
    print(f"{filt}: {f.num_excluded} of {ok.size} position samples excluded (set change within +-h)")
    assert ok.sum() >= 0.7 * ok.size
    # the engine's gradient of its own FP32 estimate vs the FP64 loss: compare
    # the host FP64 gradient (same formula) to FD, and the engine to the host
    assert rel_err(hx64[sample][ok], f.fd[ok], RTOL_FD).max() <= RTOL_FD
    assert rel_err(hp64[sample[:16]], fd.power(sample[:16]), RTOL_FD).max() <= RTOL_FD


def test_backward_bitwise_reproducible(cuda, oracle_mod):
    k, r = 64, 0.05
    ph, q, t, _idx, _cnt = setup_problem(oracle_mod, 60000, 30000, k, r, "epanechnikov", seed=80)
    a = engine_grads(cuda, ph, q, t, k, r, "epanechnikov")
    b = engine_grads(cuda, ph, q, t, k, r, "epanechnikov")
    c = engine_grads(cuda, ph, q, t, k, r, "epanechnikov", reuse=False)
    d = engine_grads(cuda, ph, q, t, k, r, "epanechnikov", chunk=7001)
    e = engine_grads(cuda, ph, q, t, k, r, "epanechnikov", reuse=False, chunk=4096)
    for x in (b, c, d, e):
        assert np.array_equal(a["gpow"], x["gpow"])
        assert np.array_equal(a["gpos"], x["gpos"])


def test_backward_min_found_and_edges(cuda, oracle_mod):
    k, r = 16, 0.02
    ph, q, t, idx, cnt = setup_problem(oracle_mod, 3000, 2000, k, r, "box", seed=90, min_found=8)
    q.pos[:5, :3] += 10.0            # far queries: no neighbours
    idx, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
    res = engine_grads(cuda, ph, q, t, k, r, "box", min_found=8)
    hp, hx = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, res["g"][:, :3].astype(np.float64),
                                      "box", 1.0, 8)
    assert rel_err(res["gpow"][:, :3], hp, 1e-6).max() <= RTOL_HOST
    assert rel_err(res["gpos"][:, :3], hx, 1e-6).max() <= RTOL_HOST


@pytest.mark.parametrize("n", [2000, 10000])
def test_backward_long_segments(cuda, oracle_mod, n):
    """Photons in hundreds of neighbour lists (few photons, many queries, a
    wide radius): the adjoint sorts each photon's segment of pairs with a
    256-slot register network when it holds 129-256 values and in place
    through L2 above that; both must give the host gradient, and chunking
    must not change a bit."""
    k, r = 64, 0.5
    ph, q, t, idx, cnt = setup_problem(oracle_mod, n, 30000, k, r, "epanechnikov", seed=97)
    seg = np.bincount(idx[idx != np.uint32(0xFFFFFFFF)].astype(np.int64), minlength=n)
    assert (seg > 256).any()
    if n == 10000:
        assert ((seg > 128) & (seg <= 256)).any()
    res = engine_grads(cuda, ph, q, t, k, r, "epanechnikov")
    assert np.array_equal(res["nbr"], idx) and np.array_equal(res["count"], cnt)
    hp, hx = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, res["g"][:, :3].astype(np.float64),
                                      "epanechnikov")
    assert rel_err(res["gpow"][:, :3], hp, 1e-6).max() <= RTOL_HOST
    assert rel_err(res["gpos"][:, :3], hx, 1e-6).max() <= RTOL_HOST
    chunked = engine_grads(cuda, ph, q, t, k, r, "epanechnikov", chunk=7001)
    assert np.array_equal(res["gpow"], chunked["gpow"]) and np.array_equal(res["gpos"], chunked["gpos"])


def test_backward_skewed_segments(cuda, oracle_mod):
    """Twelve photons near every query, the rest far away: a mean of 12
    pairs per photon (the placement path) with twelve segments of 20,000
    pairs, which a block sorts in place through L2."""
    k, r = 8, 2.0
    ph = gen.photons(20000, seed=99, caustic_frac=0.2)
    ph.pos[12:, :3] += 50.0
    q = gen.queries(30000, seed=100)
    idx, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
    seg = np.bincount(idx[idx != np.uint32(0xFFFFFFFF)].astype(np.int64), minlength=ph.n)
    assert (seg > 8192).sum() == 12 and seg.sum() <= 256 * ph.n
    t = oracle_mod.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, "cone") * 0.9
    res = engine_grads(cuda, ph, q, t, k, r, "cone")
    assert np.array_equal(res["nbr"], idx) and np.array_equal(res["count"], cnt)
    hp, hx = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, res["g"][:, :3].astype(np.float64),
                                      "cone")
    assert rel_err(res["gpow"][:, :3], hp, 1e-6).max() <= RTOL_HOST
    assert rel_err(res["gpos"][:, :3], hx, 1e-6).max() <= RTOL_HOST
    chunked = engine_grads(cuda, ph, q, t, k, r, "cone", chunk=9999)
    assert np.array_equal(res["gpow"], chunked["gpow"]) and np.array_equal(res["gpos"], chunked["gpos"])


def test_autograd_wrapper(cuda, oracle_mod):
    from mnrt_b200.autograd import RadianceEstimate
    k, r = 16, 0.06
    ph = gen.photons(8000, seed=95, caustic_frac=0.2)
    q = gen.queries(3000, seed=96)
    pos = to_dev(ph.pos, cuda).requires_grad_(True)
    pw = to_dev(ph.pow, cuda).requires_grad_(True)
    rad = RadianceEstimate.apply(pos, pw, to_dev(q.pos, cuda), to_dev(q.nrm, cuda), k, r, "epanechnikov")
    loss = (rad.double() ** 2).sum()
    loss.backward()
    idx, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
    g = 2.0 * rad.detach().double().cpu().numpy()
    hp, hx = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, g.astype(np.float32).astype(np.float64),
                                      "epanechnikov")
    assert rel_err(pw.grad.cpu().numpy()[:, :3], hp, 1e-6).max() <= RTOL_HOST
    assert rel_err(pos.grad.cpu().numpy()[:, :3], hx, 1e-6).max() <= RTOL_HOST
