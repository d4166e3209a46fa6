"""Batched maps (pm_batch_*) against per-map pm_build + pm_query: neighbour
rows, counts, r^2 and radiance bit-identical for every map, including empty
maps, maps smaller than a leaf, maps without queries, mixed k and filters;
CUDA-graph replay identical to eager execution."""
import numpy as np
import pytest
import torch

from mnrt_b200 import gen
from mnrt_b200.batch import PhotonMapBatch, make_desc
from mnrt_b200.photon_map import PhotonMap

pytestmark = pytest.mark.gpu


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


SIZES = [(0, 50), (1, 40), (5, 30), (32, 20), (33, 0), (1000, 300), (50000, 4000), (20000, 2500), (3000, 1000)]
DESCS = [dict(k=8, r_max=0.2, filter="box"), dict(k=1, r_max=0.5, filter="cone"), dict(k=16, r_max=0.3, filter="box"),
         dict(k=32, r_max=0.1, filter="epanechnikov"), dict(k=16, r_max=0.05, filter="box"),
         dict(k=64, r_max=0.05, filter="cone", min_found=8), dict(k=128, r_max=0.05, filter="epanechnikov"),
         dict(k=100, r_max=0.05, filter="cone"), dict(k=48, r_max=0.08, filter="box")]


def make_batch():
    phs, qs = [], []
    for i, (n, nq) in enumerate(SIZES):
        ph = gen.photons(n, seed=300 + i, caustic_frac=0.2) if n else gen.PhotonSet(
            np.zeros((0, 4), np.float32), np.zeros((0, 4), np.float32), np.zeros((0, 3), np.float32), "packed")
        if n > 200:
            ph.pos[100:150, :3] = ph.pos[7, :3]       # coincident photons: ties broken by index
        q = gen.queries(nq, seed=400 + i)
        phs.append(ph)
        qs.append(q)
    poff = np.concatenate([[0], np.cumsum([p.n for p in phs])]).astype(np.uint32)
    qoff = np.concatenate([[0], np.cumsum([q.n for q in qs])]).astype(np.uint32)
    pos = np.concatenate([p.pos for p in phs]).astype(np.float32)
    pw = np.concatenate([p.pow for p in phs]).astype(np.float32)
    qp = np.concatenate([q.pos for q in qs]).astype(np.float32)
    qn = np.concatenate([q.nrm for q in qs]).astype(np.float32)
    return phs, qs, poff, qoff, pos, pw, qp, qn


def per_map_reference(dev, phs, qs):
    res = []
    for ph, q, d in zip(phs, qs, DESCS):
        pm = PhotonMap(max(ph.n, 1), global_q_radius_max=d["r_max"])
        pm.build(to_dev(ph.pos, dev), to_dev(ph.pow, dev))
        if q.n:
            o = pm.query(to_dev(q.pos, dev), to_dev(q.nrm, dev), want_nbr=True, **d)
            torch.cuda.synchronize()
            res.append({k: v.cpu().numpy() for k, v in o.items()})
        else:
            res.append(None)
        pm.close()
    return res


def compare(out, ref, qoff):
    rad, r2, cnt = out["rad"].cpu().numpy(), out["r2"].cpu().numpy(), out["count"].cpu().numpy()
    nbr = out["nbr"].cpu().numpy()
    noff = 0
    for i, (r, d) in enumerate(zip(ref, DESCS)):
        a, b = int(qoff[i]), int(qoff[i + 1])
        if r is None:
            assert a == b
            continue
        assert np.array_equal(rad[a:b], r["rad"]), f"map {i} radiance"
        assert np.array_equal(r2[a:b], r["r2"]), f"map {i} r2"
        assert np.array_equal(cnt[a:b], r["count"]), f"map {i} count"
        rows = nbr[noff:noff + (b - a) * d["k"]].reshape(b - a, d["k"])
        assert np.array_equal(rows, r["nbr"]), f"map {i} neighbours"
        noff += (b - a) * d["k"]


@pytest.mark.parametrize("wide", [False, True])
def test_batch_matches_per_map(cuda, wide):
    phs, qs, poff, qoff, pos, pw, qp, qn = make_batch()
    ref = per_map_reference(cuda, phs, qs)
    b = PhotonMapBatch()
    b.set_tuning(leaf_size=16, warps_per_block=4, rounds_per_chunk=5, wide=wide)
    b.build(to_dev(pos, cuda), to_dev(pw, cuda), poff)
    out = b.query(DESCS, to_dev(qp, cuda), to_dev(qn, cuda), qoff, want_nbr=True)
    torch.cuda.synchronize()
    compare(out, ref, qoff)
    assert b.info().device_errors == 0


def test_batch_graph_replay(cuda):
    phs, qs, poff, qoff, pos, pw, qp, qn = make_batch()
    d_pos, d_pw, d_qp, d_qn = (to_dev(x, cuda) for x in (pos, pw, qp, qn))
    b = PhotonMapBatch()
    out = b.outputs(DESCS, qoff, cuda, want_nbr=True)
    b.capture(d_pos, d_pw, poff, DESCS, d_qp, d_qn, qoff, out)
    for _ in range(2):
        for v in out.values():
            v.zero_()
        b.launch()
    torch.cuda.synchronize()
    compare(out, per_map_reference(cuda, phs, qs), qoff)
    # new photon values in the same buffers are picked up by the next replay
    pw2 = pw.copy()
    pw2[:, :3] *= 2.0
    d_pw.copy_(to_dev(pw2, cuda))
    b.launch()
    torch.cuda.synchronize()
    for ph, a, z in zip(phs, poff[:-1], poff[1:]):
        ph.pow = pw2[a:z]
    compare(out, per_map_reference(cuda, phs, qs), qoff)
