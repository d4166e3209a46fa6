"""The multi-GPU divisions of the path, run shard after shard on one GPU (the
shards never wait on one another, so running them in turn is exact):
batch maps divided by LPT give every map the bits of the undivided batch;
a map's queries divided into ranges give the bits of the undivided query;
the adjoint's per-range partial gradients, summed in float64 as the
all-reduce sums them, match the undivided adjoint to the partials' own
float32 rounding."""
import numpy as np
import pytest
import torch

from mnrt_b200 import gen
from mnrt_b200.batch import PhotonMapBatch
from mnrt_b200.photon_map import PhotonMap
from mnrt_b200.shard import lpt_assign, map_costs, query_range
from tests.test_gpu_batch import DESCS, make_batch, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3, 8])
def test_lpt_shards_match_undivided_batch(cuda, world):
    phs, qs, poff, qoff, pos, pw, qp, qn = make_batch()
    full = PhotonMapBatch()
    full.build(to_dev(pos, cuda), to_dev(pw, cuda), poff)
    ref = full.query(DESCS, to_dev(qp, cuda), to_dev(qn, cuda), qoff, want_nbr=True)
    torch.cuda.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref.items()}
    nbr_off = np.concatenate([[0], np.cumsum([q.n * d["k"] for q, d in zip(qs, DESCS)])])
    parts = lpt_assign(map_costs([p.n for p in phs], [q.n for q in qs]), world)
    assert sorted(i for p in parts for i in p) == list(range(len(phs)))
    for mine in parts:
        if not mine:
            continue
        sp = np.concatenate([[0], np.cumsum([phs[i].n for i in mine])]).astype(np.uint32)
        sq = np.concatenate([[0], np.cumsum([qs[i].n for i in mine])]).astype(np.uint32)
        cat = lambda xs: to_dev(np.concatenate(xs).astype(np.float32), cuda)
        b = PhotonMapBatch()
        b.build(cat([phs[i].pos for i in mine]), cat([phs[i].pow for i in mine]), sp)
        if sq[-1] == 0:
            b.close()
            continue
        out = b.query([DESCS[i] for i in mine], cat([qs[i].pos for i in mine]), cat([qs[i].nrm for i in mine]), sq,
                      want_nbr=True)
        torch.cuda.synchronize()
        got = {k: v.cpu().numpy() for k, v in out.items()}
        no = 0
        for j, i in enumerate(mine):
            a, z, fa = int(sq[j]), int(sq[j + 1]), int(qoff[i])
            assert np.array_equal(got["rad"][a:z], ref["rad"][fa:fa + z - a]), i
            assert np.array_equal(got["count"][a:z], ref["count"][fa:fa + z - a]), i
            m = (z - a) * DESCS[i]["k"]
            assert np.array_equal(got["nbr"][no:no + m], ref["nbr"][nbr_off[i]:nbr_off[i] + m]), i
            no += m
        assert b.info().device_errors == 0
        b.close()
    full.close()


@pytest.mark.parametrize("world", [2, 5])
def test_query_ranges_match_undivided_query_and_adjoint(cuda, world):
    n, nq, k, r = 60000, 20000, 64, 0.05
    ph, q = gen.photons(n, seed=91, caustic_frac=0.2), gen.queries(nq, seed=92)
    pm = PhotonMap(n, global_q_radius_max=r, knn_target_count=k)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    kw = dict(k=k, r_max=r, filter="cone")
    qp, qn = to_dev(q.pos, cuda), to_dev(q.nrm, cuda)
    full = pm.query(qp, qn, want_nbr=True, **kw)
    g = torch.zeros((nq, 4), dtype=torch.float32, device=cuda)
    g[:, :3] = torch.from_numpy(np.random.default_rng(93).standard_normal((nq, 3)).astype(np.float32)).to(cuda)
    gp_full, gx_full = pm.query_backward(qp, qn, g, nbr=full["nbr"], count=full["count"], **kw)
    torch.cuda.synchronize()
    sum_p = np.zeros((n, 3))
    sum_x = np.zeros((n, 3))
    max_p = max_x = 0.0
    for rank in range(world):
        a, b = query_range(nq, rank, world)
        o = pm.query(qp[a:b], qn[a:b], want_nbr=True, **kw)
        gp, gx = pm.query_backward(qp[a:b], qn[a:b], g[a:b], nbr=o["nbr"], count=o["count"], **kw)
        torch.cuda.synchronize()
        for key in ("rad", "r2", "count", "nbr"):
            assert torch.equal(o[key], full[key][a:b]), (rank, key)
        gp, gx = gp[:, :3].double().cpu().numpy(), gx[:, :3].double().cpu().numpy()
        sum_p += gp
        sum_x += gx
        max_p, max_x = max(max_p, float(np.abs(gp).max())), max(max_x, float(np.abs(gx).max()))
    fp, fx = gp_full[:, :3].double().cpu().numpy(), gx_full[:, :3].double().cpu().numpy()
    assert (np.abs(sum_p - fp) <= (world + 1) * 2.0 ** -24 * max(max_p, float(np.abs(fp).max()))).all()
    assert (np.abs(sum_x - fx) <= (world + 1) * 2.0 ** -24 * max(max_x, float(np.abs(fx).max()))).all()
    assert pm.info().device_errors == 0
    pm.close()
