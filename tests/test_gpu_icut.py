"""Illumination cuts on the GPU against the oracle, on the engine's exported
tree (PhotonMap.cpp:287-452, GPU/illumcut.cu, GPU/photon_knn.cu:338-433,
598-716).

Bars: slot levels, centres, photon-derived normals, photon-sum estimates,
coarse and final cut marks bit-exact; node-centre irradiance within 1e-5 of
the FP64 oracle estimate (floor 1e-6 of the mean); interpolated irradiance
within 1e-6 relative of the oracle's FP64 interpolation over the engine's cut,
and the same number of cut nodes reached per query."""
import numpy as np
import pytest
import torch

from mnrt_b200 import _lib as L
from mnrt_b200 import gen
from mnrt_b200.photon_map import PhotonMap, RayChunk, ShadingPoints

pytestmark = pytest.mark.gpu


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def built_map(cuda, n, leaf, r, k, seed=700):
    ph = gen.photons(n, seed=seed + n, caustic_frac=0.2)
    pm = PhotonMap(n, global_q_radius_max=r, knn_target_count=k)
    pm.set_tuning(leaf_size=leaf)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    return ph, pm


def rel_err(got, ref):
    floor = 1e-6 * max(np.abs(ref).mean(), 1e-30)
    return (np.abs(got - ref) / np.maximum(np.abs(ref), floor)).max()


@pytest.mark.parametrize("n,leaf,k,r,use_leafs,level_emin,iters,acc", [
    (60000, 16, 50, 0.1, True, 12, 4, 0.2),      # the reference's defaults (cut = every leaf)
    (60000, 16, 50, 0.1, False, 6, 4, 0.2),
    (40000, 8, 20, 0.05, False, 9, 2, 0.1),
    (20000, 32, 100, 0.1, False, 3, 8, 0.3),
])
def test_icut_matches_oracle(cuda, oracle_mod, n, leaf, k, r, use_leafs, level_emin, iters, acc):
    ph, pm = built_map(cuda, n, leaf, r, k)
    pm.icut_build(use_leafs=use_leafs, level_emin=level_emin, refine_iters=iters, accuracy=acc)
    torch.cuda.synchronize()
    cut = pm.icut_export()
    nodes, tpos, tpow = pm.export_tree()
    o = oracle_mod.icut(nodes, tpow, use_leafs=use_leafs, level_emin=level_emin)
    assert np.array_equal(cut["level"], o["level"])
    assert np.array_equal(cut["center"].view(np.uint32), o["center"].view(np.uint32))
    assert np.array_equal(cut["normal"].view(np.uint32), o["normal"].view(np.uint32))
    assert np.array_equal(cut["est"].view(np.uint32), o["est"].view(np.uint32))
    assert np.array_equal(cut["coarse"], o["coarse"])
    # node-centre irradiance: exact kNN estimate at the centres with the slot normals (box, min_found 8)
    valid = cut["level"] != 0xFFFFFFFF
    cen, nrm = cut["center"].copy(), cut["normal"]
    cen[:, 3] = 0
    nb, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(cen, k, r)
    want = oracle_mod.radiance_fp64(ph.pos, ph.pow, cen, nrm, nb, cnt, k, r, "box", 1.0, 8)
    assert rel_err(cut["exact"][valid, :3], want[valid]) <= 1e-5
    fin = oracle_mod.icut_final(nodes, cut["coarse"], cut["est"], cut["exact"], iters, acc)
    assert np.array_equal(cut["final"], fin)
    if not use_leafs:
        assert 0 < cut["coarse"].sum() and cut["final"].sum() >= 1
    # interpolation at wall queries
    q = gen.queries(3000, seed=n + 1)
    got = pm.icut_interpolate(to_dev(q.pos, cuda), to_dev(q.nrm, cuda), r_max=r).cpu().numpy()
    irr, reached = oracle_mod.icut_interp(nodes, cut["final"], cut["center"], cut["normal"], cut["exact"], q.pos,
                                          q.nrm, r)
    assert np.array_equal(got[:, 3].astype(np.uint32), reached)
    assert rel_err(got[:, :3], irr) <= 1e-6
    assert pm.info().device_errors == 0


def test_icut_approximates_the_photon_estimate(cuda):
    """The interpolated irradiance follows the exact-kNN estimate it is built from."""
    n, k, r = 200000, 50, 0.05
    ph, pm = built_map(cuda, n, 16, r, k, seed=900)
    pm.icut_build()
    q = gen.queries(20000, seed=901)
    qp, qn = to_dev(q.pos, cuda), to_dev(q.nrm, cuda)
    interp = pm.icut_interpolate(qp, qn)[:, :3].sum(1).cpu().numpy()
    direct = pm.query(qp, qn, k=k, r_max=r, min_found=8)["rad"][:, :3].sum(1).cpu().numpy()
    ok = direct > 0
    ratio = interp[ok] / direct[ok]
    assert abs(np.median(ratio) - 1.0) < 0.1, np.median(ratio)
    assert np.percentile(np.abs(ratio - 1.0), 75) < 0.35


def test_icut_caller_normals_and_compat_node_query(cuda, oracle_mod):
    n, k, r = 30000, 30, 0.1
    ph, pm = built_map(cuda, n, 16, r, k, seed=950)
    ns = pm.icut_slot_count()
    centers = pm.icut_node_centers().cpu().numpy()
    # the caller's geometry: the inward normal of the nearest wall of the unit room
    c = centers[:, :3]
    dist = np.stack([c[:, 0], 1 - c[:, 0], c[:, 1], 1 - c[:, 1], c[:, 2]], 1)
    walls = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1]], np.float32)
    normals = np.zeros((ns, 4), np.float32)
    normals[:, :3] = walls[np.argmin(dist, 1)]
    pm.icut_build(use_leafs=False, level_emin=6, node_normals=to_dev(normals, cuda), mode=L.PM_MODE_ZHOU_COMPAT)
    cut = pm.icut_export()
    assert np.array_equal(cut["normal"][:, :3], normals[:, :3])
    assert np.array_equal(cut["center"], centers)
    # node-centre irradiance in compat mode = the compat query at the centres
    cen = to_dev(cut["center"], cuda)
    ref = pm.query(cen, to_dev(normals, cuda), mode=L.PM_MODE_ZHOU_COMPAT, min_found=8)["rad"].cpu().numpy()
    assert np.array_equal(cut["exact"][:, :3].view(np.uint32), ref[:, :3].view(np.uint32))
    nodes, tpos, tpow = pm.export_tree()
    o = oracle_mod.icut(nodes, tpow, use_leafs=False, level_emin=6, normals=normals)
    assert np.array_equal(cut["est"].view(np.uint32), o["est"].view(np.uint32))
    assert np.array_equal(cut["coarse"], o["coarse"])
    assert np.array_equal(cut["final"], oracle_mod.icut_final(nodes, cut["coarse"], cut["est"], cut["exact"], 4, 0.2))


def test_gather_for_with_icut(cuda):
    """GatherFor with cuts on accumulates clr.w * clr.rgb / pi * E_cut * influence
    at idx, with E_cut interpolated at the unflipped normal."""
    n, k, r = 50000, 40, 0.08
    ph, pm = built_map(cuda, n, 16, r, k, seed=1200)
    rng = np.random.default_rng(3)
    q = gen.queries(4000, seed=1201)
    nq = q.n
    dirs = np.zeros((nq, 4), np.float32)
    dirs[:, :3] = rng.normal(size=(nq, 3))
    dirs[:, :3] /= np.linalg.norm(dirs[:, :3], axis=1, keepdims=True)
    origins = q.pos.copy()
    origins[:, :3] -= dirs[:, :3]
    infl = rng.uniform(0.1, 1.0, size=(nq, 4)).astype(np.float32)
    clr = rng.uniform(0.0, 1.0, size=(nq, 4)).astype(np.float32)
    idx = rng.permutation(2 * nq)[:nq].astype(np.uint32)
    io = rng.uniform(0, 1, size=(2 * nq, 4)).astype(np.float32)
    pm.set_illum_cuts(True)
    pm.icut_build()
    d_io = to_dev(io, cuda)
    sp = ShadingPoints(to_dev(q.pos, cuda), to_dev(q.nrm, cuda))
    rays = RayChunk(to_dev(origins, cuda), to_dev(dirs, cuda), to_dev(infl, cuda))
    pm.gather_for(sp, rays, to_dev(clr, cuda), to_dev(idx.view(np.int32), cuda), d_io, None)
    e = pm.icut_interpolate(sp.pt_inter, sp.normals_s).cpu().numpy()
    inv_pi = np.float32(0.318309886183790671538)
    rad = (((clr[:, 3:4] * clr[:, :3]).astype(np.float32) * inv_pi).astype(np.float32) * e[:, :3]).astype(np.float32)
    rad = (rad * infl[:, :3]).astype(np.float32)
    want = io.copy()
    want[idx, :3] = (want[idx, :3] + rad).astype(np.float32)
    got = d_io.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # Gather (direct) never uses the cut: it matches the photon search
    io2 = np.zeros((nq, 4), np.float32)
    d2 = to_dev(io2, cuda)
    pm.gather(sp, rays, to_dev(clr, cuda), d2)
    pm.set_illum_cuts(False)
    d3 = to_dev(io2, cuda)
    pm.gather_for(sp, rays, to_dev(clr, cuda), None, d3, None)
    assert np.array_equal(d2.cpu().numpy(), d3.cpu().numpy())
    assert pm.info().device_errors == 0


def test_icut_state_rules(cuda):
    ph, pm = built_map(cuda, 5000, 16, 0.1, 20, seed=1300)
    q = gen.queries(100, seed=1301)
    qp, qn = to_dev(q.pos, cuda), to_dev(q.nrm, cuda)
    with pytest.raises(L.PMError):
        pm.icut_interpolate(qp, qn)                       # no cut yet
    pm.icut_build()
    pm.icut_interpolate(qp, qn)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))   # a rebuild drops the cut
    with pytest.raises(L.PMError):
        pm.icut_interpolate(qp, qn)
    sp = ShadingPoints(qp, qn)
    rays = RayChunk(qp.clone(), qn.clone(), torch.ones_like(qp))
    with pytest.raises(L.PMError):
        pm.gather_for(sp, rays, None, None, torch.zeros_like(qp), None, mode=L.PM_MODE_ICUT)
    # BuildMap with cuts enabled builds the cut (PhotonMap.cpp:166-168)
    pm2 = PhotonMap(ph.n, global_q_radius_max=0.1, knn_target_count=20)
    from mnrt_b200.photon_map import PhotonData
    pm2.set_illum_cuts(True)
    pm2.merge(PhotonData(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda), packed=True))
    pm2.build_map()
    assert pm2.icut_interpolate(qp, qn).shape == (100, 4)


@pytest.mark.parametrize("n", [0, 1, 20])
def test_icut_tiny_maps(cuda, n):
    """Empty map, one photon, one leaf as the whole tree: the cut is built,
    interpolation answers zeros or the single leaf, nothing faults."""
    ph = gen.photons(max(n, 1), seed=1400 + n, caustic_frac=0.0)
    pm = PhotonMap(max(n, 1), global_q_radius_max=0.2, knn_target_count=8)
    pm.build(to_dev(ph.pos[:n], cuda), to_dev(ph.pow[:n], cuda))
    pm.icut_build(min_found=0)
    q = gen.queries(64, seed=1401)
    got = pm.icut_interpolate(to_dev(q.pos, cuda), to_dev(q.nrm, cuda)).cpu().numpy()
    cut = pm.icut_export()
    assert cut["final"].shape == (2 * (pm.info().num_nodes + 1),)
    if n == 0:
        assert not got.any() and not cut["final"].any()
    else:
        assert cut["final"][0] == 1        # the root is the one leaf
        assert np.isfinite(got).all()
    assert pm.info().device_errors == 0
