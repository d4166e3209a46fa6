"""pm_gather_for against the oracle: PhotonMap::GatherFor semantics
(PhotonMap.cpp:234-270, GPU/photon_knn.cu:493-551).

Bars: the accumulated radiance within 1e-5 relative of the expression
clr.w * clr.rgb / pi * E * influence evaluated in FP32 from the FP64 oracle
estimate E (floor 1e-6 of the mean), added to the prior contents; the
reciprocal-distance accumulator within 2 ulp; untouched slots unchanged."""
import numpy as np
import pytest
import torch

from mnrt_b200 import gen
from mnrt_b200.photon_map import PhotonMap, RayChunk, ShadingPoints

pytestmark = pytest.mark.gpu


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def flip_normals(nrm, dirs):
    d = (((-dirs[:, 0]) * nrm[:, 0]).astype(np.float32) + ((-dirs[:, 1]) * nrm[:, 1]).astype(np.float32)).astype(
        np.float32) + ((-dirs[:, 2]) * nrm[:, 2]).astype(np.float32)
    out = nrm.copy()
    out[d < 0, :3] *= -1
    out[:, 3] = 0
    return out


def make_case(seed, n_ph=30000, n=4000):
    rng = np.random.default_rng(seed)
    ph = gen.photons(n_ph, seed=seed, caustic_frac=0.2)
    q = gen.queries(n, seed=seed + 1)
    dirs = np.zeros((n, 4), np.float32)
    dirs[:, :3] = rng.normal(size=(n, 3))
    dirs[:, :3] /= np.linalg.norm(dirs[:, :3], axis=1, keepdims=True)
    origins = q.pos.copy()
    origins[:, :3] -= dirs[:, :3] * rng.uniform(0.1, 2.0, size=(n, 1)).astype(np.float32)
    infl = rng.uniform(0.1, 1.0, size=(n, 4)).astype(np.float32)
    clr = rng.uniform(0.0, 1.0, size=(n, 4)).astype(np.float32)
    return ph, q, dirs, origins, infl, clr


def expected(oracle_mod, ph, q, dirs, origins, infl, clr, k, r, min_found, filt, io_rad, io_rec, idx):
    nrm = flip_normals(q.nrm, dirs)
    nb, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
    e = oracle_mod.radiance_fp64(ph.pos, ph.pow, q.pos, nrm, nb, cnt, k, r, filt, 1.0, min_found).astype(np.float32)
    c = clr if clr is not None else np.ones_like(infl)
    inv_pi = np.float32(0.318309886183790671538)
    rad = (((c[:, 3:4] * c[:, :3]).astype(np.float32) * inv_pi).astype(np.float32) * e).astype(np.float32)
    rad = (rad * infl[:, :3]).astype(np.float32)
    out = io_rad.copy()
    out[idx, :3] = (out[idx, :3] + rad).astype(np.float32)
    rec = None
    if io_rec is not None:
        dv = (q.pos[:, :3] - origins[:, :3]).astype(np.float32)
        d2 = ((dv[:, 0] * dv[:, 0] + dv[:, 1] * dv[:, 1]).astype(np.float32) + dv[:, 2] * dv[:, 2]).astype(np.float32)
        rec = io_rec.copy()
        rec[idx] = (rec[idx] + (1.0 / np.sqrt(d2.astype(np.float64))).astype(np.float32)).astype(np.float32)
    return out, rec


@pytest.mark.parametrize("use_idx,use_recip,use_clr", [(True, True, True), (False, False, True), (False, False, False)])
def test_gather_for_matches_oracle(cuda, oracle_mod, use_idx, use_recip, use_clr):
    ph, q, dirs, origins, infl, clr = make_case(120)
    n = q.n
    k, r = 50, 0.06
    rng = np.random.default_rng(5)
    slots = 3 * n
    idx = rng.permutation(slots)[:n].astype(np.uint32) if use_idx else np.arange(n, dtype=np.uint32)
    io_rad = rng.uniform(0, 1, size=(slots if use_idx else n, 4)).astype(np.float32)
    io_rec = rng.uniform(0, 1, size=(slots if use_idx else n,)).astype(np.float32) if use_recip else None
    pm = PhotonMap(ph.n, global_q_radius_max=r, knn_target_count=k)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    d_rad = to_dev(io_rad, cuda)
    d_rec = to_dev(io_rec, cuda) if use_recip else None
    sp = ShadingPoints(to_dev(q.pos, cuda), to_dev(q.nrm, cuda))
    rays = RayChunk(to_dev(origins, cuda), to_dev(dirs, cuda), to_dev(infl, cuda))
    c = to_dev(clr, cuda) if use_clr else None
    if use_clr:
        pm.gather_for(sp, rays, c, to_dev(idx.view(np.int32), cuda) if use_idx else None, d_rad, d_rec)
    else:   # the visualisation form: white, no photon-count rule
        pm.gather_for(sp, rays, None, None, d_rad, None, min_found=0)
    torch.cuda.synchronize()
    exp_rad, exp_rec = expected(oracle_mod, ph, q, dirs, origins, infl, clr if use_clr else None, k, r,
                                8 if use_clr else 0, "box", io_rad, io_rec, idx)
    got = d_rad.cpu().numpy()
    # increments within 1e-5 of the oracle's, plus the FP32 rounding of the sum
    inc_ref = exp_rad[:, :3].astype(np.float64) - io_rad[:, :3]
    inc_got = got[:, :3].astype(np.float64) - io_rad[:, :3]
    tol = 1e-5 * np.abs(inc_ref) + 2 * np.finfo(np.float32).eps * np.abs(exp_rad[:, :3])
    assert (np.abs(inc_got - inc_ref) <= tol).all(), np.abs(inc_got - inc_ref).max()
    assert np.array_equal(got[:, 3], io_rad[:, 3])
    untouched = np.setdiff1d(np.arange(got.shape[0]), idx)
    assert np.array_equal(got[untouched], io_rad[untouched])
    if use_recip:
        assert np.allclose(d_rec.cpu().numpy(), exp_rec, rtol=2.4e-7, atol=0)
    assert pm.info().device_errors == 0


def test_gather_normal_flip_and_min_found(cuda, oracle_mod):
    """Rays arriving from behind flip the normal (the front test then sees the
    photons of the other side); estimates from fewer than 8 photons vanish."""
    ph, q, dirs, origins, infl, clr = make_case(130, n_ph=2000, n=1500)
    dirs[:, :3] = q.nrm[:, :3]          # every ray travels along the normal: all flipped
    k, r = 16, 0.03
    pm = PhotonMap(ph.n, global_q_radius_max=r, knn_target_count=k)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    io_rad = np.zeros((q.n, 4), np.float32)
    d_rad = to_dev(io_rad, cuda)
    sp = ShadingPoints(to_dev(q.pos, cuda), to_dev(q.nrm, cuda))
    rays = RayChunk(to_dev(origins, cuda), to_dev(dirs, cuda), to_dev(infl, cuda))
    pm.gather(sp, rays, to_dev(clr, cuda), d_rad)
    torch.cuda.synchronize()
    exp_rad, _ = expected(oracle_mod, ph, q, dirs, origins, infl, clr, k, r, 8, "box", io_rad, None,
                          np.arange(q.n))
    assert np.allclose(d_rad.cpu().numpy(), exp_rad, rtol=1e-5, atol=1e-9)


def test_merge_scale_build_pipeline(cuda, oracle_mod):
    """PhotonMap.merge -> scale_flux -> build_map (the reference's build
    sequence, RTCore.cpp:526-620 -> PhotonMap.cpp:157-193) equals building the
    valid photons, scaled, directly: same tree order and bit-identical query."""
    from mnrt_b200.photon_map import PhotonData
    ph = gen.photons(30000, seed=150, caustic_frac=0.2, layout="reference")
    valid = (np.arange(ph.n) % 4 != 1).astype(np.uint32) * 3
    half = ph.n // 2
    pm = PhotonMap(ph.n, global_q_radius_max=0.06, knn_target_count=40)
    total = 0
    for a, b in ((0, half), (half, ph.n)):     # two tracing passes merged in turn
        total += pm.merge(PhotonData(to_dev(ph.pos[a:b], cuda), to_dev(ph.pow[a:b], cuda)),
                          to_dev(valid[a:b].view(np.int32), cuda))
    assert total == int((valid != 0).sum())
    pm.scale_flux(0.25)
    pm.build_map()
    keep = valid != 0
    ref_pos, ref_pow = ph.pos[keep].copy(), ph.pow[keep].copy()
    ref_pow[:, :3] *= np.float32(0.25)
    pm2 = PhotonMap(ph.n, global_q_radius_max=0.06)
    pm2.build(to_dev(ref_pos, cuda), to_dev(ref_pow, cuda), packed=False)
    q = gen.queries(3000, seed=151)
    a = pm.query(to_dev(q.pos, cuda), to_dev(q.nrm, cuda), want_nbr=True, k=40, r_max=0.06, filter="cone")
    b = pm2.query(to_dev(q.pos, cuda), to_dev(q.nrm, cuda), want_nbr=True, k=40, r_max=0.06, filter="cone")
    torch.cuda.synchronize()
    for key in ("rad", "nbr", "r2", "count"):
        assert torch.equal(a[key], b[key]), key
    pm.clear()
    pm.build_map()
    assert pm.info().num_photons == 0
