"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bars (stated per test):
  * neighbour index sets, their order, counts and r^2: bit-exact;
  * radiance: relative error <= 1e-5 against the FP64 oracle on the same
    neighbour sets for every nonzero FP64 value, however small (no absolute
    floor), and exactly 0 where the FP64 value is 0.  The count of values
    below 1e-6 of the mean estimate (where a floored bar would have judged
    absolute error instead) is reported beside the relative errors.
"""
import numpy as np
import pytest
import torch

from mnrt_b200 import gen
from mnrt_b200 import _lib as L
from mnrt_b200.photon_map import PhotonMap

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def run(ph, q, dev, k, r_max, filt="box", cone_k=1.0, min_found=0, brute=False, sorted_queries=True, leaf=16,
        packed=True, tuning=None):
    pm = PhotonMap(max(ph.n, 1), global_q_radius_max=r_max)
    pm.set_tuning(leaf_size=leaf, **(tuning or {}))
    pm.build(to_dev(ph.pos, dev), to_dev(ph.pow, dev), packed=packed)
    out = pm.query(to_dev(q.pos, dev), to_dev(q.nrm, dev), want_nbr=True, brute_force=brute, k=k, r_max=r_max,
                   filter=filt, cone_k=cone_k, min_found=min_found, sorted_queries=sorted_queries)
    torch.cuda.synchronize()
    res = {kk: v.cpu().numpy() for kk, v in out.items()}
    res["info"] = pm.info()
    res["pm"] = pm
    return res


def radiance_errors(got, ref):
    """Relative radiance errors of FP32 results against FP64 values, per
    channel, with no absolute floor: |got - ref| / |ref| where ref != 0, and
    0 / inf where ref == 0 and got is / is not exactly 0.  Returns a dict of
    the max and mean relative error, the count of zero references, and the
    count of nonzero references below 1e-6 of the mean |ref| (the values a
    floored bar would have judged on absolute error) with their max error."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    nz = ref != 0.0
    rel = np.zeros_like(ref)
    rel[nz] = np.abs(got[nz] - ref[nz]) / np.abs(ref[nz])
    rel[~nz] = np.where(got[~nz] == 0.0, 0.0, np.inf)
    floor = 1e-6 * np.abs(ref).mean() if ref.size else 0.0
    small = nz & (np.abs(ref) < floor)
    return {"max": float(rel.max()) if rel.size else 0.0, "mean": float(rel.mean()) if rel.size else 0.0,
            "values": int(ref.size), "zero": int((~nz).sum()), "below_floor": int(small.sum()),
            "below_floor_max": float(rel[small].max()) if small.any() else 0.0}


def format_errors(e):
    return (f"max rel err {e['max']:.2e}, mean {e['mean']:.2e} over {e['values']:,} values "
            f"({e['zero']:,} exact zeros; {e['below_floor']:,} below 1e-6 of the mean, max {e['below_floor_max']:.2e})")


def check_against_oracle(oracle_mod, ph, q, res, k, r_max, filt, cone_k=1.0, min_found=0, pos_ref=None, pow_ref=None,
                         oracle_knn=None, threads=0):
    """Bit-exact neighbour lists, counts and r^2, and radiance within RTOL of
    the FP64 oracle (no floor); returns the error summary of radiance_errors."""
    pos_ref = ph.pos if pos_ref is None else pos_ref
    pow_ref = ph.pow if pow_ref is None else pow_ref
    if oracle_knn is None:
        oracle_knn = oracle_mod.KdTree(pos_ref, threads=threads).knn(q.pos, k, r_max, threads=threads)
    idx, _d2, cnt, r2 = oracle_knn
    nbr = res["nbr"].view(np.uint32)
    assert np.array_equal(res["count"].view(np.uint32), cnt), "neighbour counts differ"
    bad = np.where((nbr != idx).any(1))[0]
    assert bad.size == 0, f"{bad.size} queries with different neighbour lists, first {bad[:5]}"
    assert np.array_equal(res["r2"], r2), "r^2 differs"
    ref = oracle_mod.radiance_fp64(pos_ref, pow_ref, q.pos, q.nrm, idx, cnt, k, r_max, filt, cone_k, min_found,
                                   threads=threads)
    e = radiance_errors(res["rad"][:, :3], ref)
    assert e["max"] <= RTOL, f"radiance: {format_errors(e)}"
    assert np.array_equal(res["rad"][:, 3], cnt.astype(np.float32))
    return e


@pytest.mark.parametrize("filt", ["box", "cone", "epanechnikov"])
def test_small_config_parity(cuda, oracle_mod, filt):
    """Small configuration: 65,536 room photons, 16,384 wall queries, k = 50, R = 0.1."""
    cfg = gen.CONFIGS["small"]
    ph = gen.photons(cfg["n"], seed=100, caustic_frac=0.0, power_mean=cfg["power_mean"])
    q = gen.queries(cfg["nq"], seed=101)
    res = run(ph, q, cuda, cfg["k"], cfg["r_max"], filt)
    assert res["info"].device_errors == 0
    err = check_against_oracle(oracle_mod, ph, q, res, cfg["k"], cfg["r_max"], filt)
    print(f"small config {filt}: {format_errors(err)}")


KERNELS = [dict(kbuf_layout=0), dict(kbuf_layout=1, queries_per_warp=1), dict(kbuf_layout=1, queries_per_warp=2),
           dict(kbuf_layout=1, queries_per_warp=4), dict(kbuf_layout=1, queries_per_warp=8),
           dict(kbuf_layout=1, queries_per_warp=1, rounds_per_chunk=1), dict(kbuf_layout=2),
           dict(kbuf_layout=2, rounds_per_chunk=1, leaf_size=4)]


@pytest.mark.parametrize("kern", KERNELS, ids=["heap", "g32", "g16", "g8", "g4", "g32r1", "wide", "wide_l4"])
@pytest.mark.parametrize("k,filt", [(100, "cone"), (16, "box"), (128, "epanechnikov")])
def test_kernel_variants_bitwise_equal(cuda, oracle_mod, kern, k, filt):
    """Every k-buffer layout / queries-per-warp variant gives the same bits."""
    ph = gen.photons(60000, seed=31, caustic_frac=0.2)
    ph.pos[100:160, :3] = ph.pos[7, :3]               # a pile of coincident photons
    q = gen.queries(6000, seed=32)
    q.pos[:20, :3] = ph.pos[7, :3]
    ref = run(ph, q, cuda, k, 0.05, filt, brute=True)
    tun = {"rounds_per_chunk": 5, **kern}
    leaf = tun.pop("leaf_size", 16)
    res = run(ph, q, cuda, k, 0.05, filt, tuning=tun, leaf=leaf)
    for key in ("nbr", "count", "r2", "rad"):
        assert np.array_equal(res[key], ref[key]), key
    assert res["info"].device_errors == 0
    check_against_oracle(oracle_mod, ph, q, res, k, 0.05, filt)


def test_tree_matches_bruteforce_and_order_invariance(cuda):
    ph = gen.photons(40000, seed=7, caustic_frac=0.2)
    q = gen.queries(5000, seed=8)
    a = run(ph, q, cuda, 64, 0.05, "cone", cone_k=1.2)
    b = run(ph, q, cuda, 64, 0.05, "cone", cone_k=1.2, brute=True)
    c = run(ph, q, cuda, 64, 0.05, "cone", cone_k=1.2, sorted_queries=False)
    for key in ("nbr", "count", "r2", "rad"):
        assert np.array_equal(a[key], b[key]), key
        assert np.array_equal(a[key], c[key]), key


@pytest.mark.parametrize("leaf", [1, 4, 16, 32, 33, 48, 64])
def test_leaf_sizes_and_tuning(cuda, oracle_mod, leaf):
    ph = gen.photons(20000, seed=9, caustic_frac=0.3, caustic_sigma=0.005)
    q = gen.queries(3000, seed=10)
    res = run(ph, q, cuda, 32, 0.08, "epanechnikov", leaf=leaf,
              tuning=dict(warps_per_block=2, rounds_per_chunk=3))
    check_against_oracle(oracle_mod, ph, q, res, 32, 0.08, "epanechnikov")


@pytest.mark.parametrize("leaf", [33, 64])
@pytest.mark.parametrize("layout,qpw", [(0, 1), (1, 1), (1, 2), (1, 4), (1, 8), (2, 1)])
def test_large_leaves_every_layout(cuda, oracle_mod, leaf, layout, qpw):
    """Leaves of more than 32 photons (up to 64: two per lane) in every
    k-buffer layout: the heap and group layouts scan them 32 photons at a
    time, the wide layout in two halves."""
    ph = gen.photons(30000, seed=31, caustic_frac=0.3, caustic_sigma=0.005)
    q = gen.queries(2500, seed=32)
    for k in (16, 100):
        res = run(ph, q, cuda, k, 0.08, "cone", leaf=leaf,
                  tuning=dict(warps_per_block=4, rounds_per_chunk=8, queries_per_warp=qpw, kbuf_layout=layout))
        assert res["info"].leaf_size == leaf
        check_against_oracle(oracle_mod, ph, q, res, k, 0.08, "cone")


@pytest.mark.parametrize("k", [1, 2, 100, 128])
def test_k_extremes(cuda, oracle_mod, k):
    ph = gen.photons(30000, seed=11 + k)
    q = gen.queries(2000, seed=12)
    res = run(ph, q, cuda, k, 0.07, "box", min_found=8)
    check_against_oracle(oracle_mod, ph, q, res, k, 0.07, "box", min_found=8)


def test_duplicates_and_ties(cuda, oracle_mod):
    """Coincident photons and equal distances: ties broken by caller index."""
    ph = gen.photons(5000, seed=13)
    ph.pos[1000:1300, :3] = ph.pos[5, :3]           # 301 photons at one point
    ph.pos[2000:2010, :3] = ph.pos[6, :3]
    q = gen.queries(600, seed=14)
    q.pos[:50, :3] = ph.pos[5, :3]                   # queries on the pile
    q.pos[50:60, :3] = ph.pos[6, :3]
    grid = np.stack(np.meshgrid(np.arange(8), np.arange(8), indexing="ij"), -1).reshape(-1, 2) / 8.0
    ph.pos[3000:3064, 0] = grid[:, 0]                # lattice: many exactly equal distances
    ph.pos[3000:3064, 1] = 0.0
    ph.pos[3000:3064, 2] = grid[:, 1]
    q.pos[60:70, :3] = [0.0625, 0.0, 0.0625]
    for k in (16, 128):
        res = run(ph, q, cuda, k, 0.3, "cone")
        check_against_oracle(oracle_mod, ph, q, res, k, 0.3, "cone")


@pytest.mark.parametrize("leaf", [16, 64])
def test_edge_maps(cuda, oracle_mod, leaf):
    """Empty and tiny maps, including single-leaf trees of up to 64 photons."""
    q = gen.queries(300, seed=15)
    for n in (0, 1, 2, 5, 16, 17, 33, 63, 64, 65):
        ph = gen.photons(n, seed=16 + n) if n else gen.PhotonSet(np.zeros((0, 4), np.float32),
                                                                  np.zeros((0, 4), np.float32),
                                                                  np.zeros((0, 3), np.float32), "packed")
        res = run(ph, q, cuda, 8, 2.0, "box", leaf=leaf)
        if n == 0:
            assert (res["count"] == 0).all() and (res["rad"] == 0).all()
            assert (res["nbr"].view(np.uint32) == 0xFFFFFFFF).all()
        else:
            check_against_oracle(oracle_mod, ph, q, res, 8, 2.0, "box")


def test_far_queries_and_nonfinite(cuda):
    ph = gen.photons(2000, seed=17)
    q = gen.queries(100, seed=18)
    q.pos[:10, :3] += 50.0          # nothing within R
    q.pos[10, 0] = np.nan           # flagged, zero output
    res = run(ph, q, cuda, 10, 0.1, "box")
    assert (res["count"][:11] == 0).all() and (res["rad"][:11] == 0).all()
    assert res["info"].device_errors & L.PM_DEVERR_QNONFINITE


def test_reference_layout_ingest(cuda, oracle_mod):
    """MNRT's PhotonData layout (azimuth / polar angles in .w) gives the same
    packed directions on the GPU as the oracle's ingest, bit for bit."""
    ph = gen.photons(20000, seed=19, layout="reference")
    q = gen.queries(2000, seed=20)
    res = run(ph, q, cuda, 40, 0.06, "box", packed=False)
    op, ow = oracle_mod.pack_reference(ph.pos, ph.pow)
    _, tpos, tpow = res["pm"].export_tree()
    order = tpos[:, 3].view(np.uint32)
    assert np.array_equal(tpow[:, 3].view(np.uint32), ow[order, 3].view(np.uint32))
    check_against_oracle(oracle_mod, ph, q, res, 40, 0.06, "box", pos_ref=op, pow_ref=ow)


def test_tree_structure(cuda):
    """Every photon in exactly one leaf; leaves <= leaf size; child boxes
    bound their photons and nest in their parent's box; nodes 64-byte."""
    ph = gen.photons(50000, seed=21, caustic_frac=0.2)
    leaf = 16
    pm = PhotonMap(ph.n, global_q_radius_max=0.1)
    pm.set_tuning(leaf_size=leaf)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    nodes, tpos, tpow = pm.export_tree()
    assert np.array_equal(np.sort(tpos[:, 3].view(np.uint32)), np.arange(ph.n, dtype=np.uint32))
    assert np.array_equal(tpos[:, :3], ph.pos[tpos[:, 3].view(np.uint32), :3])
    f = nodes.view(np.float32)
    seen = np.zeros(ph.n, np.int32)
    stack = [(0, 0, None)]
    visited = 0
    while stack:
        node, side, pbox = stack.pop()
        base = side * 8
        lo, hi = f[node, base:base + 3], f[node, base + 3:base + 6]
        ref, cnt = nodes[node, base + 6], nodes[node, base + 7]
        if pbox is not None:
            assert (lo >= pbox[0]).all() and (hi <= pbox[1]).all()
        if cnt > 0:
            assert cnt <= leaf
            seen[ref:ref + cnt] += 1
            pts = tpos[ref:ref + cnt, :3]
            assert (pts >= lo).all() and (pts <= hi).all()
        else:
            visited += 1
            stack.append((ref, 0, (lo, hi)))
            stack.append((ref, 1, (lo, hi)))
    assert (seen == 1).all()
    assert visited == nodes.shape[0] - 1


GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", ["small_k50_r01", "caustic_k16_r005", "sparse_k128_r002"])
@pytest.mark.parametrize("filt", ["box", "cone", "epanechnikov"])
def test_engine_reproduces_golden(cuda, name, filt):
    """The CUDA path against the committed fixtures: neighbour lists, counts and
    r^2 bit-exact; radiance within RTOL of the fixture's FP64 value."""
    with np.load(GOLDEN / f"{name}.npz") as z:
        g = {key: z[key] for key in z.files}
    k, r = int(g["k"]), float(g["r_max"])
    ph = gen.PhotonSet(g["pos"], g["pow"], np.zeros((g["pos"].shape[0], 3), np.float32), "packed")
    q = gen.QuerySet(g["qpos"], g["qnrm"])
    res = run(ph, q, cuda, k, r, filt)
    assert np.array_equal(res["nbr"].view(np.uint32), g["idx"])
    assert np.array_equal(res["count"].view(np.uint32), g["count"])
    assert np.array_equal(res["r2"], g["r2"])
    e = radiance_errors(res["rad"][:, :3], g[f"rad_{filt}"])
    assert e["max"] <= RTOL, format_errors(e)


@pytest.mark.parametrize("filt", ["box", "cone", "epanechnikov"])
def test_engine_reproduces_adjoint_golden(cuda, filt):
    """The CUDA adjoint against the committed FP64 gradients (the oracle and
    the numpy restatement agreed on them): neighbour lists bit-exact, the
    gradients within 1e-5 relative of the fixture."""
    with np.load(GOLDEN / "adjoint_k16_r025.npz") as z:
        g = {key: z[key] for key in z.files}
    k, r = int(g["k"]), float(g["r_max"])
    pm = PhotonMap(g["pos"].shape[0], global_q_radius_max=r, knn_target_count=k)
    pm.build(to_dev(g["pos"], cuda), to_dev(g["pow"], cuda))
    qp, qn = to_dev(g["qpos"], cuda), to_dev(g["qnrm"], cuda)
    out = pm.query(qp, qn, want_nbr=True, k=k, r_max=r, filter=filt)
    grad = torch.zeros((qp.shape[0], 4), dtype=torch.float32, device=cuda)
    grad[:, :3] = torch.from_numpy(g[f"g_{filt}"]).to(cuda)   # FP32, as the fixture's gradients took it
    gp, gx = pm.query_backward(qp, qn, grad, nbr=out["nbr"], count=out["count"], k=k, r_max=r, filter=filt)
    torch.cuda.synchronize()
    assert np.array_equal(out["nbr"].cpu().numpy().view(np.uint32), g["idx"])
    for got, want in ((gp[:, :3].cpu().numpy(), g[f"gpow_{filt}"]), (gx[:, :3].cpu().numpy(), g[f"gpos_{filt}"])):
        floor = 1e-6 * np.abs(want).max()
        assert (np.abs(got - want) / np.maximum(np.abs(want), floor)).max() <= 1e-5
    assert pm.info().device_errors == 0


def test_engine_reproduces_ingest_golden(cuda):
    """Reference-layout photons (azimuth / polar angle): the GPU ingest gives
    the fixture's packed direction bits."""
    with np.load(GOLDEN / "reference_ingest.npz") as z:
        pos, pw, bits = z["pos"], z["pow"], z["oct_bits"]
    pm = PhotonMap(pos.shape[0], global_q_radius_max=0.1)
    pm.build(to_dev(pos, cuda), to_dev(pw, cuda), packed=False)
    _, tpos, tpow = pm.export_tree()
    order = tpos[:, 3].view(np.uint32)
    assert np.array_equal(tpow[:, 3].view(np.uint32), bits[order])


def test_autotune_keeps_results_exact(cuda, oracle_mod):
    """pm_autotune picks a setting from its grid, leaves the map built with it,
    and the query results stay bit-exact against the oracle."""
    ph = gen.photons(80000, seed=140, caustic_frac=0.2)
    q = gen.queries(20000, seed=141)
    pm = PhotonMap(ph.n, global_q_radius_max=0.05)
    d_pos, d_pow, d_qp, d_qn = (to_dev(x, cuda) for x in (ph.pos, ph.pow, q.pos, q.nrm))
    t = pm.autotune(d_pos, d_pow, d_qp, d_qn, max_sample=4096, k=64, r_max=0.05, filter="cone")
    assert t.leaf_size in (16, 24, 32, 48, 64) and t.warps_per_block in (2, 4, 8) and t.rounds_per_chunk in (8, 32)
    assert t.queries_per_warp in (1, 2) and t.kbuf_layout in (0, 1, 2) and t.query_ms > 0
    out = pm.query(d_qp, d_qn, want_nbr=True, k=64, r_max=0.05, filter="cone")
    torch.cuda.synchronize()
    res = {kk: v.cpu().numpy() for kk, v in out.items()}
    check_against_oracle(oracle_mod, ph, q, res, 64, 0.05, "cone")


def _morton39(p, lo, scale):
    """Host restatement of the engine's 39-bit Morton code: the top 13 bits of
    each axis' 16-bit quantisation, interleaved with x most significant."""
    q = np.clip((p[:, :3].astype(np.float32) - lo.astype(np.float32)).astype(np.float32) * np.float32(scale),
                0.0, 65535.0).astype(np.float32)
    q = np.nan_to_num(q).astype(np.uint64) >> np.uint64(3)

    def spread(v):
        v = v & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x0000FF0000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00F00F00F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0C30C30C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x249249249249)
        return v
    return (spread(q[:, 0]) << np.uint64(2)) | (spread(q[:, 1]) << np.uint64(1)) | spread(q[:, 2])


@pytest.mark.parametrize("n", [1, 2, 3, 2047, 2048, 2049, 4097, 65537, 100003, 4194305])
def test_radix_sort_and_scan_through_tree_order(cuda, n):
    """The exported tree order is exactly the order of (Morton code, caller
    index) -- the device radix sort, whose last pass moves the photons into
    tree order, checked end to end at odd sizes around the 2,048-key sort tile,
    and above 2,048 tiles (4,194,304 keys), where a pass scans the whole
    digit-major array instead of one row per digit -- and the compaction scan
    kept exactly the nodes that hold more than leaf_size photons."""
    ph = gen.photons(n, seed=600 + n, caustic_frac=0.3)
    ph.pos[: n // 3, :3] = np.round(ph.pos[: n // 3, :3] * 64) / 64   # many equal codes: ties by index
    pm = PhotonMap(n, global_q_radius_max=0.1)
    pm.set_tuning(leaf_size=16)
    pm.build(to_dev(ph.pos, cuda), to_dev(ph.pow, cuda))
    nodes, tpos, _ = pm.export_tree()
    info = pm.info()
    lo = np.array(info.bounds_min, np.float32)
    hi = np.array(info.bounds_max, np.float32)
    ext = np.float32(max(hi - lo))
    scale = np.float32(65536.0) / ext if ext > 0 else np.float32(0)
    idx = tpos[:, 3].view(np.uint32)
    codes = _morton39(ph.pos[idx], lo, scale)
    dc = np.diff(codes.astype(np.int64))
    di = np.diff(idx.astype(np.int64))
    assert ((dc > 0) | ((dc == 0) & (di > 0))).all(), "tree order is not (code, index) order"
    # every kept node holds more than leaf_size photons: leaves of at most 16, internal slots otherwise
    cnts = nodes[:, [7, 15]]
    assert (cnts <= 16).all()


@pytest.mark.parametrize("chunks,pinned", [(1, True), (3, True), (1, False), (4, False), (16, True)])
def test_build_query_host_matches_device_calls(cuda, chunks, pinned):
    """pm_build_query_host (host buffers, chunked and overlapped) gives the
    bits of pm_build + pm_query on device buffers: a page-locked radiance
    array written in place by the query kernel, a pageable one through a
    device copy."""
    from mnrt_b200.photon_map import PhotonMap
    ph = gen.photons(80000, seed=71, caustic_frac=0.2)
    q = gen.queries(30001, seed=72)
    pm = PhotonMap(ph.n, global_q_radius_max=0.05, knn_target_count=64)
    h = lambda a: (torch.from_numpy(np.ascontiguousarray(a)).pin_memory() if pinned
                   else torch.from_numpy(np.ascontiguousarray(a)))
    out = None if pinned else torch.empty((q.n, 4), dtype=torch.float32)   # None: a page-locked output
    got = pm.build_query_host(h(ph.pos), h(ph.pow), h(q.pos), h(q.nrm), out=out, chunks=chunks, filter="cone",
                              min_found=8)
    torch.cuda.synchronize()
    pm2 = PhotonMap(ph.n, global_q_radius_max=0.05, knn_target_count=64)
    pm2.build(torch.from_numpy(ph.pos).to(cuda), torch.from_numpy(ph.pow).to(cuda))
    want = pm2.query(torch.from_numpy(q.pos).to(cuda), torch.from_numpy(q.nrm).to(cuda), filter="cone",
                     min_found=8)["rad"].cpu()
    assert torch.equal(got.view(torch.int32), want.view(torch.int32))
    assert pm.info().device_errors == 0


def test_build_query_host_misaligned_pinned_output(cuda):
    """A page-locked output that is not 16-byte aligned cannot take the
    kernel's float4 stores: it goes through the device copy and still gets
    the device calls' bits."""
    from mnrt_b200.photon_map import PhotonMap
    ph = gen.photons(20000, seed=77, caustic_frac=0.2)
    q = gen.queries(3001, seed=78)
    pm = PhotonMap(ph.n, global_q_radius_max=0.05, knn_target_count=32)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    buf = torch.zeros(q.n * 4 + 1, dtype=torch.float32).pin_memory()
    out = buf[1:].view(q.n, 4)
    assert out.data_ptr() % 16 != 0
    pm.build_query_host(pin(ph.pos), pin(ph.pow), pin(q.pos), pin(q.nrm), out=out, filter="cone")
    torch.cuda.synchronize()
    pm2 = PhotonMap(ph.n, global_q_radius_max=0.05, knn_target_count=32)
    pm2.build(torch.from_numpy(ph.pos).to(cuda), torch.from_numpy(ph.pow).to(cuda))
    want = pm2.query(torch.from_numpy(q.pos).to(cuda), torch.from_numpy(q.nrm).to(cuda), filter="cone")["rad"].cpu()
    assert torch.equal(out.view(torch.int32), want.view(torch.int32))
    assert pm.info().device_errors == 0


def test_build_query_host_empty_inputs(cuda):
    from mnrt_b200.photon_map import PhotonMap
    ph = gen.photons(1000, seed=73)
    q = gen.queries(10, seed=74)
    pm = PhotonMap(ph.n, global_q_radius_max=0.1, knn_target_count=8)
    z4 = torch.zeros((0, 4), dtype=torch.float32)
    out = pm.build_query_host(torch.from_numpy(ph.pos), torch.from_numpy(ph.pow), z4, z4)
    torch.cuda.synchronize()
    assert out.shape == (0, 4)
    out = pm.build_query_host(z4, z4, torch.from_numpy(q.pos), torch.from_numpy(q.nrm))
    torch.cuda.synchronize()
    assert out.shape == (10, 4) and not out.any()
    assert pm.info().device_errors == 0


@pytest.mark.parametrize("k,filt", [(1, "cone"), (2, "cone"), (2, "epanechnikov"), (5, "cone")])
def test_channel_imbalanced_flux_small_k(cuda, oracle_mod, k, filt):
    """Per-channel accuracy of the FP32 fast path: when one channel's flux sits
    almost entirely in low-weight neighbours (the k-th at weight zero), that
    channel alone must trigger the FP64 re-evaluation."""
    ph = gen.photons(60000, seed=910, caustic_frac=0.2)
    rng = np.random.default_rng(911)
    tiny = rng.random(ph.n) < 0.5
    ph.pow[tiny, 2] *= np.float32(1e-4)          # half the photons carry almost no blue
    ph.pow[~tiny, 0] *= np.float32(1e-4)         # the other half almost no red
    q = gen.queries(5000, seed=912)
    res = run(ph, q, cuda, k, 1.5, filt, leaf=32, tuning=dict(kbuf_layout=2))
    assert res["info"].device_errors == 0
    check_against_oracle(oracle_mod, ph, q, res, k, 1.5, filt)

