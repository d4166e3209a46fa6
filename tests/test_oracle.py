"""CPU tests of the oracle: contract pieces, kNN, FP64 estimate (no GPU)."""
import ctypes as C

import numpy as np
import pytest

from mnrt_b200 import gen
from tests import np_restate


def test_oct_encode_matches_numpy(oracle_mod):
    lib = oracle_mod.load()
    rng = np.random.default_rng(1)
    d = rng.normal(size=(4000, 3)).astype(np.float32)
    d[:8] = [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [0, 0, 0], [1e-30, -1e-30, 0]]
    ours = gen.oct_encode(d)
    ref = np.array([lib.orc_oct_encode(*map(float, v)) for v in d], np.uint32)
    assert np.array_equal(ours, ref)


def test_oct_decode_and_front_match_numpy(oracle_mod):
    lib = oracle_mod.load()
    rng = np.random.default_rng(2)
    bits = rng.integers(0, 2**32, size=3000, dtype=np.uint64).astype(np.uint32)
    dec = gen.oct_decode(bits)
    out = (C.c_float * 3)()
    for b, v in zip(bits[:500], dec[:500]):
        lib.orc_oct_decode(int(b), out)
        assert np.array_equal(np.array(out[:], np.float32), v)
    n4 = np.zeros((3000, 4), np.float32)
    n4[:, :3] = rng.normal(size=(3000, 3))
    fr = np_restate.front(n4, bits)
    ref = np.array([lib.orc_front(float(n[0]), float(n[1]), float(n[2]), int(b)) for n, b in zip(n4, bits)], bool)
    assert np.array_equal(fr, ref)


def test_oct_roundtrip_accuracy():
    rng = np.random.default_rng(3)
    d = rng.normal(size=(20000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    back = gen.oct_decode(gen.oct_encode(d.astype(np.float32))).astype(np.float64)
    back /= np.linalg.norm(back, axis=1, keepdims=True)
    ang = np.arccos(np.clip((back * d).sum(1), -1, 1))
    assert ang.max() < 1e-4   # 16-bit octahedral: ~4e-5 rad worst case


def test_deterministic_sincos_accuracy(oracle_mod):
    lib = oracle_mod.load()
    out = (C.c_double * 2)()
    xs = np.concatenate([np.linspace(0, 2 * np.pi, 2001), np.linspace(-7, 7, 301), [np.pi / 4, np.pi / 2, np.pi]])
    for x in xs:
        lib.orc_sincos(float(x), out)
        assert abs(out[0] - np.sin(x)) < 4e-16 and abs(out[1] - np.cos(x)) < 4e-16


def test_spherical_ingest_matches_direction(oracle_mod):
    ph = gen.photons(3000, seed=5, layout="reference")
    pos, pw = oracle_mod.pack_reference(ph.pos, ph.pow)
    assert np.array_equal(pos[:, 3].view(np.uint32), np.arange(3000, dtype=np.uint32))
    dec = gen.oct_decode(pw[:, 3].view(np.uint32)).astype(np.float64)
    dec /= np.linalg.norm(dec, axis=1, keepdims=True)
    d = ph.dirs.astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    assert np.arccos(np.clip((dec * d).sum(1), -1, 1)).max() < 2e-4


def _small_case(n, nq, seed, dup=False):
    ph = gen.photons(n, seed=seed, caustic_frac=0.2, caustic_sigma=0.02)
    q = gen.queries(nq, seed=seed + 1)
    if dup:   # exact duplicates and equal-distance ties
        ph.pos[n // 2:n // 2 + 40, :3] = ph.pos[0, :3]
        q.pos[:5, :3] = ph.pos[0, :3]
    return ph, q


@pytest.mark.parametrize("k,r_max", [(1, 0.2), (8, 0.15), (50, 0.3), (128, 1.0), (40, 0.02)])
def test_knn_brute_matches_numpy(oracle_mod, k, r_max):
    ph, q = _small_case(700, 60, seed=11 + k, dup=True)
    idx, d2, cnt, r2 = oracle_mod.knn_brute(ph.pos, q.pos, k, r_max)
    ridx, rd2, rcnt, rr2 = np_restate.knn(ph.pos, q.pos, k, r_max)
    assert np.array_equal(cnt, rcnt)
    assert np.array_equal(idx, ridx)
    assert np.array_equal(d2, rd2)
    assert np.array_equal(r2, rr2)


def test_knn_kdtree_matches_brute(oracle_mod):
    ph, q = _small_case(30000, 3000, seed=21, dup=True)
    for k, r in [(50, 0.1), (100, 0.05), (16, 0.01)]:
        a = oracle_mod.knn_brute(ph.pos, q.pos, k, r)
        b = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_knn_edge_cases(oracle_mod):
    ph, q = _small_case(50, 10, seed=31)
    empty = np.zeros((0, 4), np.float32)
    idx, d2, cnt, r2 = oracle_mod.knn_brute(empty, q.pos, 5, 0.5)
    assert (cnt == 0).all() and (idx == 0xFFFFFFFF).all()
    idx, d2, cnt, r2 = oracle_mod.knn_brute(ph.pos, q.pos, 80, 10.0)   # k > n
    assert (cnt == 50).all() and (idx[:, 50:] == 0xFFFFFFFF).all()
    assert np.allclose(r2, np.float32(10.0) * np.float32(10.0))
    t = oracle_mod.KdTree(empty)
    assert (t.knn(q.pos, 3, 1.0)[2] == 0).all()


@pytest.mark.parametrize("filt", ["box", "cone", "epanechnikov"])
def test_radiance_fp64_matches_numpy(oracle_mod, filt):
    ph, q = _small_case(900, 80, seed=41)
    k, r = 30, 0.25
    idx, d2, cnt, r2 = oracle_mod.knn_brute(ph.pos, q.pos, k, r)
    ck = float(np.float32(1.1)) if filt == "cone" else 1.0   # the C ABI passes k_c as FP32
    a = oracle_mod.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt, ck, 8)
    b = np_restate.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt, ck, 8)
    assert np.allclose(a, b, rtol=1e-12, atol=0)
    assert (a > 0).any()


@pytest.mark.parametrize("n", [1, 33, 1000, 20011])
def test_kdtree_multithreaded_build_matches_sequential(oracle_mod, n):
    """The CPU baseline's multithreaded build makes the same splits: the same
    tree order of the points and the same exact kNN answers."""
    from mnrt_b200 import gen
    ph = gen.photons(n, seed=70 + n, caustic_frac=0.3)
    q = gen.queries(300, seed=71)
    a, b = oracle_mod.KdTree(ph.pos), oracle_mod.KdTree(ph.pos, threads=4)
    assert np.array_equal(a.order(), b.order())
    for x, y in zip(a.knn(q.pos, 24, 0.15, threads=2), b.knn(q.pos, 24, 0.15, threads=2)):
        assert np.array_equal(x, y)
