"""CPU: the oracle's FP64 reference gradient against FP64 central finite
differences (h = 1e-4) of the squared-error loss, for every filter.  This pins
the host gradient independently of the GPU; the GPU adjoint is then checked
against both (tests/test_gpu_backward.py)."""
import numpy as np
import pytest

from mnrt_b200 import gen
from tests.fd import LossFD

TOL = 1e-3   # relative, against FP64 central differences


def problem(oracle_mod, filt, n=3000, nq=1500, k=16, r=0.1, seed=60, min_found=0):
    ph = gen.photons(n, seed=seed, caustic_frac=0.2, caustic_sigma=0.02)
    q = gen.queries(nq, seed=seed + 1)
    idx, _d2, cnt, _r2 = oracle_mod.KdTree(ph.pos).knn(q.pos, k, r)
    e = oracle_mod.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, min_found)
    rng = np.random.default_rng(seed + 2)
    tpow = ph.pow.copy()
    tpow[:, :3] *= rng.uniform(0.5, 1.5, size=(n, 3)).astype(np.float32)
    t = oracle_mod.radiance_fp64(ph.pos, tpow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, min_found)
    g = 2.0 * (e - t)
    return ph, q, idx, cnt, t, g


def rel_err(a, b):
    floor = 1e-3 * max(np.abs(b).max(), 1e-300)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


@pytest.mark.parametrize("filt", ["box", "cone", "epanechnikov"])
def test_oracle_gradient_matches_finite_differences(oracle_mod, filt):
    k, r = 16, 0.1
    ph, q, idx, cnt, t, g = problem(oracle_mod, filt, k=k, r=r)
    gpow, gpos = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, g, filt)
    fd = LossFD(oracle_mod, ph.pos, ph.pow, q.pos, q.nrm, t, k, r, filt)
    rng = np.random.default_rng(5)
    # photons that are some query's k-th neighbour exercise the r^2 path
    kth = np.unique(idx[cnt == k, k - 1])
    sample = np.concatenate([rng.choice(ph.n, 30, replace=False), rng.choice(kth, 30, replace=False)])
    res = fd.position(sample)
    ok = ~res.excluded
    assert ok.sum() >= 0.8 * ok.size, f"{res.num_excluded} of {ok.size} samples excluded"
    err = rel_err(gpos[sample][ok], res.fd[ok])
    assert err.max() <= TOL, err.max()
    fp = fd.power(sample[:20])
    assert rel_err(gpow[sample[:20]], fp).max() <= TOL
    assert np.abs(gpos[sample]).max() > 0


def test_oracle_gradient_min_found_zeroes(oracle_mod):
    k, r = 16, 0.02
    ph, q, idx, cnt, t, g = problem(oracle_mod, "box", n=800, nq=300, k=k, r=r, min_found=8)
    gpow, gpos = oracle_mod.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, g, "box", 1.0, 8)
    # photons only used by queries below min_found get no gradient
    used = np.zeros(ph.n, bool)
    for qi in np.where(cnt >= 8)[0]:
        used[idx[qi, :cnt[qi]]] = True
    assert (gpow[~used] == 0).all() and (gpos[~used] == 0).all()
