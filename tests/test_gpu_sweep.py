"""Randomized parity sweep: seeded random configurations (photon count,
caustic share, duplicated positions, query count and clustering, k, R,
filter, leaf size, k-buffer layout, queries per warp, rounds per chunk)
against the oracle, with the bars of test_gpu_parity (neighbour lists,
counts and r^2 bit-exact; radiance within 1e-5 of FP64).  Such a sweep found
a channel whose flux sat on the k-th neighbour; the case is pinned in
test_gpu_parity.test_channel_imbalanced_flux_small_k."""
import numpy as np
import pytest

from mnrt_b200 import gen
from tests.test_gpu_parity import check_against_oracle, run

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
