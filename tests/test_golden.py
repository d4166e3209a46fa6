"""The oracle against the committed golden fixtures (CPU, no GPU).

The fixtures in tests/golden/ are written by tests/golden/make_golden.py from
the C++ oracle and the numpy restatement together; these tests pin the oracle
(brute force and kd-tree CPU baseline) to them bit for bit, so any drift of
the checker shows up here before it can hide a GPU parity failure.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "reference_ingest" and not p.stem.startswith("adjoint"))


def load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {key: z[key] for key in z.files}


def test_fixtures_present():
    assert len(CASES) >= 3 and (GOLDEN / "reference_ingest.npz").exists()
    assert (GOLDEN / "adjoint_k16_r025.npz").exists()


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(oracle_mod, name):
    g = load(name)
    k, r = int(g["k"]), float(g["r_max"])
    for res in (oracle_mod.knn_brute(g["pos"], g["qpos"], k, r), oracle_mod.KdTree(g["pos"]).knn(g["qpos"], k, r)):
        idx, d2, cnt, r2 = res
        assert np.array_equal(idx, g["idx"])
        assert np.array_equal(d2, g["d2"])
        assert np.array_equal(cnt, g["count"])
        assert np.array_equal(r2, g["r2"])
    for filt in ("box", "cone", "epanechnikov"):
        rad = oracle_mod.radiance_fp64(g["pos"], g["pow"], g["qpos"], g["qnrm"], g["idx"], g["count"], k, r, filt)
        assert np.allclose(rad, g[f"rad_{filt}"], rtol=1e-12, atol=0), filt


def test_oracle_reproduces_ingest_golden(oracle_mod):
    g = load("reference_ingest")
    _, pw = oracle_mod.pack_reference(g["pos"], g["pow"])
    assert np.array_equal(pw[:, 3].view(np.uint32), g["oct_bits"])


@pytest.mark.parametrize("filt", ["box", "cone", "epanechnikov"])
def test_oracle_reproduces_adjoint_golden(oracle_mod, filt):
    """The oracle's FP64 adjoint (dL/dpower, dL/dposition) against the fixture
    written where it agreed with the independent numpy restatement."""
    g = load("adjoint_k16_r025")
    k, r = int(g["k"]), float(g["r_max"])
    idx, _d2, cnt, _r2 = oracle_mod.knn_brute(g["pos"], g["qpos"], k, r)
    assert np.array_equal(idx, g["idx"]) and np.array_equal(cnt, g["count"])
    gp, gx = oracle_mod.backward_fp64(g["pos"], g["pow"], g["qpos"], g["qnrm"], idx, cnt, k, r,
                                      g[f"g_{filt}"].astype(np.float64), filt)
    for got, want in ((gp, g[f"gpow_{filt}"]), (gx, g[f"gpos_{filt}"])):
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
        assert np.abs(want).max() > 0
