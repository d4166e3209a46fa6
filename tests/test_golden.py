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
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "reference_ingest")


def load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {key: z[key] for key in z.files}


def test_fixtures_present():
    assert len(CASES) >= 3 and (GOLDEN / "reference_ingest.npz").exists()


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
