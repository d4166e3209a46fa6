"""Writes the golden fixtures in this folder (run from the repository root):

    python tests/golden/make_golden.py

The reference ships no golden vectors, known-answer tests or fixtures for the
photon-map path, so these are the project's own: seeded inputs of the small
configuration's shape (room photons, wall queries) with the expected exact
neighbour lists, counts, r^2 and FP64 radiance for the box, cone and
Epanechnikov filters, the FP64 adjoint (dL/dpower, dL/dposition of a
squared-error loss) for each filter, plus the packed direction bits of
reference-layout (azimuth / polar angle) photons.  Every expected array is
computed twice, by the C++ oracle (oracle/pm_oracle.cpp) and by the
independent numpy restatement (tests/np_restate.py); the script refuses to
write a fixture on which they disagree.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from mnrt_b200 import gen  # noqa: E402
from oracle import oracle  # noqa: E402
from tests import np_restate  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    # name: photons, queries, k, R, seeds, caustic fraction, duplicate pile
    "small_k50_r01": dict(n=2048, nq=256, k=50, r_max=0.1, seed=500, caustic=0.0, dup=False),
    "caustic_k16_r005": dict(n=3000, nq=200, k=16, r_max=0.05, seed=510, caustic=0.2, dup=True),
    "sparse_k128_r002": dict(n=1500, nq=128, k=128, r_max=0.02, seed=520, caustic=0.2, dup=False),
}


def make_case(name: str, c: dict) -> dict:
    ph = gen.photons(c["n"], seed=c["seed"], caustic_frac=c["caustic"], power_mean=1.0 / 65536)
    q = gen.queries(c["nq"], seed=c["seed"] + 1)
    if c["dup"]:   # coincident photons and queries on them: ties broken by index
        ph.pos[100:140, :3] = ph.pos[3, :3]
        q.pos[:6, :3] = ph.pos[3, :3]
    k, r = c["k"], c["r_max"]
    idx, d2, cnt, r2 = oracle.knn_brute(ph.pos, q.pos, k, r)
    nidx, nd2, ncnt, nr2 = np_restate.knn(ph.pos, q.pos, k, r)
    for a, b, what in ((idx, nidx, "idx"), (d2, nd2, "d2"), (cnt, ncnt, "count"), (r2, nr2, "r2")):
        if not np.array_equal(a, b):
            raise SystemExit(f"{name}: oracle and numpy restatement disagree on {what}")
    out = dict(pos=ph.pos, pow=ph.pow, qpos=q.pos, qnrm=q.nrm, k=np.uint32(k), r_max=np.float32(r),
               idx=idx, d2=d2, count=cnt, r2=r2)
    for filt in ("box", "cone", "epanechnikov"):
        a = oracle.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, 0)
        b = np_restate.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, 0)
        if not np.allclose(a, b, rtol=1e-12, atol=0):
            raise SystemExit(f"{name}: FP64 radiance ({filt}) disagrees")
        out[f"rad_{filt}"] = a
    return out


def make_adjoint() -> dict:
    """dL/dpower and dL/dposition for L = sum |E - T|^2, T the estimate of
    powers scaled by seeded U[0.5, 1.5] on the same neighbour sets."""
    ph = gen.photons(1024, seed=540, caustic_frac=0.2, power_mean=1.0 / 65536)
    q = gen.queries(128, seed=541)
    k, r = 16, 0.25
    idx, _d2, cnt, _r2 = oracle.knn_brute(ph.pos, q.pos, k, r)
    tpow = ph.pow.copy()
    tpow[:, :3] *= np.random.default_rng(542).uniform(0.5, 1.5, size=(ph.n, 3)).astype(np.float32)
    out = dict(pos=ph.pos, pow=ph.pow, qpos=q.pos, qnrm=q.nrm, k=np.uint32(k), r_max=np.float32(r), idx=idx,
               count=cnt)
    for filt in ("box", "cone", "epanechnikov"):
        e = oracle.radiance_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, 0)
        t = oracle.radiance_fp64(ph.pos, tpow, q.pos, q.nrm, idx, cnt, k, r, filt, 1.0, 0)
        g = (2.0 * (e - t)).astype(np.float32).astype(np.float64)   # dL/dE as the engine takes it, FP32
        a = oracle.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, g, filt, 1.0, 0)
        b = np_restate.backward_fp64(ph.pos, ph.pow, q.pos, q.nrm, idx, cnt, k, r, g, filt, 1.0, 0)
        for x, y, what in ((a[0], b[0], "power"), (a[1], b[1], "position")):
            if np.abs(x - y).max() > 1e-12 * np.abs(y).max():
                raise SystemExit(f"adjoint ({filt}, {what}): oracle and numpy restatement disagree")
        out[f"g_{filt}"], out[f"gpow_{filt}"], out[f"gpos_{filt}"] = g.astype(np.float32), a[0], a[1]
    return out


def make_ingest() -> dict:
    ph = gen.photons(512, seed=530, layout="reference")
    pos, pw = oracle.pack_reference(ph.pos, ph.pow)
    return dict(pos=ph.pos, pow=ph.pow, oct_bits=pw[:, 3].view(np.uint32).copy())


def main() -> int:
    for name, c in CASES.items():
        np.savez_compressed(OUT / f"{name}.npz", **make_case(name, c))
        print("wrote", name)
    np.savez_compressed(OUT / "reference_ingest.npz", **make_ingest())
    print("wrote reference_ingest")
    np.savez_compressed(OUT / "adjoint_k16_r025.npz", **make_adjoint())
    print("wrote adjoint_k16_r025")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
