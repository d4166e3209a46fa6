"""Second, independent restatement of the estimate in numpy (small cases only).

Used to cross-check the C++ oracle, whose parity against the reference is
unpinned.  Follows the same sources (paths inside jonike/mnrt):
GPU/photon_knn.cu:113-235 (strict d^2 < r^2, front test, r^2 rule) and
:518-519 (min_found).
"""
from __future__ import annotations

import numpy as np

from mnrt_b200.gen import oct_decode


def d2_f32(q: np.ndarray, p: np.ndarray) -> np.ndarray:
    """(nq, n) FP32 squared distances with the engine's operation order."""
    q = q[:, None, :3].astype(np.float32)
    p = p[None, :, :3].astype(np.float32)
    dx = (p[..., 0] - q[..., 0]).astype(np.float32)
    dy = (p[..., 1] - q[..., 1]).astype(np.float32)
    dz = (p[..., 2] - q[..., 2]).astype(np.float32)
    xx, yy, zz = dx * dx, dy * dy, dz * dz
    return ((xx + yy).astype(np.float32) + zz).astype(np.float32)


def knn(pos4: np.ndarray, q4: np.ndarray, k: int, r_max: float):
    r2max = np.float32(r_max) * np.float32(r_max)
    d2 = d2_f32(q4, pos4)
    nq, n = d2.shape
    idx = np.full((nq, k), 0xFFFFFFFF, np.uint32)
    dd = np.full((nq, k), np.inf, np.float32)
    cnt = np.zeros(nq, np.uint32)
    r2 = np.full(nq, r2max, np.float32)
    ar = np.arange(n)
    for q in range(nq):
        m = d2[q] < r2max
        cand = ar[m]
        order = np.lexsort((cand, d2[q][m]))   # by d2, then index
        sel = cand[order][:k]
        c = len(sel)
        idx[q, :c] = sel
        dd[q, :c] = d2[q][sel]
        cnt[q] = c
        if c == k:
            r2[q] = d2[q][sel[-1]]
    return idx, dd, cnt, r2


def front(n4: np.ndarray, dirbits: np.ndarray) -> np.ndarray:
    d = oct_decode(dirbits)
    a = (n4[:, 0].astype(np.float32) * -d[:, 0]).astype(np.float32)
    b = (n4[:, 1].astype(np.float32) * -d[:, 1]).astype(np.float32)
    c = (n4[:, 2].astype(np.float32) * -d[:, 2]).astype(np.float32)
    return ((a + b).astype(np.float32) + c) > 0


def radiance_fp64(pos4, pow4, q4, n4, nbr, cnt, k, r_max, filt="box", cone_k=1.0, min_found=0):
    nq = q4.shape[0]
    out = np.zeros((nq, 3))
    dirbits = pow4[:, 3].view(np.uint32)
    for q in range(nq):
        c = int(cnt[q])
        r2 = float(np.float64(np.float32(r_max)) ** 2)   # R is an FP32 parameter of the C ABI
        if c == k:
            dv = pos4[nbr[q, k - 1], :3].astype(np.float64) - q4[q, :3].astype(np.float64)
            r2 = float(dv @ dv)
        if c < min_found or not r2 > 0:
            continue
        sel = nbr[q, :c].astype(np.int64)
        fr = front(np.repeat(n4[q:q + 1], c, axis=0), dirbits[sel])
        dv = pos4[sel, :3].astype(np.float64) - q4[q, :3].astype(np.float64)
        d2 = (dv * dv).sum(1)
        if filt == "cone":
            w = 1.0 - np.sqrt(d2) / (cone_k * np.sqrt(r2))
            norm = 1.0 / ((1.0 - 2.0 / (3.0 * cone_k)) * np.pi * r2)
        elif filt == "epanechnikov":
            w = 1.0 - d2 / r2
            norm = 2.0 / (np.pi * r2)
        else:
            w = np.ones_like(d2)
            norm = 1.0 / (np.pi * r2)
        out[q] = ((w * fr)[:, None] * pow4[sel, :3].astype(np.float64)).sum(0) * norm
    return out
