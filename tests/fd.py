"""FP64 central finite differences of the squared-error loss through the
photon-map estimate (test infrastructure for the adjoint checks).

    L(x, Phi) = sum_q sum_c (E_qc - T_qc)^2

E follows the engine's contract: the neighbour set of a query is the k
photons with the smallest (FP32 d^2, index) below R^2, and the estimate over
that set is evaluated in FP64 (the oracle's radiance_fp64).  Moving one
photon p changes only the queries whose set contains p or could gain p, and
their new set is the k nearest among their old k + 1 nearest plus p, so each
finite difference re-evaluates a few hundred queries exactly instead of the
whole map.  The loss is evaluated in FP64 with the moved photon at an FP64
position (exact +-h steps); the neighbour sets are decided on the positions
rounded to FP32, as the engine sees them.  A sample whose neighbour set (or
k-th neighbour) changes inside [-h, +h] sits on a kink of L and is excluded;
the count is reported.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.spatial import cKDTree

from tests.np_restate import front


def _d2_f32(q: np.ndarray, p: np.ndarray) -> np.ndarray:
    """FP32 d^2 with the engine's operation order; q (m, 3), p (m, c, 3)."""
    q = q[:, None, :].astype(np.float32)
    p = p.astype(np.float32)
    dx = (p[..., 0] - q[..., 0]).astype(np.float32)
    dy = (p[..., 1] - q[..., 1]).astype(np.float32)
    dz = (p[..., 2] - q[..., 2]).astype(np.float32)
    return ((dx * dx + dy * dy).astype(np.float32) + dz * dz).astype(np.float32)


@dataclass
class FDResult:
    fd: np.ndarray          # (s, 3) finite differences (nan where excluded)
    excluded: np.ndarray    # (s, 3) bool
    num_excluded: int
    scale: np.ndarray = None   # (s,) smallest (k+1)-th neighbour distance of the queries the photon moves


class LossFD:
    def __init__(self, oracle_mod, pos4, pow4, q4, n4, target, k: int, r_max: float, filt: str, cone_k: float = 1.0,
                 min_found: int = 0):
        self.o = oracle_mod
        self.pos = np.ascontiguousarray(pos4, np.float32)
        self.pw = np.ascontiguousarray(pow4, np.float32)
        self.q = np.ascontiguousarray(q4, np.float32)
        self.n = np.ascontiguousarray(n4, np.float32)
        self.t = np.asarray(target, np.float64)
        self.k, self.R, self.filt, self.cone_k, self.min_found = k, r_max, filt, cone_k, min_found
        self.r2max = np.float32(r_max) * np.float32(r_max)
        idx, _d2, cnt, r2 = oracle_mod.KdTree(self.pos).knn(self.q, k + 1, r_max)
        self.idx1, self.cnt1 = idx, cnt
        self.rk = np.sqrt(r2.astype(np.float64))            # k+1-th distance bound (or R)
        self.qtree = cKDTree(self.q[:, :3].astype(np.float64))

    def _rows(self, qsel: np.ndarray, p: int, newpos: np.ndarray):
        """New k-NN rows (caller indices, -1 padded) and counts of queries qsel
        with photon p at newpos."""
        k = self.k
        cand = self.idx1[qsel].astype(np.int64)
        cand = np.where(cand == 0xFFFFFFFF, -1, cand)
        cand = np.where(cand == p, -1, cand)                 # p is re-added below
        cand = np.concatenate([cand, np.full((len(qsel), 1), p, np.int64)], axis=1)
        pts = np.where(cand[..., None] >= 0, self.pos[np.maximum(cand, 0), :3], np.float32(np.inf))
        pts[cand == p] = newpos
        d2 = _d2_f32(self.q[qsel, :3], pts)
        d2 = np.where(cand >= 0, d2, np.float32(np.inf))
        ok = d2 < self.r2max
        key_d = np.where(ok, d2, np.float32(np.inf))
        key_i = np.where(ok, cand, np.iinfo(np.int64).max)
        order = np.lexsort((key_i, key_d), axis=1)
        rows = np.take_along_axis(np.where(ok, cand, -1), order, axis=1)[:, :k]
        cnt = np.minimum(ok.sum(1), k)
        return rows, cnt

    def _loss(self, qsel, rows, cnt, p: int = -1, xp=None):
        """FP64 loss of the queries qsel over fixed neighbour rows, with photon
        p at the FP64 position xp (None: where it is)."""
        k = self.k
        valid = rows >= 0
        safe = np.where(valid, rows, 0)
        pts = self.pos[safe, :3].astype(np.float64)
        if xp is not None:
            pts[rows == p] = np.asarray(xp, np.float64)
        dv = pts - self.q[qsel, None, :3].astype(np.float64)
        d2 = (dv * dv).sum(-1)
        last = np.take_along_axis(d2, np.maximum(cnt - 1, 0)[:, None], axis=1)[:, 0]
        R2 = float(np.float64(np.float32(self.R))) ** 2
        r2 = np.where(cnt == k, last, R2)
        alive = (cnt > 0) & (cnt >= self.min_found) & (r2 > 0)
        r2s = np.where(alive, r2, 1.0)[:, None]
        if self.filt == "cone":
            w = 1.0 - np.sqrt(d2) / (self.cone_k * np.sqrt(r2s))
            norm = 1.0 / ((1.0 - 2.0 / (3.0 * self.cone_k)) * np.pi * r2s)
        elif self.filt == "epanechnikov":
            w = 1.0 - d2 / r2s
            norm = 2.0 / (np.pi * r2s)
        else:
            w = np.ones_like(d2)
            norm = 1.0 / (np.pi * r2s)
        nrm = np.repeat(self.n[qsel], rows.shape[1], axis=0)
        fr = front(nrm, self.pw[safe.ravel(), 3].view(np.uint32)).reshape(rows.shape)
        wt = np.where(valid & fr, w, 0.0)
        e = (wt[..., None] * self.pw[safe, :3].astype(np.float64)).sum(1) * norm
        e = np.where(alive[:, None], e, 0.0)
        return float(((e - self.t[qsel]) ** 2).sum())

    @staticmethod
    def _same_set(a, b, cnt_a, cnt_b, k):
        """Same neighbour sets and the same k-th neighbour (order inside a set
        does not move the estimate)."""
        if not np.array_equal(cnt_a, cnt_b):
            return False
        if not np.array_equal(np.sort(a, axis=1), np.sort(b, axis=1)):
            return False
        full = cnt_a == k
        return np.array_equal(a[full, k - 1], b[full, k - 1])

    def _affected(self, p: int, h: float) -> np.ndarray:
        x = self.pos[p, :3].astype(np.float64)
        near = np.array(self.qtree.query_ball_point(x, self.R + 2 * h), dtype=np.int64)
        if near.size == 0:
            return near
        dist = np.sqrt(((self.q[near, :3].astype(np.float64) - x) ** 2).sum(1))
        has_p = (self.idx1[near] == p).any(1)
        could_enter = dist - 2 * h < self.rk[near]
        return near[has_p | could_enter]

    def _central(self, p: int, qsel, base, a: int, h: float):
        """FP64 central difference along axis a with step h, or None if a
        neighbour set (or k-th neighbour) changes inside [-h, +h]; the sets are
        decided on the FP32-rounded positions, as the engine would see them."""
        rows0, cnt0 = base
        x = self.pos[p, :3].astype(np.float64)
        for sgn in (1.0, -1.0, 0.5, -0.5):
            y = x.copy()
            y[a] += sgn * h
            r, c = self._rows(qsel, p, y.astype(np.float32))
            if not self._same_set(r, rows0, c, cnt0, self.k):
                return None
        xp, xm = x.copy(), x.copy()
        xp[a] += h
        xm[a] -= h
        return (self._loss(qsel, rows0, cnt0, p, xp) - self._loss(qsel, rows0, cnt0, p, xm)) / (2.0 * h)

    def position(self, photons, h: float = 1e-4) -> FDResult:
        """dL/dx_p by FP64 central differences with step h and h/2, combined by
        Richardson extrapolation (4 D(h/2) - D(h)) / 3 (fourth order); plain
        D(h) is kept in .plain."""
        out = np.full((len(photons), 3), np.nan)
        plain = np.full((len(photons), 3), np.nan)
        excl = np.zeros((len(photons), 3), bool)
        scale = np.full(len(photons), np.inf)
        for s, p in enumerate(photons):
            p = int(p)
            qsel = self._affected(p, h)
            if qsel.size == 0:
                out[s] = plain[s] = 0.0
                continue
            scale[s] = self.rk[qsel].min()
            base = self._rows(qsel, p, self.pos[p, :3])
            for a in range(3):
                d1 = self._central(p, qsel, base, a, h)
                d2 = self._central(p, qsel, base, a, h / 2) if d1 is not None else None
                if d1 is None or d2 is None:
                    excl[s, a] = True
                    continue
                plain[s, a] = d1
                out[s, a] = (4.0 * d2 - d1) / 3.0
        r = FDResult(out, excl, int(excl.sum()), scale)
        r.plain = plain
        return r

    def power(self, photons, h: float = 1e-4) -> np.ndarray:
        """d L / d Phi_p by central differences (the sets do not depend on power)."""
        out = np.zeros((len(photons), 3))
        for s, p in enumerate(photons):
            qsel = self._affected(int(p), 0.0)
            if qsel.size == 0:
                continue
            rows, cnt = self._rows(qsel, int(p), self.pos[p, :3])
            for c in range(3):
                keep = self.pw.copy()
                scale = max(abs(float(keep[p, c])), 1e-12)
                dh = h * scale
                self.pw = keep.copy()
                self.pw[p, c] = keep[p, c] + dh
                up = float(self.pw[p, c])
                lp = self._loss(qsel, rows, cnt)
                self.pw[p, c] = keep[p, c] - dh
                dn = float(self.pw[p, c])
                lm = self._loss(qsel, rows, cnt)
                self.pw = keep
                out[s, c] = (lp - lm) / (up - dn)
        return out
