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



def backward_fp64(pos4, pow4, q4, n4, nbr, cnt, k, r_max, grad, filt="box", cone_k=1.0, min_found=0):
    """dL/dpower and dL/dposition (n, 3) of L given dL/dE (grad, (nq, 3)) for
    the estimate E_q = norm(r2_q) * sum_p f_qp w(d2_qp, r2_q) power_p, where
    r2_q is the k-th neighbour's d2 (a function of its position) when k were
    found, else R^2.  Derived from that formula: dE/dpower_p = norm f w;
    dE/dx_p = norm f power_p dw/dd2 * 2 (x_p - q), plus, for the k-th
    neighbour, (dnorm/dr2 S + norm sum_p' f power_p' dw/dr2) * 2 (x_k - q)."""
    n = pos4.shape[0]
    gpow = np.zeros((n, 3))
    gpos = np.zeros((n, 3))
    dirbits = pow4[:, 3].view(np.uint32)
    kc = float(np.float32(cone_k))
    for q in range(q4.shape[0]):
        c = int(cnt[q])
        qp = q4[q, :3].astype(np.float64)
        if not np.isfinite(qp).all():
            continue
        r2 = float(np.float64(np.float32(r_max)) ** 2)
        if c == k:
            dv = pos4[nbr[q, k - 1], :3].astype(np.float64) - qp
            r2 = float(dv @ dv)
        if c == 0 or c < min_found or not r2 > 0:
            continue
        sel = nbr[q, :c].astype(np.int64)
        fr = front(np.repeat(n4[q:q + 1], c, axis=0), dirbits[sel]).astype(np.float64)
        dx = pos4[sel, :3].astype(np.float64) - qp
        d2 = (dx * dx).sum(1)
        phi = pow4[sel, :3].astype(np.float64)
        if filt == "cone":
            d, r = np.sqrt(d2), np.sqrt(r2)
            w = 1.0 - d / (kc * r)
            dw_dd2 = np.where(d > 0, -1.0 / (2.0 * kc * np.where(d > 0, d, 1.0) * r), 0.0)
            dw_dr2 = d / (2.0 * kc * r2 * r)
            norm = 1.0 / ((1.0 - 2.0 / (3.0 * kc)) * np.pi * r2)
        elif filt == "epanechnikov":
            w, dw_dd2, dw_dr2 = 1.0 - d2 / r2, np.full_like(d2, -1.0 / r2), d2 / (r2 * r2)
            norm = 2.0 / (np.pi * r2)
        else:
            w, dw_dd2, dw_dr2 = np.ones_like(d2), np.zeros_like(d2), np.zeros_like(d2)
            norm = 1.0 / (np.pi * r2)
        g = grad[q].astype(np.float64)
        np.add.at(gpow, sel, (fr * w)[:, None] * (norm * g)[None, :])
        coef = fr * dw_dd2 * norm * (phi @ g)
        if c == k:
            S = ((fr * w)[:, None] * phi).sum(0)
            T = ((fr * dw_dr2)[:, None] * phi).sum(0)
            coef[k - 1] += g @ (-norm / r2 * S + norm * T)
        np.add.at(gpos, sel, 2.0 * coef[:, None] * dx)
    return gpow, gpos

# ---------------------------------------------------------------------------
# Illumination cuts (GPU/illumcut.cu, PhotonMap.cpp:287-452,
# GPU/photon_knn.cu:338-433) on a tree in the engine's node layout.  This
# restatement uses the closed form of the cover pass (a slot's cover is the OR
# of the marks on its path below the root) that the engine's kernel uses; the
# C++ oracle runs the reference's literal level loop, so the two check each
# other.

KINV = 0xFFFFFFFF
F32 = np.float32


def median_tree(pos4: np.ndarray, leaf: int):
    """A binary tree in the engine's layout (node 0 = super-root whose slot 0
    is the root; nodes as 16 uint32 = two slots {lo xyz, hi xyz, ref, cnt})
    over pos4: split at the median of the box's longest axis until a slot
    holds at most `leaf` photons.  Returns (nodes, order): tree position i
    holds photon order[i]."""
    order: list[int] = []
    nodes: list = [None]

    def slot_of(ids):
        pts = pos4[ids, :3].astype(np.float32)
        lo, hi = pts.min(0), pts.max(0)
        if len(ids) <= leaf:
            first = len(order)
            order.extend(int(i) for i in ids)
            return (lo, hi, first, len(ids))
        j = len(nodes)
        nodes.append(None)
        a = int(np.argmax(hi - lo))
        srt = ids[np.argsort(pos4[ids, a], kind="stable")]
        h = len(srt) // 2
        nodes[j] = (slot_of(srt[:h]), slot_of(srt[h:]))
        return (lo, hi, j, 0)

    root = slot_of(np.arange(pos4.shape[0]))
    empty = (np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32), KINV, 0)
    nodes[0] = (root, empty)
    out = np.zeros((len(nodes), 16), np.uint32)
    for j, (s0, s1) in enumerate(nodes):
        for side, (lo, hi, ref, cnt) in enumerate((s0, s1)):
            w = out[j, 8 * side: 8 * side + 8]
            w[0:3] = np.asarray(lo, np.float32).view(np.uint32)
            w[3:6] = np.asarray(hi, np.float32).view(np.uint32)
            w[6], w[7] = ref, cnt
    return out, np.asarray(order, np.int64)


def _slot(nodes, sid):
    w = nodes[sid >> 1, 8 * (sid & 1): 8 * (sid & 1) + 8]
    return w[0:3].view(np.float32), w[3:6].view(np.float32), int(w[6]), int(w[7])


def _butterfly(p):
    p = [F32(v) for v in p]
    for o in (16, 8, 4, 2, 1):
        p = [F32(p[l] + p[l ^ o]) for l in range(32)]
    return p[0]


def _dot3(a, b):
    return F32(F32(F32(a[0] * b[0]) + F32(a[1] * b[1])) + F32(a[2] * b[2]))


def icut_slots(nodes):
    """level (KINV for empty slots), first, end, center (ns, 4)."""
    ns = 2 * nodes.shape[0]
    level = np.full(ns, KINV, np.uint32)
    first = np.zeros(ns, np.uint32)
    end = np.zeros(ns, np.uint32)
    center = np.zeros((ns, 4), np.float32)
    if _slot(nodes, 0)[2] == KINV:
        return level, first, end, center
    stack = [(0, 0)]
    while stack:
        sid, lvl = stack.pop()
        lo, hi, ref, cnt = _slot(nodes, sid)
        level[sid] = lvl
        e = [F32(hi[a] - lo[a]) for a in range(3)]
        for a in range(3):
            center[sid, a] = F32(lo[a] + F32(F32(0.5) * e[a]))
        center[sid, 3] = max(e[0], max(e[1], e[2]))
        if cnt > 0:
            first[sid], end[sid] = ref, ref + cnt
            continue
        j = ref   # leftmost and rightmost leaves
        while _slot(nodes, 2 * j)[3] == 0:
            j = _slot(nodes, 2 * j)[2]
        first[sid] = _slot(nodes, 2 * j)[2]
        j = ref
        while _slot(nodes, 2 * j + 1)[3] == 0:
            j = _slot(nodes, 2 * j + 1)[2]
        _, _, r1, c1 = _slot(nodes, 2 * j + 1)
        end[sid] = r1 + c1
        stack.append((2 * ref, lvl + 1))
        stack.append((2 * ref + 1, lvl + 1))
    return level, first, end, center


def icut_normals(tpow4, first, end):
    ns = len(first)
    normal = np.zeros((ns, 4), np.float32)
    d = oct_decode(tpow4[:, 3].copy().view(np.uint32)).astype(np.float32)
    for s in range(ns):
        cnt = int(end[s]) - int(first[s])
        p = [[F32(0)] * 32 for _ in range(3)]
        if 0 < cnt < 5000:
            for i in range(int(first[s]), int(end[s])):
                l = (i - int(first[s])) & 31
                ln = F32(np.sqrt(_dot3(d[i], d[i])))
                if ln > 0:
                    for a in range(3):
                        p[a][l] = F32(p[a][l] - F32(d[i, a] / ln))
        v = [_butterfly(p[a]) for a in range(3)]
        ln = F32(np.sqrt(_dot3(v, v)))
        if ln > 0:
            normal[s, :3] = [F32(v[a] / ln) for a in range(3)]
    return normal


def icut_estimate(tpow4, first, end, center, normal):
    ns = len(first)
    est = np.zeros((ns, 4), np.float32)
    fr_bits = tpow4[:, 3].copy().view(np.uint32)
    for s in range(ns):
        cnt = int(end[s]) - int(first[s])
        n = normal[s]
        if not (0 < cnt < 5000 and _dot3(n, n) > 0):
            continue
        idx = np.arange(int(first[s]), int(end[s]))
        fr = front(np.repeat(n[None], len(idx), 0), fr_bits[idx])
        p = [[F32(0)] * 32 for _ in range(3)]
        for t, i in enumerate(idx):
            if fr[t]:
                for a in range(3):
                    p[a][t & 31] = F32(p[a][t & 31] + tpow4[i, a])
        side = center[s, 3]
        if side > 0:
            a2 = F32(side * side)
            est[s, :3] = [F32(_butterfly(p[a]) / a2) for a in range(3)]
    return est


def icut_coarse(nodes, level, est, use_leafs, level_emin):
    ns = 2 * nodes.shape[0]
    valid = level != KINV
    leaf = np.array([_slot(nodes, s)[3] > 0 for s in range(ns)]) & valid
    if use_leafs:
        return leaf.astype(np.uint32), None
    on = valid & (level == level_emin) & ~np.all(est[:, :3] == 0, axis=1)
    if not on.any():
        emin = np.full(3, np.inf, np.float32)
    else:
        emin = np.zeros(3, np.float32)
        for a in range(3):
            mx = np.abs(est[on, a]).max()
            if mx > 0:
                scale = 1099511627776.0 / float(mx)
                tot = sum(int(np.rint(float(v) * scale)) for v in est[on, a])
                emin[a] = F32((float(tot) / scale) / float(on.sum()))
    m0 = valid & np.all(est[:, :3] >= emin, axis=1)
    m = m0.copy()
    for s in range(ns):
        lo, hi, ref, cnt = _slot(nodes, s)
        if valid[s] and cnt == 0 and m0[2 * ref] == m0[2 * ref + 1]:
            m[s] = False
    pslot = {1: 0}
    for j in range(1, nodes.shape[0]):
        for side in range(2):
            _, _, ref, cnt = _slot(nodes, 2 * j + side)
            if ref != KINV and cnt == 0:
                pslot[ref] = 2 * j + side
    coarse = np.zeros(ns, np.uint32)
    for s in range(ns):
        if not valid[s]:
            continue
        if s == 0:
            coarse[s] = 1 if leaf[s] else int(m[0])
            continue
        cov, p = False, pslot[s >> 1]
        while p != 0:
            cov = cov or bool(m[p])
            p = pslot[p >> 1]
        coarse[s] = (0 if cov else 1) if leaf[s] else int(m[s] and not cov)
    return coarse, emin


def icut_final(nodes, coarse, est, exact, iters, accuracy):
    ns = 2 * nodes.shape[0]
    work = coarse.astype(bool)
    fin = np.zeros(ns, bool)
    acc = F32(accuracy)
    for _ in range(iters):
        nxt = np.zeros(ns, bool)
        for s in np.nonzero(work)[0]:
            _, _, ref, cnt = _slot(nodes, int(s))
            ok = cnt > 0 or all(abs(F32(est[s, a] - exact[s, a])) < F32(acc * exact[s, a]) for a in range(3))
            if ok:
                fin[s] = True
            else:
                nxt[2 * ref] = nxt[2 * ref + 1] = True
        work = nxt
    return (fin | work).astype(np.uint32)


def icut_interp(nodes, fin, center, normal, exact, q4, n4, r_max):
    r2 = F32(F32(r_max) * F32(r_max))
    out = np.zeros((q4.shape[0], 3))
    reached = np.zeros(q4.shape[0], np.uint32)
    for qi in range(q4.shape[0]):
        q, qn = q4[qi, :3].astype(np.float32), n4[qi, :3].astype(np.float32)
        acc, ws = np.zeros(3), 0.0
        todo = [0]
        while todo:
            sid = todo.pop()
            lo, hi, ref, cnt = _slot(nodes, sid)
            if ref == KINV:
                continue
            g = [max(max(F32(lo[a] - q[a]), F32(q[a] - hi[a])), F32(0)) for a in range(3)]
            if not (_dot3(g, g) < r2):
                continue
            if cnt == 0 and not fin[sid]:
                todo += [2 * ref, 2 * ref + 1]
                continue
            nn = normal[sid]
            if _dot3(nn, nn) == 0 or not center[sid, 3] > 0:
                continue
            dq = [F32(center[sid, a] - q[a]) for a in range(3)]
            t = F32(F32(np.sqrt(_dot3(dq, dq))) / center[sid, 3])
            rbf = F32(F32(1) - F32(t * t)) if t <= 1 else F32(0)
            w = F32(rbf * max(F32(0), _dot3(nn, qn)))
            if w == 0:
                continue
            reached[qi] += 1
            acc += float(w) * exact[sid, :3].astype(np.float64)
            ws += float(w)
        if ws != 0.0:
            out[qi] = acc / ws
    return out, reached
