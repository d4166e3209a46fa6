"""ctypes wrapper of the CPU oracle (oracle/pm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs.  The engine never imports it.
Parity is unpinned (the reference ships no golden vectors and cannot be
compiled here); see the header of pm_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_lib = None


def _build() -> None:
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    src = HERE / "pm_oracle.cpp"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        _build()
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    u32, f32, i32 = C.c_uint32, C.c_float, C.c_int
    sig = {
        "orc_version": (i32, []),
        "orc_d2": (f32, [f32] * 6),
        "orc_oct_encode": (u32, [f32, f32, f32]),
        "orc_oct_decode": (None, [u32, P]),
        "orc_front": (i32, [f32, f32, f32, u32]),
        "orc_sincos": (None, [C.c_double, P]),
        "orc_spherical_to_oct": (u32, [f32, f32]),
        "orc_pack_reference_photons": (None, [P, P, u32, P, P]),
        "orc_knn_brute": (None, [P, u32, P, u32, u32, f32, P, P, P, P, i32]),
        "orc_kdtree_build": (P, [P, u32]),
        "orc_kdtree_build_mt": (P, [P, u32, C.c_int]),
        "orc_kdtree_order": (None, [P, P]),
        "orc_kdtree_free": (None, [P]),
        "orc_knn_kdtree": (None, [P, P, u32, u32, f32, P, P, P, P, i32]),
        "orc_radiance_fp64": (None, [P, P, P, P, u32, P, P, u32, f32, i32, f32, u32, P, i32]),
        "orc_compat": (None, [P, u32, P, P, P, P, u32, u32, f32, u32, i32, f32, u32, P, P, P, P, i32]),
        "orc_backward_fp64": (None, [P, P, P, P, u32, u32, P, P, u32, f32, i32, f32, u32, P, P, P]),
        "orc_icut_slots": (None, [P, u32, P, P, P, P]),
        "orc_icut_normals": (None, [P, u32, P, P, P]),
        "orc_icut_estimate": (None, [P, u32, P, P, P, P, P]),
        "orc_icut_coarse": (None, [P, u32, P, P, i32, u32, P, P]),
        "orc_icut_final": (None, [P, u32, P, P, P, u32, f32, P]),
        "orc_icut_interp": (None, [P, u32, P, P, P, P, P, P, u32, f32, P, P, i32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _c(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def pack_reference(pos4: np.ndarray, pow4: np.ndarray):
    """Reference-layout photons -> packed records (pos.w = index, pow.w = oct)."""
    lib = load()
    pos4, pow4 = _c(pos4, np.float32), _c(pow4, np.float32)
    n = pos4.shape[0]
    op = np.empty_like(pos4)
    ow = np.empty_like(pow4)
    lib.orc_pack_reference_photons(pos4.ctypes.data, pow4.ctypes.data, n, op.ctypes.data, ow.ctypes.data)
    return op, ow


def knn_brute(pos4, q4, k: int, r_max: float, threads: int = 0):
    """Exact kNN by definition.  Returns (idx (nq,k) uint32, d2 (nq,k), count (nq,), r2 (nq,))."""
    lib = load()
    pos4, q4 = _c(pos4, np.float32), _c(q4, np.float32)
    n, nq = pos4.shape[0], q4.shape[0]
    idx = np.empty((nq, k), np.uint32)
    d2 = np.empty((nq, k), np.float32)
    cnt = np.empty(nq, np.uint32)
    r2 = np.empty(nq, np.float32)
    lib.orc_knn_brute(pos4.ctypes.data, n, q4.ctypes.data, nq, k, r_max, idx.ctypes.data, d2.ctypes.data,
                      cnt.ctypes.data, r2.ctypes.data, threads)
    return idx, d2, cnt, r2


class KdTree:
    """The CPU baseline: median-split point kd-tree + bounded-heap kNN."""

    def __init__(self, pos4: np.ndarray, threads: int = 1):
        """threads = 1: the sequential build; otherwise the top levels' halves
        build on their own threads (0 = every hardware thread), same tree."""
        self._lib = load()
        self._pos = _c(pos4, np.float32)
        if threads == 1:
            self._h = self._lib.orc_kdtree_build(self._pos.ctypes.data, self._pos.shape[0])
        else:
            self._h = self._lib.orc_kdtree_build_mt(self._pos.ctypes.data, self._pos.shape[0], int(threads))

    def order(self) -> np.ndarray:
        """Caller indices of the points in tree order."""
        out = np.empty(self._pos.shape[0], np.uint32)
        self._lib.orc_kdtree_order(self._h, out.ctypes.data)
        return out

    def knn(self, q4, k: int, r_max: float, threads: int = 0):
        q4 = _c(q4, np.float32)
        nq = q4.shape[0]
        idx = np.empty((nq, k), np.uint32)
        d2 = np.empty((nq, k), np.float32)
        cnt = np.empty(nq, np.uint32)
        r2 = np.empty(nq, np.float32)
        self._lib.orc_knn_kdtree(self._h, q4.ctypes.data, nq, k, r_max, idx.ctypes.data, d2.ctypes.data,
                                 cnt.ctypes.data, r2.ctypes.data, threads)
        return idx, d2, cnt, r2

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_kdtree_free(self._h)
            self._h = None


FILTER_IDS = {"box": 0, "cone": 1, "epanechnikov": 2}


def radiance_fp64(pos4, pow4, q4, n4, nbr, count, k: int, r_max: float, filt: str = "box", cone_k: float = 1.0,
                  min_found: int = 0, threads: int = 0) -> np.ndarray:
    """FP64 estimate over the given neighbour sets; (nq, 3) float64."""
    lib = load()
    pos4, pow4, q4, n4 = (_c(a, np.float32) for a in (pos4, pow4, q4, n4))
    nbr, count = _c(nbr, np.uint32), _c(count, np.uint32)
    nq = q4.shape[0]
    out = np.empty((nq, 3), np.float64)
    lib.orc_radiance_fp64(pos4.ctypes.data, pow4.ctypes.data, q4.ctypes.data, n4.ctypes.data, nq, nbr.ctypes.data,
                          count.ctypes.data, k, r_max, FILTER_IDS[filt], cone_k, min_found, out.ctypes.data, threads)
    return out


def backward_fp64(pos4, pow4, q4, n4, nbr, count, k: int, r_max: float, grad, filt: str = "box",
                  cone_k: float = 1.0, min_found: int = 0):
    """FP64 host reference gradient of L given dL/dE (grad, (nq, 3)): returns
    (dL/dpower (n, 3), dL/dposition (n, 3)) for the given neighbour sets."""
    lib = load()
    pos4, pow4, q4, n4 = (_c(a, np.float32) for a in (pos4, pow4, q4, n4))
    nbr, count = _c(nbr, np.uint32), _c(count, np.uint32)
    grad = _c(grad, np.float64)
    n, nq = pos4.shape[0], q4.shape[0]
    gp = np.empty((n, 3), np.float64)
    gx = np.empty((n, 3), np.float64)
    lib.orc_backward_fp64(pos4.ctypes.data, pow4.ctypes.data, q4.ctypes.data, n4.ctypes.data, n, nq, nbr.ctypes.data,
                          count.ctypes.data, k, r_max, FILTER_IDS[filt], cone_k, min_found, grad.ctypes.data,
                          gp.ctypes.data, gx.ctypes.data)
    return gp, gx


def compat(nodes, tpos4, tpow4, q4, n4, k: int, r_max: float, iters: int = 2, filt: str = "box",
           cone_k: float = 1.0, min_found: int = 0, threads: int = 0):
    """ZHOU_COMPAT answer on an exported tree: (radius, count, r2_used, rad (nq, 3) FP64)."""
    lib = load()
    nodes = _c(nodes, np.uint32)
    tpos4, tpow4, q4, n4 = (_c(a, np.float32) for a in (tpos4, tpow4, q4, n4))
    nq = q4.shape[0]
    radius = np.empty(nq, np.float32)
    count = np.empty(nq, np.uint32)
    r2 = np.empty(nq, np.float32)
    rad = np.empty((nq, 3), np.float64)
    lib.orc_compat(nodes.ctypes.data, nodes.shape[0] - 1, tpos4.ctypes.data, tpow4.ctypes.data, q4.ctypes.data,
                   n4.ctypes.data, nq, k, r_max, iters, FILTER_IDS[filt], cone_k, min_found, radius.ctypes.data,
                   count.ctypes.data, r2.ctypes.data, rad.ctypes.data, threads)
    return radius, count, r2, rad


def icut(nodes, tpow4, use_leafs: bool = True, level_emin: int = 12, normals=None):
    """Illumination-cut slot records and coarse cut on an exported tree.

    Returns a dict: level, first, end, center (ns, 4), normal (ns, 4) (the
    given normals, or the photon-derived ones), est (ns, 4), coarse, emin."""
    lib = load()
    nodes = _c(nodes, np.uint32)
    tpow4 = _c(tpow4, np.float32)
    m = nodes.shape[0] - 1
    ns = 2 * (m + 1)
    level = np.empty(ns, np.uint32)
    first = np.empty(ns, np.uint32)
    end = np.empty(ns, np.uint32)
    center = np.empty((ns, 4), np.float32)
    lib.orc_icut_slots(nodes.ctypes.data, m, level.ctypes.data, first.ctypes.data, end.ctypes.data, center.ctypes.data)
    if normals is None:
        normal = np.empty((ns, 4), np.float32)
        lib.orc_icut_normals(tpow4.ctypes.data, ns, first.ctypes.data, end.ctypes.data, normal.ctypes.data)
    else:
        normal = _c(normals, np.float32).copy()
        normal[:, 3] = 0.0
    est = np.empty((ns, 4), np.float32)
    lib.orc_icut_estimate(tpow4.ctypes.data, ns, first.ctypes.data, end.ctypes.data, center.ctypes.data,
                          normal.ctypes.data, est.ctypes.data)
    coarse = np.empty(ns, np.uint32)
    emin = np.full(3, np.nan, np.float32)
    lib.orc_icut_coarse(nodes.ctypes.data, m, level.ctypes.data, est.ctypes.data, int(bool(use_leafs)), level_emin,
                        coarse.ctypes.data, emin.ctypes.data)
    return {"level": level, "first": first, "end": end, "center": center, "normal": normal, "est": est,
            "coarse": coarse, "emin": emin}


def icut_final(nodes, coarse, est4, exact4, iters: int = 4, accuracy: float = 0.2):
    """Final cut marks from a coarse cut and the node-centre irradiance."""
    lib = load()
    nodes = _c(nodes, np.uint32)
    coarse = _c(coarse, np.uint32)
    est4, exact4 = _c(est4, np.float32), _c(exact4, np.float32)
    m = nodes.shape[0] - 1
    fin = np.empty(2 * (m + 1), np.uint32)
    lib.orc_icut_final(nodes.ctypes.data, m, coarse.ctypes.data, est4.ctypes.data, exact4.ctypes.data, iters,
                       accuracy, fin.ctypes.data)
    return fin


def icut_interp(nodes, fin, center4, normal4, exact4, q4, n4, r_max: float, threads: int = 0):
    """Irradiance interpolated from a cut: (irr (nq, 3) FP64, cut slots of nonzero weight (nq,))."""
    lib = load()
    nodes, fin = _c(nodes, np.uint32), _c(fin, np.uint32)
    center4, normal4, exact4, q4, n4 = (_c(a, np.float32) for a in (center4, normal4, exact4, q4, n4))
    nq = q4.shape[0]
    out = np.empty((nq, 3), np.float64)
    reached = np.empty(nq, np.uint32)
    lib.orc_icut_interp(nodes.ctypes.data, nodes.shape[0] - 1, fin.ctypes.data, center4.ctypes.data,
                        normal4.ctypes.data, exact4.ctypes.data, q4.ctypes.data, n4.ctypes.data, nq, r_max,
                        out.ctypes.data, reached.ctypes.data, threads)
    return out, reached


def threads_available() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
