"""Batches of photon maps over the C ABI (pm_batch_*): many maps of uneven
size built by one sort and one tree and queried by one persistent launch,
optionally recorded in a CUDA graph.  No counterpart in the reference, which
builds and gathers one map per call."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .photon_map import _ptr, _stream


def _offsets(x) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.uint32))
    if a.ndim != 1 or a.size < 2 or a[0] != 0:
        raise ValueError("offsets must be a 1-D array starting at 0 with num_maps + 1 entries")
    return a


def make_desc(k: int, r_max: float, filter="box", cone_k: float = 1.0, min_found: int = 0) -> L.QueryDesc:
    return L.QueryDesc(k=int(k), r_max=float(r_max), filter=L.FILTERS[filter] if isinstance(filter, str) else int(filter),
                       cone_k=float(cone_k), mode=L.PM_MODE_EXACT, min_found=int(min_found),
                       order=L.PM_ORDER_SORTED, refine_iters=2)


class PhotonMapBatch:
    def __init__(self):
        self._lib = L.load()
        h = C.c_void_p()
        st = self._lib.pm_batch_create(C.byref(h))
        if st != L.PM_OK:
            raise L.PMError(st, "pm_batch_create failed")
        self._h = h
        self._keep = []

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != L.PM_OK:
            raise L.PMError(st, self._lib.pm_batch_last_error(self._h).decode())

    def set_tuning(self, leaf_size: int = 32, warps_per_block: int = 4, rounds_per_chunk: int = 8,
                   wide: bool = True) -> None:
        """wide: traverse the 32-wide tree (else the binary one)."""
        self._check(self._lib.pm_batch_set_tuning(self._h, leaf_size, warps_per_block, rounds_per_chunk, int(wide)))

    def build(self, pos: torch.Tensor, pw: torch.Tensor, photon_offsets, packed: bool = True, stream=None) -> None:
        off = _offsets(photon_offsets)
        n = int(off[-1])
        fmt = L.PM_PHOTONS_PACKED if packed else L.PM_PHOTONS_REFERENCE
        self._check(self._lib.pm_batch_build(self._h, _ptr(pos) if n else None, _ptr(pw) if n else None,
                                             off.ctypes.data, off.size - 1, fmt, _stream(stream)))

    @staticmethod
    def _descs(descs):
        arr = (L.QueryDesc * len(descs))()
        for i, d in enumerate(descs):
            arr[i] = d if isinstance(d, L.QueryDesc) else make_desc(**d)
        return arr

    def outputs(self, descs, query_offsets, device, want_nbr: bool = False) -> dict:
        off = _offsets(query_offsets)
        nq = int(off[-1])
        out = {"rad": torch.empty((max(nq, 1), 4), dtype=torch.float32, device=device),
               "r2": torch.empty((max(nq, 1),), dtype=torch.float32, device=device),
               "count": torch.empty((max(nq, 1),), dtype=torch.int32, device=device)}
        if want_nbr:
            ks = [d.k if isinstance(d, L.QueryDesc) else d["k"] for d in descs]
            total = int(sum(int(off[i + 1] - off[i]) * int(ks[i]) for i in range(len(ks))))
            out["nbr"] = torch.empty((max(total, 1),), dtype=torch.int32, device=device)
        return out

    def query(self, descs, qpos: torch.Tensor, qnrm: torch.Tensor, query_offsets, want_nbr: bool = False,
              out: dict | None = None, stream=None) -> dict:
        off = _offsets(query_offsets)
        arr = self._descs(descs)
        if out is None:
            out = self.outputs(descs, off, qpos.device, want_nbr)
        self._check(self._lib.pm_batch_query(self._h, arr, _ptr(qpos), _ptr(qnrm), off.ctypes.data, _ptr(out["rad"]),
                                             _ptr(out.get("nbr")), _ptr(out.get("r2")), _ptr(out.get("count")),
                                             _stream(stream)))
        return out

    def capture(self, pos, pw, photon_offsets, descs, qpos, qnrm, query_offsets, out: dict, packed: bool = True):
        poff, qoff = _offsets(photon_offsets), _offsets(query_offsets)
        arr = self._descs(descs)
        self._keep = [poff, qoff, arr]
        fmt = L.PM_PHOTONS_PACKED if packed else L.PM_PHOTONS_REFERENCE
        self._check(self._lib.pm_batch_capture(self._h, _ptr(pos), _ptr(pw), poff.ctypes.data, poff.size - 1, fmt, arr,
                                               _ptr(qpos), _ptr(qnrm), qoff.ctypes.data, _ptr(out["rad"]),
                                               _ptr(out.get("nbr")), _ptr(out.get("r2")), _ptr(out.get("count"))))

    def autotune(self, pos, pw, photon_offsets, descs, qpos, qnrm, query_offsets, out: dict, packed: bool = True,
                 stream=None) -> L.Tuning:
        """Times build + query over leaf sizes, warps per block and rounds per
        chunk; keeps the fastest and leaves the batch built with it."""
        poff, qoff = _offsets(photon_offsets), _offsets(query_offsets)
        arr = self._descs(descs)
        best = L.Tuning()
        fmt = L.PM_PHOTONS_PACKED if packed else L.PM_PHOTONS_REFERENCE
        self._check(self._lib.pm_batch_autotune(self._h, _ptr(pos), _ptr(pw), poff.ctypes.data, poff.size - 1, fmt, arr,
                                                _ptr(qpos), _ptr(qnrm), qoff.ctypes.data, _ptr(out["rad"]),
                                                C.byref(best), _stream(stream)))
        return best

    def launch(self, stream=None) -> None:
        self._check(self._lib.pm_batch_launch(self._h, _stream(stream)))

    def info(self, stream=None) -> L.MapInfo:
        i = L.MapInfo()
        self._check(self._lib.pm_batch_get_info(self._h, C.byref(i), _stream(stream)))
        return i
