"""ctypes binding of the engine's C ABI (include/pmgpu.h).

The shared library is built in-tree by mnrt_b200.build.  Loading fails loudly
when it is missing: there is no CPU fallback anywhere in the engine.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpmgpu.so"

PM_OK, PM_ERR_INVALID, PM_ERR_CUDA, PM_ERR_OOM, PM_ERR_STATE, PM_ERR_DEVICE, PM_ERR_UNSUPPORTED = 0, -1, -2, -3, -4, -5, -6
PM_PHOTONS_REFERENCE, PM_PHOTONS_PACKED = 0, 1
PM_FILTER_BOX, PM_FILTER_CONE, PM_FILTER_EPANECHNIKOV = 0, 1, 2
PM_MODE_EXACT, PM_MODE_ZHOU_COMPAT, PM_MODE_ICUT = 0, 1, 2
PM_ORDER_SORTED, PM_ORDER_AS_GIVEN = 0, 1
PM_MAX_K = 128
PM_NOALLOC_MAX_QUERIES = 262144
PM_DEVERR_STACK, PM_DEVERR_NONFINITE, PM_DEVERR_QNONFINITE, PM_DEVERR_WAIT = 0x1, 0x2, 0x4, 0x8
PM_KBUF_HEAP, PM_KBUF_GROUP, PM_KBUF_WIDE = 0, 1, 2

FILTERS = {"box": PM_FILTER_BOX, "cone": PM_FILTER_CONE, "epanechnikov": PM_FILTER_EPANECHNIKOV}


class QueryDesc(C.Structure):
    _fields_ = [("k", C.c_uint32), ("r_max", C.c_float), ("filter", C.c_int), ("cone_k", C.c_float),
                ("mode", C.c_int), ("min_found", C.c_uint32), ("order", C.c_int), ("refine_iters", C.c_uint32)]


class IcutDesc(C.Structure):
    _fields_ = [("use_leafs", C.c_int), ("level_emin", C.c_uint32), ("refine_iters", C.c_uint32),
                ("accuracy", C.c_float)]


class MapInfo(C.Structure):
    _fields_ = [("num_photons", C.c_uint32), ("num_nodes", C.c_uint32), ("leaf_size", C.c_uint32),
                ("device_errors", C.c_uint32), ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3),
                ("max_power", C.c_float), ("launches", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("leaf_size", C.c_uint32), ("warps_per_block", C.c_int), ("rounds_per_chunk", C.c_int),
                ("queries_per_warp", C.c_int), ("kbuf_layout", C.c_int), ("build_ms", C.c_float),
                ("query_ms", C.c_float)]


class Timings(C.Structure):
    _fields_ = [("build_ms", C.c_float), ("build_sort_ms", C.c_float), ("query_ms", C.c_float),
                ("query_sort_ms", C.c_float), ("query_kernel_ms", C.c_float), ("build_launches", C.c_uint32),
                ("query_launches", C.c_uint32)]


ALLOC_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_void_p), C.c_size_t, C.c_void_p)
FREE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)

_VP, _FP, _UP = C.c_void_p, C.c_void_p, C.c_void_p
_U32, _I, _F = C.c_uint32, C.c_int, C.c_float

# name -> (restype, argtypes); every symbol declared in include/pmgpu.h
SIGNATURES = {
    "pm_create": (_I, [C.POINTER(C.c_void_p), _U32, C.POINTER(C.c_float), C.POINTER(C.c_float), _F]),
    "pm_destroy": (_I, [_VP]),
    "pm_set_allocator": (_I, [_VP, ALLOC_FN, FREE_FN, _VP]),
    "pm_set_tuning": (_I, [_VP, _U32, _I, _I, _I, _I]),
    "pm_reserve": (_I, [_VP, _U32, _U32]),
    "pm_autotune": (_I, [_VP, _FP, _FP, _U32, _I, C.POINTER(QueryDesc), _FP, _FP, _U32, _U32, C.POINTER(Tuning), _VP]),
    "pm_build": (_I, [_VP, _FP, _FP, _U32, _I, _VP]),
    "pm_query": (_I, [_VP, C.POINTER(QueryDesc), _FP, _FP, _U32, _FP, _UP, _FP, _UP, _VP]),
    "pm_build_query_host": (_I, [_VP, _FP, _FP, _U32, _I, C.POINTER(QueryDesc), _FP, _FP, _U32, _FP, _U32, _VP]),
    "pm_query_bruteforce": (_I, [_VP, C.POINTER(QueryDesc), _FP, _FP, _U32, _FP, _UP, _FP, _UP, _VP]),
    "pm_query_noalloc": (_I, [_VP, C.POINTER(QueryDesc), _FP, _FP, _U32, _FP, _UP, _FP, _UP, _VP]),
    "pm_query_backward": (_I, [_VP, C.POINTER(QueryDesc), _FP, _FP, _U32, _FP, _UP, _FP, _UP, _FP, _FP, _VP]),
    "pm_set_backward_chunk": (_I, [_VP, _U32]),
    "pm_gather_for": (_I, [_VP, C.POINTER(QueryDesc), _FP, _FP, _FP, _FP, _FP, _FP, _UP, _U32, _FP, _FP, _VP]),
    "pm_scale_flux": (_I, [_VP, _F, _VP]),
    "pm_merge": (_I, [_VP, _FP, _FP, _UP, _U32, C.POINTER(C.c_uint32), _VP]),
    "pm_build_merged": (_I, [_VP, _I, _VP]),
    "pm_clear_merged": (_I, [_VP]),
    "pm_merged_count": (_I, [_VP, C.POINTER(C.c_uint32)]),
    "pm_compute_query_radii": (_I, [_VP, C.POINTER(QueryDesc), _FP, _U32, _FP, _VP]),
    "pm_get_info": (_I, [_VP, C.POINTER(MapInfo), _VP]),
    "pm_set_profiling": (_I, [_VP, _I]),
    "pm_last_timings": (_I, [_VP, C.POINTER(Timings)]),
    "pm_query_stats": (_I, [_VP, _VP, _U32]),
    "pm_clear_errors": (_I, [_VP, _VP]),
    "pm_export_tree": (_I, [_VP, _VP, _U32, _VP, _VP, _U32]),
    "pm_icut_build": (_I, [_VP, C.POINTER(IcutDesc), C.POINTER(QueryDesc), _FP, _VP]),
    "pm_icut_slot_count": (_I, [_VP, C.POINTER(C.c_uint32)]),
    "pm_icut_node_centers": (_I, [_VP, _FP, _VP]),
    "pm_icut_interpolate": (_I, [_VP, _F, _FP, _FP, _U32, _FP, _VP]),
    "pm_icut_export": (_I, [_VP, _U32, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "pm_batch_create": (_I, [C.POINTER(C.c_void_p)]),
    "pm_batch_destroy": (_I, [_VP]),
    "pm_batch_set_tuning": (_I, [_VP, _U32, _I, _I, _I]),
    "pm_batch_build": (_I, [_VP, _FP, _FP, _VP, _U32, _I, _VP]),
    "pm_batch_query": (_I, [_VP, _VP, _FP, _FP, _VP, _FP, _UP, _FP, _UP, _VP]),
    "pm_batch_capture": (_I, [_VP, _FP, _FP, _VP, _U32, _I, _VP, _FP, _FP, _VP, _FP, _UP, _FP, _UP]),
    "pm_batch_launch": (_I, [_VP, _VP]),
    "pm_batch_get_info": (_I, [_VP, C.POINTER(MapInfo), _VP]),
    "pm_batch_last_error": (C.c_char_p, [_VP]),
    "pm_batch_autotune": (_I, [_VP, _FP, _FP, _VP, _U32, _I, _VP, _FP, _FP, _VP, _FP, C.POINTER(Tuning), _VP]),
    "pm_last_error": (C.c_char_p, [_VP]),
    "pm_status_string": (C.c_char_p, [_I]),
    "pm_abi_version": (_I, []),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libpmgpu.so (once) and declares every entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"engine library {p} is missing; build it with `python -m mnrt_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class PMError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


def check(status: int, handle=None) -> None:
    if status != PM_OK:
        lib = load()
        msg = lib.pm_last_error(handle).decode() if handle else lib.pm_status_string(status).decode()
        raise PMError(status, msg or lib.pm_status_string(status).decode())
