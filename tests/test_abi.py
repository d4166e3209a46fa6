"""C-ABI tests that need no GPU: the library loads, exports every declared
symbol, and rejects invalid calls before touching the device."""
import ctypes as C
import re
from pathlib import Path

import pytest

from mnrt_b200 import _lib as L

HEADER = Path(__file__).resolve().parent.parent / "include" / "pmgpu.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pm_[a-z_]+)\s*\(", text)) - {"pm_alloc_fn", "pm_free_fn"})


def test_header_declares_the_bound_symbols():
    assert set(declared_functions()) == set(L.SIGNATURES)


def test_library_exports_every_declared_symbol(engine_lib):
    for name in declared_functions():
        assert hasattr(engine_lib, name), name
    assert engine_lib.pm_abi_version() == 1


def _create(lib, r_max=0.1):
    h = C.c_void_p()
    assert lib.pm_create(C.byref(h), 1000, None, None, r_max) == L.PM_OK
    return h


def test_create_validation(engine_lib):
    h = C.c_void_p()
    assert engine_lib.pm_create(C.byref(h), 10, None, None, 0.0) == L.PM_ERR_INVALID
    assert engine_lib.pm_create(C.byref(h), 10, None, None, float("nan")) == L.PM_ERR_INVALID
    assert engine_lib.pm_create(None, 10, None, None, 0.1) == L.PM_ERR_INVALID
    h = _create(engine_lib)
    assert engine_lib.pm_destroy(h) == L.PM_OK
    assert engine_lib.pm_destroy(None) == L.PM_ERR_INVALID


def test_query_validation_without_gpu(engine_lib):
    lib = engine_lib
    h = _create(lib)
    d = L.QueryDesc(k=10, r_max=0.1, filter=L.PM_FILTER_BOX, cone_k=1.0, mode=0, min_found=0, order=0, refine_iters=2)
    # nothing built yet
    assert lib.pm_query(h, C.byref(d), None, None, 0, None, None, None, None, None) == L.PM_ERR_STATE
    assert b"no photon map" in lib.pm_last_error(h)
    bad = [dict(k=0), dict(r_max=0.0), dict(r_max=float("inf")), dict(filter=7), dict(mode=3), dict(order=9),
           dict(filter=L.PM_FILTER_CONE, cone_k=0.5)]
    for b in bad:
        dd = L.QueryDesc(**{**{f: getattr(d, f) for f, _ in L.QueryDesc._fields_}, **b})
        assert lib.pm_query(h, C.byref(dd), None, None, 0, None, None, None, None, None) == L.PM_ERR_INVALID, b
    dd = L.QueryDesc(**{**{f: getattr(d, f) for f, _ in L.QueryDesc._fields_}, "k": L.PM_MAX_K + 1})
    assert lib.pm_query(h, C.byref(dd), None, None, 0, None, None, None, None, None) == L.PM_ERR_UNSUPPORTED
    assert lib.pm_query(h, None, None, None, 0, None, None, None, None, None) == L.PM_ERR_INVALID
    lib.pm_destroy(h)


def test_build_validation_without_gpu(engine_lib):
    lib = engine_lib
    h = _create(lib)
    assert lib.pm_build(h, None, None, 10, L.PM_PHOTONS_PACKED, None) == L.PM_ERR_INVALID
    assert lib.pm_build(h, 16, 32, 10, 5, None) == L.PM_ERR_INVALID
    assert lib.pm_build(h, 17, 32, 10, L.PM_PHOTONS_PACKED, None) == L.PM_ERR_INVALID   # misaligned
    assert lib.pm_build(h, 16, 32, 5000, L.PM_PHOTONS_PACKED, None) == L.PM_ERR_INVALID  # > max_photons
    assert lib.pm_set_tuning(h, 0, 4, 8, 4, 1) == L.PM_ERR_INVALID
    assert lib.pm_set_tuning(h, 65, 4, 8, 4, 1) == L.PM_ERR_INVALID   # leaves hold at most 64 photons
    assert lib.pm_set_tuning(h, 64, 4, 8, 4, 1) == L.PM_OK
    assert lib.pm_set_tuning(h, 16, 9, 8, 4, 1) == L.PM_ERR_INVALID
    assert lib.pm_set_tuning(h, 16, 4, 8, 3, 1) == L.PM_ERR_INVALID
    assert lib.pm_set_tuning(h, 16, 4, 8, 4, 3) == L.PM_ERR_INVALID
    assert lib.pm_set_tuning(h, 16, 4, 8, 4, 1) == L.PM_OK
    assert lib.pm_scale_flux(h, 2.0, None) == L.PM_ERR_STATE
    lib.pm_destroy(h)


def test_allocator_failure_is_reported(engine_lib):
    """An injected allocation failure surfaces as PM_ERR_OOM with no device work."""
    lib = engine_lib
    h = _create(lib)
    calls = []

    @L.ALLOC_FN
    def failing_alloc(pp, nbytes, user):
        calls.append(nbytes)
        return 1

    @L.FREE_FN
    def never_free(p, user):
        raise AssertionError("nothing was allocated")

    assert lib.pm_set_allocator(h, failing_alloc, never_free, None) == L.PM_OK
    st = lib.pm_build(h, 16, 32, 100, L.PM_PHOTONS_PACKED, None)
    assert st == L.PM_ERR_OOM
    assert calls and b"caller allocator" in lib.pm_last_error(h)
    assert lib.pm_destroy(h) == L.PM_OK


def test_status_strings(engine_lib):
    for s in (0, -1, -2, -3, -4, -5, -6):
        assert engine_lib.pm_status_string(s)


def test_backward_validation_without_gpu(engine_lib):
    lib = engine_lib
    h = _create(lib)
    d = L.QueryDesc(k=10, r_max=0.1, filter=L.PM_FILTER_EPANECHNIKOV, cone_k=1.0, mode=0, min_found=0, order=0,
                    refine_iters=2)
    assert lib.pm_query_backward(h, C.byref(d), None, None, 0, None, None, None, None, 16, 16, None) == L.PM_ERR_STATE
    dz = L.QueryDesc(**{**{f: getattr(d, f) for f, _ in L.QueryDesc._fields_}, "mode": L.PM_MODE_ZHOU_COMPAT})
    assert lib.pm_query_backward(h, C.byref(dz), None, None, 0, None, None, None, None, 16, 16, None) == L.PM_ERR_INVALID
    assert lib.pm_set_backward_chunk(h, 1000) == L.PM_OK
    assert lib.pm_set_backward_chunk(None, 1000) == L.PM_ERR_INVALID
    lib.pm_destroy(h)


def test_batch_validation_without_gpu(engine_lib):
    import numpy as np
    lib = engine_lib
    h = C.c_void_p()
    assert lib.pm_batch_create(C.byref(h)) == L.PM_OK
    bad_start = np.array([1, 5], np.uint32)
    assert lib.pm_batch_build(h, 16, 32, bad_start.ctypes.data, 1, L.PM_PHOTONS_PACKED, None) == L.PM_ERR_INVALID
    decreasing = np.array([0, 5, 3], np.uint32)
    assert lib.pm_batch_build(h, 16, 32, decreasing.ctypes.data, 2, L.PM_PHOTONS_PACKED, None) == L.PM_ERR_INVALID
    assert b"must not decrease" in lib.pm_batch_last_error(h)
    assert lib.pm_batch_build(h, 16, 32, None, 2, L.PM_PHOTONS_PACKED, None) == L.PM_ERR_INVALID
    assert lib.pm_batch_launch(h, None) == L.PM_ERR_STATE
    assert lib.pm_batch_set_tuning(h, 0, 4, 8, 1) == L.PM_ERR_INVALID
    assert lib.pm_batch_destroy(h) == L.PM_OK


def test_icut_validation_without_gpu(engine_lib):
    lib = engine_lib
    h = _create(lib)
    d = L.QueryDesc(k=10, r_max=0.1, filter=L.PM_FILTER_BOX, cone_k=1.0, mode=0, min_found=8, order=0, refine_iters=2)
    cut = L.IcutDesc(1, 12, 4, 0.2)
    assert lib.pm_icut_build(h, None, C.byref(d), None, None) == L.PM_ERR_INVALID
    assert lib.pm_icut_build(h, C.byref(cut), None, None, None) == L.PM_ERR_INVALID
    for bad in (L.IcutDesc(1, 12, 65, 0.2), L.IcutDesc(1, 12, 4, -1.0), L.IcutDesc(1, 12, 4, float("nan"))):
        assert lib.pm_icut_build(h, C.byref(bad), C.byref(d), None, None) == L.PM_ERR_INVALID
    assert lib.pm_icut_build(h, C.byref(cut), C.byref(d), 17, None) == L.PM_ERR_INVALID   # misaligned normals
    assert lib.pm_icut_build(h, C.byref(cut), C.byref(d), None, None) == L.PM_ERR_STATE   # nothing built
    icut_mode = L.QueryDesc(k=10, r_max=0.1, filter=0, cone_k=1.0, mode=L.PM_MODE_ICUT, min_found=0, order=0,
                            refine_iters=2)
    assert lib.pm_icut_build(h, C.byref(cut), C.byref(icut_mode), None, None) == L.PM_ERR_INVALID
    assert lib.pm_query(h, C.byref(icut_mode), None, None, 0, None, None, None, None, None) == L.PM_ERR_INVALID
    assert lib.pm_icut_interpolate(h, 0.0, None, None, 0, None, None) == L.PM_ERR_INVALID
    assert lib.pm_icut_interpolate(h, 0.1, None, None, 4, None, None) == L.PM_ERR_INVALID
    assert lib.pm_icut_interpolate(h, 0.1, None, None, 0, None, None) == L.PM_ERR_STATE
    n = C.c_uint32(7)
    assert lib.pm_icut_slot_count(h, C.byref(n)) == L.PM_ERR_STATE
    assert lib.pm_icut_node_centers(h, None, None) == L.PM_ERR_INVALID
    assert lib.pm_icut_export(h, 0, None, None, None, None, None, None, None) == L.PM_ERR_STATE
    lib.pm_destroy(h)


def test_counts_of_2_pow_31_are_unsupported(engine_lib):
    """Query counts stay below 2^31 (32-bit slot arithmetic in the kernels):
    larger calls are refused before any CUDA call."""
    lib = engine_lib
    h = _create(lib)
    d = L.QueryDesc(k=10, r_max=0.1, filter=L.PM_FILTER_BOX, cone_k=1.0, mode=0, min_found=0, order=0, refine_iters=2)
    big = 1 << 31
    assert lib.pm_query(h, C.byref(d), 16, 16, big, 16, None, None, None, None) == L.PM_ERR_UNSUPPORTED
    assert lib.pm_build_query_host(h, None, None, 0, L.PM_PHOTONS_PACKED, C.byref(d), 16, 16, big, 16, 1,
                                   None) == L.PM_ERR_UNSUPPORTED
    assert lib.pm_query(h, C.byref(d), 16, 16, big - 1, 16, None, None, None, None) == L.PM_ERR_STATE   # next check
    lib.pm_destroy(h)


def test_build_query_host_validation_without_gpu(engine_lib):
    lib = engine_lib
    h = _create(lib)
    d = L.QueryDesc(k=10, r_max=0.1, filter=L.PM_FILTER_BOX, cone_k=1.0, mode=0, min_found=0, order=0, refine_iters=2)
    f = lib.pm_build_query_host
    assert f(h, None, None, 0, L.PM_PHOTONS_PACKED, None, None, None, 0, None, 4, None) == L.PM_ERR_INVALID
    assert f(h, None, None, 0, 9, C.byref(d), None, None, 0, None, 4, None) == L.PM_ERR_INVALID
    assert f(h, None, None, 0, L.PM_PHOTONS_PACKED, C.byref(d), None, None, 0, None, 17, None) == L.PM_ERR_INVALID
    assert f(h, None, None, 10, L.PM_PHOTONS_PACKED, C.byref(d), None, None, 0, None, 4, None) == L.PM_ERR_INVALID
    assert f(h, 16, 16, 10, L.PM_PHOTONS_PACKED, C.byref(d), None, None, 5, None, 4, None) == L.PM_ERR_INVALID
    assert f(h, 16, 16, 5000, L.PM_PHOTONS_PACKED, C.byref(d), None, None, 0, None, 4, None) == L.PM_ERR_INVALID
    compat = L.QueryDesc(k=10, r_max=0.1, filter=0, cone_k=1.0, mode=L.PM_MODE_ZHOU_COMPAT, min_found=0, order=0,
                         refine_iters=2)
    assert f(h, None, None, 0, L.PM_PHOTONS_PACKED, C.byref(compat), None, None, 0, None, 4, None) == L.PM_ERR_INVALID
    lib.pm_destroy(h)
