"""pm_query_noalloc: the query entry point that allocates no device memory.

Some callers cannot allocate device memory when they query: a render loop that
must not stall (cudaMalloc and cudaFree synchronise the whole device), or a
host application that gives the engine a fixed memory budget at start-up and
lets nothing grow afterwards.  pm_query_noalloc serves them: its scratch lives
in one fixed array inside the library, shared by every call.

This test calls it through the C ABI twice in a row, on different query sets
and parameters, and checks each result against pm_query on the same map:
neighbour lists, counts, r^2 and radiance bit for bit (the header promises
identical results; that is stricter than the parity tests' RTOL, which the
radiance also meets).  A counting allocator on the handle shows that no call
reaches the handle's allocator.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mnrt_b200 import _lib as L
from mnrt_b200 import gen

pytestmark = pytest.mark.gpu

RTOL = 1e-5   # the radiance tolerance of the parity tests


def _dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _ptr(t):
    return None if t is None else t.data_ptr()


def _outputs(nq, k, dev):
    return {"rad": torch.empty((nq, 4), dtype=torch.float32, device=dev),
            "nbr": torch.empty((nq, k), dtype=torch.int32, device=dev),
            "r2": torch.empty((nq,), dtype=torch.float32, device=dev),
            "count": torch.empty((nq,), dtype=torch.int32, device=dev)}


def _call(lib, fn, h, desc, qpos, qnrm, out):
    stream = torch.cuda.current_stream().cuda_stream
    st = fn(h, C.byref(desc), _ptr(qpos), _ptr(qnrm), qpos.shape[0], _ptr(out["rad"]), _ptr(out["nbr"]),
            _ptr(out["r2"]), _ptr(out["count"]), stream)
    assert st == L.PM_OK, lib.pm_last_error(h).decode()


def test_query_noalloc_matches_query(cuda):
    lib = L.load()
    dev = cuda
    ph = gen.photons(200000, seed=41, caustic_frac=0.2)
    d_pos, d_pow = _dev(ph.pos, dev), _dev(ph.pow, dev)

    allocs = []

    @L.ALLOC_FN
    def counting_alloc(pp, nbytes, user):
        p = torch.cuda.caching_allocator_alloc(int(nbytes), dev.index)
        pp[0] = p
        allocs.append(p)
        return 0

    @L.FREE_FN
    def counting_free(p, user):
        torch.cuda.caching_allocator_delete(p)

    h = C.c_void_p()
    assert lib.pm_create(C.byref(h), ph.n, None, None, 0.05) == L.PM_OK
    try:
        assert lib.pm_set_allocator(h, counting_alloc, counting_free, None) == L.PM_OK
        stream = torch.cuda.current_stream().cuda_stream
        assert lib.pm_build(h, d_pos.data_ptr(), d_pow.data_ptr(), ph.n, L.PM_PHOTONS_PACKED, stream) == L.PM_OK
        torch.cuda.synchronize()
        after_build = len(allocs)

        cases = [
            # (query count, seed, k, filter, order)
            (50000, 42, 64, L.PM_FILTER_CONE, L.PM_ORDER_SORTED),
            (3001, 43, 100, L.PM_FILTER_BOX, L.PM_ORDER_SORTED),
        ]
        results = []
        for nq, seed, k, filt, order in cases:   # two calls in a row, before any pm_query
            q = gen.queries(nq, seed=seed)
            qpos, qnrm = _dev(q.pos, dev), _dev(q.nrm, dev)
            d = L.QueryDesc(k=k, r_max=0.05, filter=filt, cone_k=1.0, mode=L.PM_MODE_EXACT, min_found=0,
                            order=order, refine_iters=2)
            out = _outputs(nq, k, dev)
            _call(lib, lib.pm_query_noalloc, h, d, qpos, qnrm, out)
            torch.cuda.synchronize()
            tm = L.Timings()
            assert lib.pm_last_timings(h, C.byref(tm)) == L.PM_OK
            assert tm.query_launches > 0 and tm.query_ms == 0.0   # this call's launches, no phase times
            results.append((d, qpos, qnrm, {key: v.cpu().numpy() for key, v in out.items()}))
        assert len(allocs) == after_build, "pm_query_noalloc reached the handle's allocator"

        for d, qpos, qnrm, got in results:
            ref = _outputs(qpos.shape[0], d.k, dev)
            _call(lib, lib.pm_query, h, d, qpos, qnrm, ref)
            torch.cuda.synchronize()
            ref = {key: v.cpu().numpy() for key, v in ref.items()}
            for key in ("nbr", "count", "r2"):
                assert np.array_equal(got[key], ref[key]), key
            np.testing.assert_allclose(got["rad"], ref["rad"], rtol=RTOL, atol=0.0)
            assert np.array_equal(got["rad"].view(np.uint32), ref["rad"].view(np.uint32)), "radiance bits"
            assert (got["count"] > 0).all()

        info = L.MapInfo()
        assert lib.pm_get_info(h, C.byref(info), None) == L.PM_OK
        assert info.device_errors == 0

        # more queries than the fixed array holds: a clear error, no work
        big = L.PM_NOALLOC_MAX_QUERIES + 1
        d = results[0][0]
        st = lib.pm_query_noalloc(h, C.byref(d), qpos.data_ptr(), qnrm.data_ptr(), big, ref_rad_ptr(dev), None,
                                  None, None, None)
        assert st == L.PM_ERR_INVALID
        assert b"PM_NOALLOC_MAX_QUERIES" in lib.pm_last_error(h)
    finally:
        torch.cuda.synchronize()
        assert lib.pm_destroy(h) == L.PM_OK


_keep = []


def ref_rad_ptr(dev):
    """A valid, aligned radiance buffer pointer (never written: the call is rejected first)."""
    t = torch.empty((16, 4), dtype=torch.float32, device=dev)
    _keep.append(t)
    return t.data_ptr()
