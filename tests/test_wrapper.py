"""CPU: the Python mirror of the PhotonMap interface rejects bad arguments
before it reaches the engine (no GPU needed), and maps the reference's names
onto the C ABI descriptor."""
import numpy as np
import pytest
import torch

from mnrt_b200 import _lib as L


@pytest.fixture
def pm(engine_lib):
    from mnrt_b200.photon_map import PhotonMap
    m = PhotonMap(1000, global_q_radius_max=0.1, knn_target_count=32)
    yield m
    m.close()


def test_engine_buffers_must_be_cuda_tensors(pm):
    from mnrt_b200.photon_map import _ptr
    assert _ptr(None) is None
    with pytest.raises(ValueError, match="CUDA"):
        _ptr(torch.zeros((4, 4), dtype=torch.float32))


def test_build_checks_dtype_and_shape(pm):
    with pytest.raises(ValueError, match="float32"):
        pm.build(torch.zeros((8, 4), dtype=torch.float64), torch.zeros((8, 4), dtype=torch.float64))
    with pytest.raises(ValueError, match=r"\(n, 4\)"):
        pm.build(torch.zeros((8, 3), dtype=torch.float32), torch.zeros((8, 3), dtype=torch.float32))


def test_build_query_host_checks_host_arrays(pm):
    z = torch.zeros((8, 4), dtype=torch.float32)
    with pytest.raises(ValueError, match="contiguous float32"):
        pm.build_query_host(z, z, z.double(), z)
    with pytest.raises(ValueError, match="contiguous float32"):
        pm.build_query_host(z, z, z.t().contiguous().t(), z)   # not contiguous
    with pytest.raises(ValueError, match="contiguous float32"):
        pm.build_query_host(z[:, :3].contiguous(), z, z, z)


def test_descriptor_defaults_and_names(pm):
    d = pm.desc(filter="cone", cone_k=1.5, min_found=8)
    assert d.k == 32 and np.isclose(d.r_max, 0.1) and d.filter == L.PM_FILTER_CONE
    assert np.isclose(d.cone_k, 1.5) and d.min_found == 8 and d.mode == L.PM_MODE_EXACT
    assert d.order == L.PM_ORDER_SORTED and d.refine_iters == 2
    d = pm.desc(k=7, r_max=0.5, filter="epanechnikov", sorted_queries=False)
    assert d.k == 7 and d.filter == L.PM_FILTER_EPANECHNIKOV and d.order == L.PM_ORDER_AS_GIVEN
    with pytest.raises(KeyError):
        pm.desc(filter="gaussian")


def test_set_knn_target_count_sets_the_default_k(pm):
    pm.set_knn_target_count(64)
    assert pm.desc().k == 64


def test_tuning_is_validated_by_the_engine(pm):
    pm.set_tuning(leaf_size=16, warps_per_block=2, rounds_per_chunk=8, queries_per_warp=1, kbuf_layout=2)
    with pytest.raises(L.PMError):
        pm.set_tuning(leaf_size=16, warps_per_block=9)
    with pytest.raises(L.PMError):
        pm.set_tuning(leaf_size=16, rounds_per_chunk=0)


def test_batch_offsets_and_descriptors(engine_lib):
    from mnrt_b200.batch import PhotonMapBatch, _offsets, make_desc
    assert _offsets([0, 5, 5, 9]).tolist() == [0, 5, 5, 9]
    for bad in ([5, 9], [0], [[0, 1], [1, 2]]):
        with pytest.raises(ValueError, match="offsets"):
            _offsets(bad)
    d = make_desc(16, 0.05, filter="epanechnikov", min_found=8)
    assert d.k == 16 and d.filter == L.PM_FILTER_EPANECHNIKOV and d.min_found == 8 and d.mode == L.PM_MODE_EXACT
    arr = PhotonMapBatch._descs([d, dict(k=4, r_max=0.1, filter="cone")])
    assert arr[0].k == 16 and arr[1].k == 4 and arr[1].filter == L.PM_FILTER_CONE
    b = PhotonMapBatch()
    with pytest.raises(L.PMError):
        b.set_tuning(leaf_size=0)
    b.close()
    b.close()   # closing twice is harmless
