"""The allocation-free directed-Hausdorff entry point against the regular one.

rtdl_b200_scene_directed_hausdorff_noalloc serves callers that cannot
allocate device memory during the query (their allocator owns the device heap,
they run inside a CUDA graph they do not own, or they sit in a real-time loop).
It takes its scratch from a fixed device array, so this test calls it twice in
a row -- the second call must not see the first call's leftovers -- and checks
the witness and the per-query nearest arrays bit for bit against
rtdl_b200_scene_directed_hausdorff.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import rtdl_b200 as rt
from rtdl_b200 import _native, workloads

pytestmark = pytest.mark.gpu


def _device_records(records):
    import torch

    return torch.from_numpy(records.view(np.uint8).copy()).cuda()


def _noalloc(scene, d_queries, nq, d_dist, d_ids, d_witness, stream):
    lib = _native.load_library()
    err = _native.error_buffer()
    status = lib.rtdl_b200_scene_directed_hausdorff_noalloc(
        scene.handle, d_queries.data_ptr(), nq, d_dist.data_ptr(), d_ids.data_ptr(), d_witness.data_ptr(), stream,
        err, len(err))
    return status, err.value.decode()


@pytest.mark.parametrize("case", ["hausdorff_2d", "clustered_3d"])
def test_noalloc_matches_regular_entry_point_twice(gpu, case):
    import torch

    if case == "hausdorff_2d":
        a, b = workloads.hausdorff_2d(1 << 16)
        queries, search = a, b
    else:
        queries, search = workloads.clustered_3d(200_000, 150_000)
    nq = len(queries)
    with rt.B200Scene(rt.pack_points(records=search)) as scene:
        expected, exp_dist, exp_ids = scene.directed_hausdorff(rt.pack_points(records=queries), with_nearest=True)
        d_queries = _device_records(queries)
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):  # the second call reuses the scratch the first one left behind
            d_dist = torch.full((nq,), -1.0, dtype=torch.float64, device="cuda")
            d_ids = torch.zeros(nq, dtype=torch.int32, device="cuda")
            d_witness = torch.zeros(24, dtype=torch.uint8, device="cuda")
            status, msg = _noalloc(scene, d_queries, nq, d_dist, d_ids, d_witness, stream)
            assert status == 0, msg
            torch.cuda.synchronize()
            w = _native.RtdlB200Witness.from_buffer_copy(d_witness.cpu().numpy().tobytes())
            assert w.status == 0
            assert w.distance == expected["distance"]
            assert (w.source_id, w.target_id) == (expected["source_id"], expected["target_id"])
            assert np.array_equal(d_dist.cpu().numpy().view(np.uint64), exp_dist.view(np.uint64))
            assert np.array_equal(d_ids.cpu().numpy().view(np.uint32), exp_ids)


def _check_against_regular(scene, queries, stream):
    import torch

    nq = len(queries)
    expected, exp_dist, exp_ids = scene.directed_hausdorff(rt.pack_points(records=queries), with_nearest=True)
    d_queries = _device_records(queries)
    d_dist = torch.full((nq,), -1.0, dtype=torch.float64, device="cuda")
    d_ids = torch.zeros(nq, dtype=torch.int32, device="cuda")
    d_witness = torch.zeros(24, dtype=torch.uint8, device="cuda")
    status, msg = _noalloc(scene, d_queries, nq, d_dist, d_ids, d_witness, stream)
    assert status == 0, msg
    torch.cuda.synchronize()
    w = _native.RtdlB200Witness.from_buffer_copy(d_witness.cpu().numpy().tobytes())
    assert w.status == 0
    assert w.distance == expected["distance"]
    assert (w.source_id, w.target_id) == (expected["source_id"], expected["target_id"])
    assert np.array_equal(d_dist.cpu().numpy().view(np.uint64), exp_dist.view(np.uint64))
    assert np.array_equal(d_ids.cpu().numpy().view(np.uint32), exp_ids)


def test_noalloc_large_3d_then_small_2d(gpu):
    """A smaller call after a larger one on another scene and dimension: the
    scratch still holds the large call's per-query data past the small call's
    end and its reduction partials, which the small call must not read."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    big_q, big_s = workloads.clustered_3d(250_000, 180_000)
    with rt.B200Scene(rt.pack_points(records=big_s)) as scene:
        _check_against_regular(scene, big_q, stream)
    a, b = workloads.hausdorff_2d(3_000)
    with rt.B200Scene(rt.pack_points(records=b)) as scene:
        _check_against_regular(scene, a, stream)


def test_noalloc_rejects_more_queries_than_its_scratch_holds(gpu):
    import torch

    queries, search = workloads.clustered_3d(1000, 262_145)
    with rt.B200Scene(rt.pack_points(records=search)) as scene:
        d_queries = _device_records(queries)
        d_witness = torch.zeros(24, dtype=torch.uint8, device="cuda")
        lib = _native.load_library()
        err = _native.error_buffer()
        status = lib.rtdl_b200_scene_directed_hausdorff_noalloc(
            scene.handle, d_queries.data_ptr(), len(queries), None, None, d_witness.data_ptr(), None, err, len(err))
        assert status == 1
        assert "262144" in err.value.decode()
