"""Concurrent calls on worker threads, each with its own CUDA stream, give the
same rows as the same call made alone.

The library promises to be re-entrant per stream (the served loop runs one
worker per stream).  These tests run KNN with k in {1, 8, 32} -- the list
kernels' shared-memory size differs per k -- and fixed-radius calls on three
threads at once, at block sizes 128 and 256, and with the tuning changed by
another thread while the calls run; every result must equal the call made
alone, bit for bit.
"""
import threading

import numpy as np
import pytest

import rtdl_b200 as rt
from rtdl_b200 import workloads
from rtdl_b200.runtime import FRN_ROW_DTYPE, KNN_ROW_DTYPE
from rtdl_b200.serve import same_rows

pytestmark = pytest.mark.gpu

_REQUESTS = [("knn_rows", 0.0, 1), ("knn_rows", 0.0, 8), ("knn_rows", 0.0, 32),
             ("fixed_radius_neighbors", 0.012, 64), ("knn_rows", 0.0, 32), ("knn_rows", 0.0, 1)]


def _device_call(scene, d_q, nq, predicate, radius, k, stream):
    import torch

    row_bytes = FRN_ROW_DTYPE.itemsize if predicate == "fixed_radius_neighbors" else KNN_ROW_DTYPE.itemsize
    rows = torch.empty(nq * k * row_bytes, dtype=torch.uint8, device="cuda")
    n = scene.query_device(d_q.data_ptr(), nq, predicate=predicate, radius=radius, limit=k,
                           rows_address=rows.data_ptr(), rows_capacity=nq * k, stream=stream.cuda_stream)
    stream.synchronize()
    dtype = FRN_ROW_DTYPE if predicate == "fixed_radius_neighbors" else KNN_ROW_DTYPE
    return rows[: n * row_bytes].cpu().numpy().view(dtype).copy()


def _alone(scene, d_q, nq):
    import torch

    s = torch.cuda.Stream()
    return {i: _device_call(scene, d_q, nq, *req, s) for i, req in enumerate(_REQUESTS)}


def _run_threads(scene, d_q, nq, expected, workers=3, rounds=4, flip_tuning=False):
    import torch

    errors = []
    stop = threading.Event()

    def worker(w):
        s = torch.cuda.Stream()
        try:
            for r in range(rounds):
                for j in range(len(_REQUESTS)):
                    i = (j + w + r) % len(_REQUESTS)
                    got = _device_call(scene, d_q, nq, *_REQUESTS[i], s)
                    if not same_rows(got, expected[i]):  # fields only: KNN rows carry 4 padding bytes
                        errors.append(f"worker {w} request {_REQUESTS[i]}: {len(got)} rows vs {len(expected[i])}")
        except Exception as ex:  # noqa: BLE001 - reported below with the worker
            errors.append(f"worker {w}: {ex}")

    def flipper():
        b = 0
        while not stop.is_set():
            rt.set_tuning(block_threads=(128, 256)[b & 1])
            b += 1
            stop.wait(0.002)

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(workers)]
    flip = threading.Thread(target=flipper) if flip_tuning else None
    if flip:
        flip.start()
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    stop.set()
    if flip:
        flip.join()
    return errors


@pytest.fixture(scope="module")
def scene_and_queries():
    import torch

    probe, build = workloads.clustered_3d(60_000, 6_000)
    scene = rt.B200Scene(rt.pack_points(records=build))
    d_q = torch.from_numpy(probe.view(np.uint8).copy()).cuda()
    yield scene, d_q, len(probe)
    scene.close()
    rt.set_tuning()


@pytest.mark.parametrize("block", [128, 256])
def test_concurrent_knn_equals_alone(gpu, scene_and_queries, block):
    scene, d_q, nq = scene_and_queries
    rt.set_tuning(block_threads=block)
    expected = _alone(scene, d_q, nq)
    errors = _run_threads(scene, d_q, nq, expected)
    rt.set_tuning()
    assert not errors, errors[:5]


def test_concurrent_calls_with_tuning_changed_meanwhile(gpu, scene_and_queries):
    """Every tuning gives the same rows; a call runs with the tuning it started with."""
    scene, d_q, nq = scene_and_queries
    rt.set_tuning()
    expected = _alone(scene, d_q, nq)
    errors = _run_threads(scene, d_q, nq, expected, rounds=3, flip_tuning=True)
    rt.set_tuning()
    assert not errors, errors[:5]
