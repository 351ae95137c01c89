"""Problem batches against one plain call per problem and against the oracle.

Every problem of a batch must get exactly the rows (same ids, same FP64
distance bits, same order) that rtdl_b200.fixed_radius_neighbors gives it
alone, which the parity tests tie to the oracle; a few problems are also
checked against the oracle directly.
"""
import numpy as np
import pytest

import rtdl_b200 as rt
from rtdl_b200 import workloads
from rtdl_b200.batch import B200ProblemBatch, concat_records
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _plain(probe, build, radius, k_max):
    view = rt.runtime.fixed_radius_neighbors(rt.pack_points(records=probe), rt.pack_points(records=build),
                                             radius=radius, k_max=k_max)
    try:
        return view.to_numpy().copy()
    finally:
        view.close()


def _same(a, b):
    assert len(a) == len(b)
    assert np.array_equal(a["query_id"], b["query_id"])
    assert np.array_equal(a["neighbor_id"], b["neighbor_id"])
    assert np.array_equal(a["distance"].view(np.uint64), b["distance"].view(np.uint64))


def _uneven_problems(count, seed, lo=64, hi=20000):
    return workloads.batched_problems(count=count, seed=seed, lo=lo, hi=hi)


@pytest.mark.parametrize("seed", [11, 12])
def test_batch_matches_plain_calls(gpu, seed):
    probs = _uneven_problems(24, seed)
    probes = [p[0] for p in probs]
    builds = [p[1] for p in probs]
    radius = [p[2] for p in probs]
    kmax = [int(k) for k in np.random.default_rng(seed).integers(1, 65, len(probs))]
    with B200ProblemBatch(builds) as batch:
        out = batch.fixed_radius_neighbors(probes, radius=radius, k_max=kmax, with_overflow=True)
    assert out.problems == len(probs)
    for p in range(len(probs)):
        _same(out.problem(p), _plain(probes[p], builds[p], radius[p], kmax[p]))
    # the overflow flags agree with the in-radius counts of the oracle on a sample
    p0 = 0
    counts = O.fixed_radius_neighbors(probes[p0], builds[p0], radius=radius[p0], k_max=1 << 30, with_counts=True)[1]
    n0 = len(probes[p0])
    assert np.array_equal(out.overflow[:n0].astype(bool), counts > kmax[p0])


def test_batch_against_oracle(gpu):
    probs = _uneven_problems(6, 21, lo=32, hi=3000)
    with B200ProblemBatch([p[1] for p in probs]) as batch:
        out = batch.fixed_radius_neighbors([p[0] for p in probs], radius=[p[2] for p in probs], k_max=64)
    for p, (probe, build, radius, _) in enumerate(probs):
        exp = O.fixed_radius_neighbors(probe, build, radius=radius, k_max=64)
        got = out.problem(p)
        assert np.array_equal(got["query_id"], exp["query_id"])
        assert np.array_equal(got["neighbor_id"], exp["neighbor_id"])
        assert np.array_equal(got["distance"].view(np.uint64), exp["distance"].view(np.uint64))


def test_batch_edge_cases(gpu):
    rng = np.random.default_rng(5)

    def pts(n, scale=1.0, ids=None):
        return workloads.records((rng.random((n, 3)) * scale).astype(np.float32).astype(np.float64), ids)

    builds = [pts(500), pts(0), pts(1), pts(7), pts(300, 10.0), pts(2000)]
    probes = [pts(0), pts(40), pts(3), pts(9), pts(33, 10.0),
              pts(70, ids=np.random.default_rng(1).permutation(70).astype(np.uint32) * 3)]  # ids out of order
    radius = [0.1, 0.2, 0.5, 0.3, 0.0, 0.08]
    kmax = [8, 4, 1, 64, 2, 16]
    with B200ProblemBatch(builds) as batch:
        out = batch.fixed_radius_neighbors(probes, radius=radius, k_max=kmax)
    assert out.row_offsets[0] == 0 and out.row_offsets[1] == 0  # no queries
    assert out.row_offsets[2] == out.row_offsets[1]  # no search points
    for p in range(len(builds)):
        _same(out.problem(p), _plain(probes[p], builds[p], radius[p], kmax[p]))


def test_batch_2d_and_single_problem(gpu):
    a, b = workloads.hausdorff_2d(5000)
    with B200ProblemBatch([b]) as batch:
        out = batch.fixed_radius_neighbors([a], radius=0.01, k_max=32)
    _same(out.problem(0), _plain(a, b, 0.01, 32))
    halves = [b[:2500], b[2500:]]
    with B200ProblemBatch(halves) as batch:
        out = batch.fixed_radius_neighbors([a[:1000], a[1000:3000]], radius=[0.02, 0.005], k_max=[10, 64])
    _same(out.problem(0), _plain(a[:1000], halves[0], 0.02, 10))
    _same(out.problem(1), _plain(a[1000:3000], halves[1], 0.005, 64))


def test_batch_heavy_queries_take_the_generic_path(gpu):
    # a dense cluster: some queries see more than 256 points in radius
    rng = np.random.default_rng(9)
    dense = workloads.records((rng.normal(0.5, 0.01, (20000, 3))).astype(np.float32).astype(np.float64))
    sparse = workloads.records(rng.random((20000, 3)).astype(np.float32).astype(np.float64))
    q1 = workloads.records((rng.normal(0.5, 0.01, (500, 3))).astype(np.float32).astype(np.float64))
    q2 = workloads.records(rng.random((500, 3)).astype(np.float32).astype(np.float64))
    with B200ProblemBatch([sparse, dense]) as batch:
        out = batch.fixed_radius_neighbors([q2, q1], radius=[0.05, 0.01], k_max=[64, 40])
    _same(out.problem(0), _plain(q2, sparse, 0.05, 64))
    _same(out.problem(1), _plain(q1, dense, 0.01, 40))


def test_batch_device_entry_point(gpu):
    import torch

    probs = _uneven_problems(10, 31)
    probes = [p[0] for p in probs]
    builds = [p[1] for p in probs]
    radius = [p[2] for p in probs]
    with B200ProblemBatch(builds) as batch:
        host = batch.fixed_radius_neighbors(probes, radius=radius, k_max=32)
        allq = concat_records(probes)
        qoff = np.zeros(len(probes) + 1, dtype=np.uint64)
        qoff[1:] = np.cumsum([len(p) for p in probes])
        d_q = torch.from_numpy(allq.view(np.uint8).copy()).cuda()
        sizes = batch.fixed_radius_neighbors_device(d_q.data_ptr(), qoff, radius=radius, k_max=32, rows_address=None,
                                                    rows_capacity=0)
        assert np.array_equal(sizes, host.row_offsets)
        rows = torch.empty(int(sizes[-1]) * 16, dtype=torch.uint8, device="cuda")
        batch.fixed_radius_neighbors_device(d_q.data_ptr(), qoff, radius=radius, k_max=32,
                                            rows_address=rows.data_ptr(), rows_capacity=int(sizes[-1]))
        torch.cuda.synchronize()
        got = np.frombuffer(rows.cpu().numpy().tobytes(), dtype=rt.runtime.FRN_ROW_DTYPE)
        _same(got, host.rows)


def test_plain_entry_points_reject_a_batch(gpu):
    probs = _uneven_problems(2, 3, lo=100, hi=200)
    with B200ProblemBatch([p[1] for p in probs]) as batch:
        from rtdl_b200 import _native

        lib = _native.load_library()
        err = _native.error_buffer()
        import ctypes

        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        q = rt.pack_points(records=probs[0][0])
        status = lib.rtdl_b200_scene_query(batch.handle, q.address, q.count, 0, 0.1, 8, ctypes.byref(rows),
                                           ctypes.byref(count), None, err, len(err))
        assert status == 1
        assert "batch" in err.value.decode()
