"""The served loop: every request's rows equal the plain per-call result for
that request alone (same ids, ranks and FP64 distance bits), whether it ran
batched with others, concurrently on another stream, or waited for memory."""
import numpy as np
import pytest

from rtdl_b200 import workloads
from rtdl_b200.serve import FRN, KNN, B200Server, replay, request_bytes, same_rows

pytestmark = pytest.mark.gpu


def _scenes():
    c = np.random.default_rng(0).random((64, 3))
    sizes = {"s0": 20_000, "s1": 60_000, "s2": 150_000}
    return {name: workloads.records(workloads._mixture(np.random.default_rng(10 + i), n, c))
            for i, (name, n) in enumerate(sizes.items())}, c


def _trace(scene_points, c, count, seed, spread_s=0.0):
    rng = np.random.default_rng(seed)
    names = sorted(scene_points)
    trace = []
    for i in range(count):
        name = names[rng.integers(len(names))]
        n = int(np.exp(rng.uniform(np.log(50), np.log(20_000))))
        q = workloads.records(workloads._mixture(np.random.default_rng(1000 + i), n, c))
        scale = (1 << 20) / len(scene_points[name])
        if rng.random() < 0.5:
            trace.append((spread_s * i / count, name, FRN, q, 0.00287 * scale ** (1 / 3),
                          int(rng.choice([8, 32, 64]))))
        else:
            trace.append((spread_s * i / count, name, KNN, q, 0.0, int(rng.choice([1, 8, 32]))))
    return trace


def _check(server, reqs):
    for r in reqs:
        assert r.error is None, r.error
        view = server.scenes[r.scene].query(r.queries, predicate=r.op, radius=r.radius, limit=r.limit)
        try:
            exp = view.to_numpy()
        finally:
            view.close()
        assert same_rows(r.rows, exp), (r.rid, r.op, r.limit, len(r.rows), len(exp))


def test_served_results_equal_alone_and_batched(gpu):
    pts, c = _scenes()
    with B200Server(streams=3, max_batch_probes=60_000) as server:
        for name, p in pts.items():
            server.add_scene(name, p)
        reqs = replay(server, _trace(pts, c, 60, 7))  # a burst: requests wait and are batched
        _check(server, reqs)
        st = server.stats()
        assert st["requests"] == 60 and st["failed"] == 0
        assert max(r.batch_size for r in reqs) > 1  # some fixed-radius requests shared a launch


def test_served_admission_waits_for_memory(gpu):
    pts, c = _scenes()
    trace = _trace(pts, c, 24, 8, spread_s=0.05)
    biggest = max(request_bytes(op, len(q), lim, 3) for _, _, op, q, _, lim in trace)
    scene_bytes = sum(len(p) * 112 for p in pts.values())
    # room for the scenes and about one request at a time
    with B200Server(streams=4, memory_budget=scene_bytes + int(1.2 * biggest)) as server:
        for name, p in pts.items():
            server.add_scene(name, p)
        reqs = replay(server, trace)
        _check(server, reqs)
        assert server.budget.used == scene_bytes  # every request released its charge


def test_served_without_batching_matches(gpu):
    pts, c = _scenes()
    with B200Server(streams=2, batching=False) as server:
        for name, p in pts.items():
            server.add_scene(name, p)
        reqs = replay(server, _trace(pts, c, 20, 9))
        _check(server, reqs)
        assert all(r.batch_size == 1 for r in reqs)


def test_multi_request_entry_point_matches_single_requests(gpu):
    import torch

    from rtdl_b200.batch import concat_records

    pts, c = _scenes()
    from rtdl_b200 import B200Scene

    with B200Scene(pts["s1"]) as scene:
        qs = [workloads.records(workloads._mixture(np.random.default_rng(70 + i), n, c))
              for i, n in enumerate([0, 37, 5000, 1, 12000])]
        radius = [0.01, 0.02, 0.005, 0.03, 0.0071]
        kmax = [5, 64, 16, 1, 40]
        allq = concat_records(qs)
        qoff = np.zeros(len(qs) + 1, dtype=np.uint64)
        qoff[1:] = np.cumsum([len(q) for q in qs])
        d_q = torch.from_numpy(allq.view(np.uint8).copy()).cuda()
        sizes = scene.fixed_radius_neighbors_multi_device(d_q.data_ptr(), qoff, radius=radius, k_max=kmax,
                                                          rows_address=None, rows_capacity=0)
        rows = torch.empty(max(int(sizes[-1]), 1) * 16, dtype=torch.uint8, device="cuda")
        scene.fixed_radius_neighbors_multi_device(d_q.data_ptr(), qoff, radius=radius, k_max=kmax,
                                                  rows_address=rows.data_ptr(), rows_capacity=int(sizes[-1]))
        torch.cuda.synchronize()
        from rtdl_b200.runtime import FRN_ROW_DTYPE

        got = np.frombuffer(rows.cpu().numpy().tobytes(), dtype=FRN_ROW_DTYPE)[: int(sizes[-1])]
        for i, q in enumerate(qs):
            view = scene.query(q, predicate=FRN, radius=radius[i], limit=kmax[i])
            exp = view.to_numpy()
            view.close()
            assert same_rows(got[int(sizes[i]): int(sizes[i + 1])], exp), i
