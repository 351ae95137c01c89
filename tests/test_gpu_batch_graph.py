"""The captured graph over prepared problem batches gives every problem the rows
of the plain batch call (and so of one plain call per problem, which the batch
tests tie to plain calls and the oracle): same ids, FP64 distance bits and
order, problem after problem across batches, on two replays in a row.  Cases
include a problem without queries, batches of dense clustered problems whose
heavy queries go through the device-driven radius refinement, coincident
points that no refinement separates (recomputed by the plain batch call), and
a row buffer too small for the rows."""
import numpy as np
import pytest

from oracle import oracle as O
from rtdl_b200 import workloads
from rtdl_b200.batch import B200ProblemBatch, B200ProblemBatchGraph, concat_records
from rtdl_b200.runtime import FRN_ROW_DTYPE

pytestmark = pytest.mark.gpu


def _split(problems, sizes):
    out, i = [], 0
    for n in sizes:
        out.append(problems[i:i + n])
        i += n
    return out


def _expected(batches, groups):
    """Rows of the plain batch call, batch by batch, problem-major."""
    rows, offsets = [], [0]
    for batch, probs in zip(batches, groups):
        out = batch.fixed_radius_neighbors([p[0] for p in probs], radius=[p[2] for p in probs],
                                           k_max=[p[3] for p in probs])
        for p in range(out.problems):
            rows.append(out.problem(p))
            offsets.append(offsets[-1] + len(out.problem(p)))
    return (np.concatenate(rows) if rows else np.zeros(0, FRN_ROW_DTYPE)), np.array(offsets, dtype=np.uint64)


def _run_graph(groups, capacity=None, replays=2):
    import torch

    batches = [B200ProblemBatch([p[1] for p in probs]) for probs in groups]
    allp = [p for probs in groups for p in probs]
    qrec = concat_records([p[0] for p in allp])
    qoff = np.zeros(len(allp) + 1, dtype=np.uint64)
    qoff[1:] = np.cumsum([len(p[0]) for p in allp])
    exp_rows, exp_off = _expected(batches, groups)
    cap = len(exp_rows) if capacity is None else capacity
    d_q = torch.from_numpy(qrec.view(np.uint8).copy()).cuda()
    d_rows = torch.zeros(max(cap, 1) * 16, dtype=torch.uint8, device="cuda")
    results = []
    try:
        with B200ProblemBatchGraph(batches, d_q.data_ptr(), qoff, radius=[p[2] for p in allp],
                                   k_max=[p[3] for p in allp], rows_address=d_rows.data_ptr(),
                                   rows_capacity=cap) as g:
            assert g.info()["problems"] == len(allp)
            for _ in range(replays):
                d_rows.fill_(0xAB)  # a replay writes every row again
                off, status = g.replay()
                n = min(cap, int(off[-1]))
                rows = np.frombuffer(d_rows[: 16 * n].cpu().numpy().tobytes(), dtype=FRN_ROW_DTYPE)
                results.append((off, status, rows))
            info = g.info()
    finally:
        for b in batches:
            b.close()
    return results, exp_rows, exp_off, info


def _same(a, b):
    assert len(a) == len(b)
    assert np.array_equal(a["query_id"], b["query_id"])
    assert np.array_equal(a["neighbor_id"], b["neighbor_id"])
    assert np.array_equal(a["distance"].view(np.uint64), b["distance"].view(np.uint64))


def test_graph_matches_plain_batches_over_several_batches(gpu):
    probs = workloads.batched_problems(count=30, seed=31, lo=64, hi=12000)
    kmax = np.random.default_rng(3).integers(1, 65, 30)
    probs = [(q, b, r, int(k)) for (q, b, r, _), k in zip(probs, kmax)]
    probs[4] = (probs[4][0][:0], probs[4][1], probs[4][2], probs[4][3])  # a problem without queries
    results, exp_rows, exp_off, info = _run_graph(_split(probs, [7, 15, 8]))
    assert info["kernel_nodes"] > 0
    for off, status, rows in results:
        assert status == 0
        assert np.array_equal(off, exp_off)
        _same(rows, exp_rows)


def test_graph_heavy_clustered_problems_refined_on_the_device(gpu):
    c = np.random.default_rng(0).random((8, 3))
    probs = []
    for i in range(6):
        rng = np.random.default_rng(40 + i)
        q = workloads.records(workloads._mixture(rng, 3000 + 500 * i, c))
        b = workloads.records(workloads._mixture(rng, 20000 + 3000 * i, c))
        probs.append((q, b, 0.02 + 0.004 * i, 64))  # hundreds of points in radius near the centres
    results, exp_rows, exp_off, _ = _run_graph(_split(probs, [3, 3]))
    for off, status, rows in results:
        assert np.array_equal(off, exp_off)
        _same(rows, exp_rows)
    q, b, r, k = probs[0]
    _same(results[0][2][: int(exp_off[1])], O.fixed_radius_neighbors(q, b, radius=r, k_max=k, threads=8))


def test_graph_coincident_points_recomputed_by_the_plain_call(gpu):
    # 400 copies of each of 3 points: every query has 400+ points at distance 0, no radius separates them
    pts = np.repeat(np.array([[0.2, 0.2, 0.2], [0.5, 0.5, 0.5], [0.8, 0.8, 0.8]]), 400, axis=0)
    b = workloads.records(pts)
    q = workloads.records(pts[::37])
    results, exp_rows, exp_off, info = _run_graph([[(q, b, 0.01, 16)], [(q, b, 0.0, 64)]])
    for off, status, rows in results:
        assert np.array_equal(off, exp_off)
        _same(rows, exp_rows)
    assert info["fallbacks"] >= 1


def test_graph_reports_rows_past_capacity(gpu):
    probs = workloads.batched_problems(count=4, seed=33, lo=200, hi=2000)
    results, exp_rows, exp_off, _ = _run_graph([probs], capacity=10, replays=1)
    off, status, rows = results[0]
    assert status & 4
    assert np.array_equal(off, exp_off)
    _same(rows, exp_rows[:10])
