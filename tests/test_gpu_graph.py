"""Captured batch graph of prepared-query aggregates (the reference's
PreparedOptixFixedRadiusRankedSummaryAggregateBatchGraph3D) against the plain
prepared-query aggregate of each request, which the summary tests tie to the
oracle and to the reference's published aggregates.

Every replay, after an update, and through the same-stream device partials,
each request's aggregate must equal the plain call's exactly (integer fields
and the FP64 distance sum bit for bit: the graph runs the same kernels in the
same order).  The set with heavy queries exercises the device-driven
refinement; the set of coincident points leaves heavy queries that no radius
separates, which the graph marks and replay recomputes by the plain call.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from rtdl_b200 import workloads
from rtdl_b200.runtime import (PreparedB200FixedRadiusNeighbors3D, PreparedB200FixedRadiusQueryPoints3D)
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "rtnn_ranked_summary_262144.json").read_text())
FIELDS = ("query_count", "bounded_neighbor_count", "nearest_id_checksum", "kth_id_checksum")


def _same(got, exp):
    for f in FIELDS:
        assert got[f] == exp[f], (f, got[f], exp[f])
    assert np.float64(got["sum_distance"]).view(np.uint64) == np.float64(exp["sum_distance"]).view(np.uint64)


def _plain(prep, pq, requests):
    return [prep.aggregate_ranked_summary_prepared_queries(pq, radius=r["radius"], k_max=r["k_max"])
            for r in requests]


def _rtnn(distribution, n):
    g = GOLDEN["distributions"][distribution]
    pts = workloads.rtnn_points(distribution, n, g["seed"])
    for c in ("x", "y", "z"):
        pts[c] = pts[c].astype(np.float32).astype(np.float64)
    return pts


@pytest.mark.parametrize("distribution", ["uniform", "clustered", "shell"])
def test_graph_equals_plain_aggregates(gpu, distribution):
    pts = _rtnn(distribution, 65_536)
    requests = [{"radius": 0.02, "k_max": 50}, {"radius": 0.01, "k_max": 64}, {"radius": 0.035, "k_max": 7},
                {"radius": 0.0, "k_max": 1}]
    prep = PreparedB200FixedRadiusNeighbors3D(pts, max_radius=0.035)
    pq = PreparedB200FixedRadiusQueryPoints3D(pts)
    try:
        exp = _plain(prep, pq, requests)
        with prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, requests) as graph:
            for _ in range(2):  # replays reuse the same buffers
                got = graph.replay()
                assert len(got) == len(requests)
                for i, (g, e) in enumerate(zip(got, exp)):
                    _same(g, e)
                    assert g["request_index"] == i and g["cuda_graph_replay"] is True
                    assert g["radius"] == requests[i]["radius"] and g["k_max"] == requests[i]["k_max"]
            dev = graph.replay_same_stream_device_partials_summary()
            assert dev["metadata"]["query_block_count"] == 1
            for g, e in zip(dev["aggregates"], exp):
                _same(g, e)
            # new requests, same count: captured again
            upd = [{"radius": 0.03, "k_max": 64}, {"radius": 0.02, "k_max": 50}, {"radius": 0.005, "k_max": 3},
                   {"radius": 0.035, "k_max": 64}]
            graph.update_requests(upd)
            assert graph.request_buffer_update_count == 1
            for g, e in zip(graph.replay(), _plain(prep, pq, upd)):
                _same(g, e)
                assert g["request_buffer_update_count"] == 1
    finally:
        pq.close()
        prep.close()


def test_graph_heavy_queries_match_oracle(gpu):
    # a dense cluster: many queries see more than 256 points in radius
    rng = np.random.default_rng(9)
    dense = workloads.records(rng.normal(0.5, 0.01, (20_000, 3)).astype(np.float32).astype(np.float64))
    q = workloads.records(rng.normal(0.5, 0.012, (3_000, 3)).astype(np.float32).astype(np.float64))
    requests = [{"radius": 0.01, "k_max": 40}, {"radius": 0.004, "k_max": 64}]
    prep = PreparedB200FixedRadiusNeighbors3D(dense, max_radius=0.01)
    pq = PreparedB200FixedRadiusQueryPoints3D(q)
    try:
        with prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, requests) as graph:
            got = graph.replay()
            assert graph.fallback_count == 0
    finally:
        pq.close()
        prep.close()
    for g, r in zip(got, requests):
        _, exp = O.ranked_summaries(q, dense, radius=r["radius"], k_max=r["k_max"], threads=8)
        for f in FIELDS:
            assert g[f] == exp[f], f
        assert g["sum_distance"] == pytest.approx(exp["sum_distance"], rel=1e-12)


def test_graph_unresolved_heavy_queries_fall_back(gpu):
    # 400 coincident points: every query at that spot has 400 points at one
    # distance, so no refined radius brings its count into [k_max, 256]
    rng = np.random.default_rng(2)
    spread = rng.random((5_000, 3))
    pts = np.concatenate([spread, np.full((400, 3), 0.25)]).astype(np.float32).astype(np.float64)
    build = workloads.records(pts)
    qp = np.concatenate([np.full((5, 3), 0.25), rng.random((500, 3))]).astype(np.float32).astype(np.float64)
    q = workloads.records(qp)
    requests = [{"radius": 0.05, "k_max": 10}, {"radius": 0.02, "k_max": 64}]
    prep = PreparedB200FixedRadiusNeighbors3D(build, max_radius=0.05)
    pq = PreparedB200FixedRadiusQueryPoints3D(q)
    try:
        exp = _plain(prep, pq, requests)
        with prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, requests) as graph:
            got = graph.replay()
            assert graph.fallback_count == 2
            for g, e in zip(got, exp):
                _same(g, e)
            dev = graph.replay_same_stream_device_partials_summary()
            assert dev["metadata"]["requests_recomputed_by_plain_call"] == 2
            for g, e in zip(dev["aggregates"], exp):
                _same(g, e)
    finally:
        pq.close()
        prep.close()
    _, ora = O.ranked_summaries(q, build, radius=0.05, k_max=10, threads=8)
    for f in FIELDS:
        assert got[0][f] == ora[f], f


def test_graph_checks_and_empty_handles(gpu):
    pts = _rtnn("uniform", 4_096)
    prep = PreparedB200FixedRadiusNeighbors3D(pts, max_radius=0.05)
    pq = PreparedB200FixedRadiusQueryPoints3D(pts)
    empty_q = PreparedB200FixedRadiusQueryPoints3D(pts[:0])
    try:
        with pytest.raises(ValueError, match="k_max <= 64"):
            prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, [{"radius": 0.01, "k_max": 65}])
        with pytest.raises(ValueError, match="max_radius"):
            prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, [{"radius": 0.06, "k_max": 8}])
        with pytest.raises(ValueError, match="at least one request"):
            prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, [])
        with prep.prepare_ranked_summary_prepared_queries_batch_graph(pq, [{"radius": 0.01, "k_max": 8}]) as graph:
            with pytest.raises(ValueError, match="request_count unchanged"):
                graph.update_requests([{"radius": 0.01, "k_max": 8}] * 2)
        with pytest.raises(RuntimeError, match="closed"):
            graph.replay()
        with prep.prepare_ranked_summary_prepared_queries_batch_graph(empty_q, [{"radius": 0.01, "k_max": 8}]) as g:
            (res,) = g.replay()
            assert res["query_count"] == 0 and res["bounded_neighbor_count"] == 0
    finally:
        empty_q.close()
        pq.close()
        prep.close()
