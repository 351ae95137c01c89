"""Prepared point-group witness (the reference's
PreparedOptixPointGroupNearestWitness2D) against the oracle's FP64
restatement of the reference's point-group kernels: threshold flags and
counts, witness rows (exact distances bit for bit) and the max-distance row.
"""
import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O
from rtdl_b200.runtime import pack_point_groups

pytestmark = pytest.mark.gpu


def _pack(pts, ids):
    return rt.pack_points(ids=ids, x=pts[:, 0], y=pts[:, 1])


def _setup(seed):
    rng = np.random.default_rng(seed)
    centres = rng.random((20, 2))
    pts = centres[rng.integers(0, 20, 12000)] + rng.normal(0.0, 0.01, (12000, 2))
    pts = np.concatenate([pts, pts[:200]]).astype(np.float32).astype(np.float64)  # duplicates
    ids = rng.permutation(len(pts)).astype(np.uint32)
    order = np.lexsort((pts[:, 1], np.floor(pts[:, 0] * 40)))  # spans of nearby points
    pts, ids = pts[order], ids[order]
    groups = []
    off = 0
    gid = 0
    while off < len(pts):
        n = int(rng.integers(0, 60))
        n = min(n, len(pts) - off)
        span = pts[off:off + n]
        lo = span.min(axis=0) if n else np.zeros(2)
        hi = span.max(axis=0) if n else np.zeros(2)
        groups.append({"id": gid, "point_offset": off, "point_count": n, "min_x": lo[0], "min_y": lo[1],
                       "max_x": hi[0], "max_y": hi[1]})
        gid += 1
        off += n
    # overlapping spans (their points take part once per group) and a group whose box misses its points
    groups.append({"id": gid, "point_offset": 100, "point_count": 300, "min_x": pts[100:400, 0].min(),
                   "min_y": pts[100:400, 1].min(), "max_x": pts[100:400, 0].max(), "max_y": pts[100:400, 1].max()})
    groups.append({"id": gid + 1, "point_offset": 5000, "point_count": 40, "min_x": 2.0, "min_y": 2.0,
                   "max_x": 2.1, "max_y": 2.1})
    q = np.concatenate([centres[rng.integers(0, 20, 2500)] + rng.normal(0.0, 0.012, (2500, 2)),
                        rng.random((500, 2))]).astype(np.float32).astype(np.float64)
    qids = rng.integers(0, 900, len(q)).astype(np.uint32)
    return pts, ids, pack_point_groups(groups), q, qids


@pytest.mark.parametrize("seed", [1, 2])
def test_point_group_matches_oracle(gpu, seed):
    pts, ids, groups, q, qids = _setup(seed)
    search = {"id": ids, "x": pts[:, 0], "y": pts[:, 1]}
    query = {"id": qids, "x": q[:, 0], "y": q[:, 1]}
    with rt.prepare_b200_point_group_nearest_witness_2d(_pack(pts, ids), groups, max_radius=0.02) as prep:
        for radius in (0.0, 0.004, 0.015):
            for threshold in (0, 1, 6):
                counts, flags, rows, max_row = O.point_group_witness(query, search, groups, radius=radius,
                                                                      threshold=threshold)
                got = prep.threshold_flags(_pack(q, qids), radius=radius, threshold=threshold)
                assert np.array_equal(got, flags)
                assert prep.count_threshold_reached(_pack(q, qids), radius=radius, threshold=threshold) == \
                    int(flags.sum())
            wit = prep.nearest_witness_rows(_pack(q, qids), radius=radius)
            assert [r["query_id"] for r in wit] == rows["query_id"].tolist()
            assert [r["neighbor_id"] for r in wit] == rows["neighbor_id"].tolist()
            assert np.array_equal(np.array([r["distance"] for r in wit]).view(np.uint64),
                                  rows["distance"].view(np.uint64))
            got_max = prep.nearest_max_distance_row(_pack(q, qids), radius=radius)
            assert got_max["query_id"] == max_row["query_id"] and got_max["neighbor_id"] == max_row["neighbor_id"]
            assert got_max["distance"] == max_row["distance"]


def test_point_group_edge_cases(gpu):
    pts = np.array([[0.0, 0.0], [0.1, 0.0], [0.2, 0.0]])
    ids = np.array([7, 3, 5], dtype=np.uint32)
    q = np.array([[0.05, 0.0], [5.0, 5.0]])
    qids = np.array([1, 2], dtype=np.uint32)
    groups = [{"id": 0, "point_offset": 0, "point_count": 3, "min_x": 0.0, "min_y": 0.0, "max_x": 0.2,
               "max_y": 0.0}]
    with rt.prepare_b200_point_group_nearest_witness_2d(_pack(pts, ids), groups, max_radius=0.1) as prep:
        wit = prep.nearest_witness_rows(_pack(q, qids), radius=0.05)
        # two points at exactly 0.05: the smaller id wins; the far query has no witness
        assert wit[0]["neighbor_id"] == 3 and wit[1]["neighbor_id"] == 0xFFFFFFFF
        assert wit[1]["distance"] == 3.4028234663852886e38
        top = prep.nearest_max_distance_row(_pack(q, qids), radius=0.05)
        assert top == {"query_id": 2, "neighbor_id": 0xFFFFFFFF, "distance": float("inf")}
        with pytest.raises(ValueError, match="max_radius"):
            prep.threshold_flags(_pack(q, qids), radius=0.2, threshold=1)
    with rt.prepare_b200_point_group_nearest_witness_2d(_pack(pts, ids), [], max_radius=0.1) as none:
        assert none.threshold_flags(_pack(q, qids), radius=0.05, threshold=0).tolist() == [1, 1]
        assert none.threshold_flags(_pack(q, qids), radius=0.05, threshold=2).tolist() == [0, 0]
        assert none.nearest_witness_rows(_pack(q, qids), radius=0.05) == ()
    with pytest.raises(RuntimeError, match="group span exceeds"):
        rt.prepare_b200_point_group_nearest_witness_2d(
            _pack(pts, ids), [{"id": 0, "point_offset": 2, "point_count": 5, "min_x": 0.0, "min_y": 0.0,
                               "max_x": 1.0, "max_y": 1.0}], max_radius=0.1)
