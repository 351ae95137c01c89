"""fixed_radius_count_threshold and the nearest in-radius witness (the
reference's count-threshold family) against the oracle, which
tests/test_oracle_golden.py pins to rows of the reference's own generic CPU
count.  Counts, flags and ids must be equal exactly; witness distances bit
for bit (exact FP64).
"""
import json
from pathlib import Path

import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pts(pts, ids=None):
    ids = np.arange(len(pts), dtype=np.uint32) if ids is None else ids
    d = {"id": ids, "x": pts[:, 0], "y": pts[:, 1]}
    if pts.shape[1] == 3:
        d["z"] = pts[:, 2]
    return d


def _pack(c):
    return rt.pack_points(ids=c["id"], x=c["x"], y=c["y"], z=c.get("z"))


def _clustered(rng, n, dim, centres, sigma=0.01):
    pts = centres[rng.integers(0, len(centres), n)] + rng.normal(0.0, sigma, (n, dim))
    bg = rng.random(n) < 0.1
    pts[bg] = rng.random((int(bg.sum()), dim))
    return np.clip(pts, 0.0, 1.0).astype(np.float32).astype(np.float64)


def _rows_equal(got, exp):
    assert len(got) == len(exp)
    for f in ("query_id", "neighbor_count", "threshold_reached"):
        assert np.array_equal(np.array([r[f] for r in got], dtype=np.int64), exp[f].astype(np.int64)), f


def test_golden_cases_through_the_cuda_path(gpu):
    data = json.loads((Path(__file__).parent / "golden" / "count_threshold_2d.json").read_text())
    for case in data["cases"]:
        q = {k: np.asarray(v, dtype=np.uint32 if k == "id" else np.float64) for k, v in case["query"].items()}
        s = {k: np.asarray(v, dtype=np.uint32 if k == "id" else np.float64) for k, v in case["search"].items()}
        got = rt.fixed_radius_count_threshold_2d(_pack(q), _pack(s), radius=case["radius"],
                                                 threshold=case["threshold"])
        exp = np.asarray(case["rows"], dtype=np.int64)
        assert [tuple(r.values()) for r in got] == [tuple(int(v) for v in row) for row in exp], case["name"]


@pytest.mark.parametrize("threshold", [0, 1, 7, 40, 300])
def test_count_threshold_2d_matches_oracle(gpu, threshold):
    rng = np.random.default_rng(50 + threshold)
    centres = rng.random((10, 2))
    s = _pts(_clustered(rng, 40000, 2, centres, 0.004))
    q = _pts(_clustered(rng, 6000, 2, centres, 0.004), ids=rng.permutation(6000).astype(np.uint32))
    radius = 0.004
    exp = O.fixed_radius_count_threshold(q, s, radius=radius, threshold=threshold, threads=8)
    _rows_equal(rt.fixed_radius_count_threshold_2d(_pack(q), _pack(s), radius=radius, threshold=threshold), exp)
    with rt.prepare_b200_fixed_radius_count_threshold_2d(_pack(s), max_radius=0.01) as prep:
        _rows_equal(prep.run(_pack(q), radius=radius, threshold=threshold), exp)
        assert prep.count_threshold_reached(_pack(q), radius=radius, threshold=threshold) == \
            int(exp["threshold_reached"].sum())
    # the queries themselves as the search set
    own = O.fixed_radius_count_threshold(q, q, radius=radius, threshold=threshold, threads=8)
    _rows_equal(rt.fixed_radius_count_threshold_2d(_pack(q), radius=radius, threshold=threshold), own)


def test_device_columns_2d(gpu):
    import torch

    rng = np.random.default_rng(8)
    s_pts, q_pts = rng.random((20000, 2)), rng.random((3000, 2))
    s, q = _pts(s_pts), _pts(q_pts, ids=(np.arange(3000, dtype=np.uint32) * 5)[::-1].copy())
    cols = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in (("ids", s["id"]), ("x", s["x"]),
                                                                            ("y", s["y"]))}
    qcols = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in (("ids", q["id"]), ("x", q["x"]),
                                                                             ("y", q["y"]))}
    ids = torch.zeros(3000, dtype=torch.int32, device="cuda")
    counts = torch.zeros(3000, dtype=torch.int32, device="cuda")
    flags = torch.zeros(3000, dtype=torch.int32, device="cuda")
    with rt.prepare_b200_fixed_radius_count_threshold_2d_device_search_columns(cols, max_radius=0.02) as prep:
        for threshold in (0, 4):
            prep.write_device_count_threshold_columns(qcols, radius=0.015, threshold=threshold, query_ids_out=ids,
                                                      neighbor_counts_out=counts, threshold_flags_out=flags)
            torch.cuda.synchronize()
            exp = O.fixed_radius_count_threshold(q, s, radius=0.015, threshold=threshold, threads=8)
            assert np.array_equal(ids.cpu().numpy().view(np.uint32), exp["query_id"])
            assert np.array_equal(counts.cpu().numpy().view(np.uint32), exp["neighbor_count"])
            assert np.array_equal(flags.cpu().numpy().view(np.uint32), exp["threshold_reached"])
    with rt.prepare_b200_fixed_radius_count_threshold_2d(_pack(s), max_radius=0.02) as host_prep:
        with pytest.raises(RuntimeError, match="device-search-column"):
            host_prep.write_device_count_threshold_columns(qcols, radius=0.015, threshold=1, query_ids_out=ids,
                                                           neighbor_counts_out=counts, threshold_flags_out=flags)


@pytest.mark.parametrize("threshold", [0, 3, 64])
def test_count_threshold_3d_device_outputs(gpu, threshold):
    import torch

    rng = np.random.default_rng(90 + threshold)
    centres = rng.random((12, 3))
    s = _pts(_clustered(rng, 50000, 3, centres))
    q = _pts(_clustered(rng, 8000, 3, centres))
    ids = torch.zeros(8000, dtype=torch.int32, device="cuda")
    counts = torch.zeros(8000, dtype=torch.int32, device="cuda")
    flags = torch.zeros(8000, dtype=torch.int32, device="cuda")
    with rt.prepare_b200_fixed_radius_count_threshold_3d(_pack(s), max_radius=0.01) as prep:
        prep.write_device_count_threshold_columns(_pack(q), radius=0.008, threshold=threshold, query_ids_out=ids,
                                                  neighbor_counts_out=counts, threshold_flags_out=flags)
    torch.cuda.synchronize()
    got_ids, got_counts, got_flags = (t.cpu().numpy().view(np.uint32) for t in (ids, counts, flags))
    assert np.array_equal(got_ids, q["id"])
    if threshold == 0:  # the reference's 3-D device contract: threshold 0 is reached with count 0
        assert not got_counts.any() and got_flags.all()
    else:
        exp = O.fixed_radius_count_threshold(q, s, radius=0.008, threshold=threshold, threads=8)
        assert np.array_equal(got_counts, exp["neighbor_count"])
        assert np.array_equal(got_flags, exp["threshold_reached"])
        assert got_flags.any() and not got_flags.all()


def test_nearest_witness_2d_matches_oracle(gpu):
    rng = np.random.default_rng(13)
    grid = np.stack(np.meshgrid(np.arange(60), np.arange(60)), -1).reshape(-1, 2).astype(np.float64) * 0.01
    s_pts = np.concatenate([grid, grid[:500], rng.random((3000, 2)) * 0.6])  # duplicates: ties broken by id
    s = _pts(s_pts, ids=rng.permutation(len(s_pts)).astype(np.uint32))
    q_pts = np.concatenate([grid[rng.integers(0, len(grid), 2000)] + rng.integers(-1, 2, (2000, 2)) * 0.005,
                            rng.random((500, 2)) * 2.0])  # many outside every radius
    q = _pts(q_pts, ids=rng.integers(0, 1500, len(q_pts)).astype(np.uint32))
    with rt.prepare_b200_fixed_radius_count_threshold_2d(_pack(s), max_radius=0.05) as prep:
        for radius in (0.0, 0.005, 0.02):
            got = prep.nearest_witness_rows(_pack(q), radius=radius)
            exp = O.nearest_witness(q, s, radius=radius, threads=8)
            assert [r["query_id"] for r in got] == exp["query_id"].tolist()
            assert [r["neighbor_id"] for r in got] == exp["neighbor_id"].tolist()
            assert np.array_equal(np.array([r["distance"] for r in got]).view(np.uint64),
                                  exp["distance"].view(np.uint64))
            assert (exp["neighbor_id"] == 0xFFFFFFFF).any()


def test_count_checks_and_empty_sets(gpu):
    rng = np.random.default_rng(2)
    s = _pts(rng.random((100, 2)))
    q = _pts(rng.random((10, 2)))
    assert rt.fixed_radius_count_threshold_2d(_pack(q), _pack(_pts(np.zeros((0, 2)))), radius=0.1) == ()
    with rt.prepare_b200_fixed_radius_count_threshold_2d(_pack(s), max_radius=0.1) as prep:
        with pytest.raises(ValueError, match="max_radius"):
            prep.run(_pack(q), radius=0.2)
        with pytest.raises(ValueError, match="threshold"):
            prep.run(_pack(q), radius=0.05, threshold=-1)
        assert prep.run(_pack(_pts(np.zeros((0, 2)))), radius=0.05) == ()
    with rt.prepare_b200_fixed_radius_count_threshold_2d(_pack(_pts(np.zeros((0, 2)))), max_radius=0.1) as empty:
        assert empty.run(_pack(q), radius=0.05) == ()
        assert empty.count_threshold_reached(_pack(q), radius=0.05, threshold=1) == 0
