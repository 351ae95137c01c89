"""Coordinates the library rejects: non-finite values and magnitudes beyond
1e18, in the query set or the search set, through the plain per-call entry
points (one query range and several), a prepared scene and the device-rows
call.  Each call must fail with the library's message and leave the library
usable: the next valid call returns the oracle's rows."""
import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MESSAGE = "point coordinates must be finite with magnitude <= 1e18"


def _cols(pts):
    d = {"id": np.arange(len(pts), dtype=np.uint32), "x": pts[:, 0].copy(), "y": pts[:, 1].copy()}
    if pts.shape[1] == 3:
        d["z"] = pts[:, 2].copy()
    return d


def _pack(c):
    return rt.pack_points(ids=c["id"], x=c["x"], y=c["y"], z=c.get("z"))


def _valid_call_still_works():
    rng = np.random.default_rng(5)
    s, q = _cols(rng.random((3000, 3))), _cols(rng.random((500, 3)))
    v = rt.runtime.fixed_radius_neighbors(_pack(q), _pack(s), radius=0.08, k_max=8)
    got = v.to_numpy()
    v.close()
    exp = O.fixed_radius_neighbors(q, s, radius=0.08, k_max=8)
    assert np.array_equal(got["query_id"], exp["query_id"])
    assert np.array_equal(got["neighbor_id"], exp["neighbor_id"])
    assert np.array_equal(got["distance"].view(np.uint64), exp["distance"].view(np.uint64))


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf, 2.0e18])
@pytest.mark.parametrize("where", ["query", "search"])
def test_plain_call_rejects_bad_coordinates(gpu, bad, where):
    rng = np.random.default_rng(11)
    s_pts, q_pts = rng.random((4000, 3)), rng.random((9000, 3))
    (q_pts if where == "query" else s_pts)[1234, 1] = bad
    with pytest.raises(RuntimeError, match=MESSAGE):
        rt.runtime.fixed_radius_neighbors(_pack(_cols(q_pts)), _pack(_cols(s_pts)), radius=0.05, k_max=16)
    _valid_call_still_works()


def test_ranged_plain_call_rejects_bad_query_in_last_range(gpu):
    """300,003 queries run in two ranges of their input order; the bad
    coordinate sits in the second, whose set is prepared while the first
    range's rows are copied."""
    rng = np.random.default_rng(12)
    s_pts, q_pts = rng.random((50000, 3)), rng.random((300003, 3))
    q_pts[-7, 2] = np.nan
    with pytest.raises(RuntimeError, match=MESSAGE):
        rt.runtime.fixed_radius_neighbors(_pack(_cols(q_pts)), _pack(_cols(s_pts)), radius=0.01, k_max=8)
    _valid_call_still_works()


@pytest.mark.parametrize("bad", [np.nan, 5.0e18])
def test_scene_rejects_bad_search_points(gpu, bad):
    rng = np.random.default_rng(13)
    s_pts = rng.random((2000, 2))
    s_pts[17, 0] = bad
    with pytest.raises(RuntimeError, match=MESSAGE):
        rt.B200Scene(_pack(_cols(s_pts)))
    _valid_call_still_works()


def test_prepared_scene_rejects_bad_queries(gpu):
    rng = np.random.default_rng(14)
    s, q_pts = _cols(rng.random((5000, 3))), rng.random((3000, 3))
    q_pts[2999, 0] = -np.inf
    with rt.B200Scene(_pack(s)) as scene:
        with pytest.raises(RuntimeError, match=MESSAGE):
            scene.query(_pack(_cols(q_pts)), predicate="fixed_radius_neighbors", radius=0.05, limit=8)
        with pytest.raises(RuntimeError, match=MESSAGE):
            scene.query(_pack(_cols(q_pts)), predicate="knn_rows", limit=4)
        # the scene stays usable
        q_ok = _cols(rng.random((300, 3)))
        v = scene.query(_pack(q_ok), predicate="knn_rows", limit=4)
        got = v.to_numpy()
        v.close()
        exp = O.knn_rows(q_ok, s, k=4)
        assert np.array_equal(got["neighbor_id"], exp["neighbor_id"])
