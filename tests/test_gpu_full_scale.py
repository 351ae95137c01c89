"""Full-size 1,048,576 x 1,048,576 3D clustered workload: properties that do not
depend on size, plus exact agreement with the oracle on a seeded sample of
queries against the full build set."""
import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O
from rtdl_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def clustered():
    probe, build = workloads.clustered_3d()
    return probe, build


def _rows_for(rows, qids):
    starts = np.searchsorted(rows["query_id"], qids, side="left")
    ends = np.searchsorted(rows["query_id"], qids, side="right")
    return np.concatenate([rows[s:e] for s, e in zip(starts, ends)])


def test_full_scale_fixed_radius_rows(gpu, clustered):
    probe, build = clustered
    with rt.B200Scene(rt.pack_points(records=build)) as scene:
        view, overflow = scene.query(rt.pack_points(records=probe), predicate="fixed_radius_neighbors",
                                     radius=workloads.CLUSTERED_RADIUS, limit=64, with_overflow=True)
        rows = view.to_numpy()
        view.close()
    n = len(probe)
    # grouped by query id, at most 64 per query, ordered by (distance, neighbor id) within a query
    assert np.all(np.diff(rows["query_id"].astype(np.int64)) >= 0)
    per_q = np.bincount(rows["query_id"], minlength=n)
    assert per_q.max() <= 64
    assert np.all(per_q[overflow.astype(bool)] == 64)
    same = rows["query_id"][1:] == rows["query_id"][:-1]
    d0, d1 = rows["distance"][:-1], rows["distance"][1:]
    n0, n1 = rows["neighbor_id"][:-1], rows["neighbor_id"][1:]
    assert np.all(~same | (d0 < d1) | ((d0 == d1) & (n0 <= n1)))
    assert np.all(rows["distance"] <= workloads.CLUSTERED_RADIUS)
    assert 25.0 < len(rows) / n < 40.0  # mean ~28.5 capped rows per probe
    # exact agreement on a seeded sample against the full build set
    sample = np.sort(np.random.default_rng(77).choice(n, 384, replace=False)).astype(np.uint32)
    exp, counts = O.fixed_radius_neighbors(probe[sample], build, radius=workloads.CLUSTERED_RADIUS, k_max=64,
                                           threads=16, with_counts=True)
    got = _rows_for(rows, sample)
    assert len(got) == len(exp)
    for f in ("query_id", "neighbor_id"):
        assert np.array_equal(got[f], exp[f])
    assert np.array_equal(got["distance"].view(np.uint64), exp["distance"].view(np.uint64))
    assert np.array_equal(overflow[sample].astype(bool), counts > 64)


def test_full_scale_knn16_rows(gpu, clustered):
    probe, build = clustered
    with rt.B200Scene(rt.pack_points(records=build)) as scene:
        view = scene.query(rt.pack_points(records=probe), predicate="knn_rows", limit=16)
        rows = view.to_numpy()
        view.close()
    assert len(rows) == 16 * len(probe)
    assert np.array_equal(rows["neighbor_rank"].reshape(-1, 16), np.tile(np.arange(1, 17, dtype=np.uint32), (len(probe), 1)))
    sample = np.sort(np.random.default_rng(78).choice(len(probe), 256, replace=False)).astype(np.uint32)
    exp = O.knn_rows(probe[sample], build, k=16, threads=16)
    got = rows.reshape(-1, 16)[sample].reshape(-1)
    for f in ("query_id", "neighbor_id", "neighbor_rank"):
        assert np.array_equal(got[f], exp[f])
    assert np.array_equal(got["distance"].view(np.uint64), exp["distance"].view(np.uint64))
