"""Full-size workloads of the benchmark: the 1,048,576 x 1,048,576 3D clustered
sets (fixed radius with k_max 64, and KNN with k = 16) and the 4,194,304 x
4,194,304 2D Hausdorff sets.  Each complete output is compared with the
oracle's digest of it (tests/golden/full_scale_digests.json, every row of
every query), a seeded sample of queries is compared row by row with the
oracle run here, and the size-independent properties are checked."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O
from rtdl_b200 import workloads

pytestmark = pytest.mark.gpu

DIGESTS = json.loads((Path(__file__).resolve().parent / "golden" / "full_scale_digests.json").read_text())


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def _first_bad_block(rows, per_q, ref):
    """The first block of queries whose rows differ from the oracle's (None when all agree)."""
    offsets = np.zeros(len(per_q) + 1, dtype=np.int64)
    np.cumsum(per_q, out=offsets[1:])
    b = ref["block_queries"]
    for i, want in enumerate(ref["block_sha256_16"]):
        lo, hi = i * b, min((i + 1) * b, len(per_q))
        if _sha(rows[offsets[lo]:offsets[hi]])[:16] != want:
            return lo, hi
    return None


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
    # the complete row set against the oracle's
    ref = DIGESTS["frn_1m"]
    assert int(overflow.astype(bool).sum()) == ref["overflow_queries"]
    assert _sha(per_q.astype(np.uint32)) == ref["counts_sha256"]
    assert len(rows) == ref["rows"]
    assert _sha(rows) == ref["rows_sha256"], f"rows differ from the oracle's in queries {_first_bad_block(rows, per_q, ref)}"


def test_full_scale_plain_call_rows(gpu, clustered):
    """The plain per-call entry point with host records and host rows
    (rtdl_b200_run_fixed_radius_neighbors_3d), the call the end-to-end
    benchmark times: 1,048,576 queries are answered in eight ranges of their
    input order whose rows are copied to the host while the next range runs.
    The complete row set must equal the oracle's."""
    probe, build = clustered
    view = rt.runtime.fixed_radius_neighbors(rt.pack_points(records=probe), rt.pack_points(records=build),
                                             radius=workloads.CLUSTERED_RADIUS, k_max=64)
    rows = view.to_numpy()
    view.close()
    ref = DIGESTS["frn_1m"]
    per_q = np.bincount(rows["query_id"], minlength=len(probe))
    assert len(rows) == ref["rows"]
    assert _sha(per_q.astype(np.uint32)) == ref["counts_sha256"]
    assert _sha(rows) == ref["rows_sha256"], f"rows differ from the oracle's in queries {_first_bad_block(rows, per_q, ref)}"


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
    # the complete row set against the oracle's (fields packed without the struct's padding)
    packed = np.zeros(len(rows), dtype=np.dtype({"names": ["query_id", "neighbor_id", "distance", "neighbor_rank"],
                                                 "formats": ["<u4", "<u4", "<f8", "<u4"],
                                                 "offsets": [0, 4, 8, 16], "itemsize": 20}))
    for f in packed.dtype.names:
        packed[f] = rows[f]
    assert _sha(packed) == DIGESTS["knn16_1m"]["rows_packed_sha256"]


def test_full_scale_hausdorff_4m(gpu):
    a, b = workloads.hausdorff_2d()
    with rt.B200Scene(rt.pack_points(records=b)) as scene:
        w, dist, nid = scene.directed_hausdorff(rt.pack_points(records=a), with_nearest=True)
    ref = DIGESTS["hausdorff_4m"]
    assert _sha(np.asarray(dist, dtype=np.float64)) == ref["nearest_distance_sha256"]
    assert _sha(np.asarray(nid, dtype=np.uint32)) == ref["nearest_id_sha256"]
    assert w["distance"] == float.fromhex(ref["witness"]["distance_hex"])
    assert (w["source_id"], w["target_id"]) == (ref["witness"]["source_id"], ref["witness"]["target_id"])
