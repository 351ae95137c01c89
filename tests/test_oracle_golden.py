"""Pins the CPU oracle (oracle/nn_oracle.c) to the reference's own outputs.

Every golden case was produced by running the reference's cpu_python_reference
(tests/golden/make_golden.py); the oracle must reproduce each row bit for bit,
including the FP64 distance and the row order."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G

CASES = G.load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_case(case):
    dim = case["dimension"]
    q = G.points_columns(case["query_points"], dim)
    s = G.points_columns(case["search_points"], dim)
    opts = case["options"]
    if case["predicate"] == "knn_rows":
        rows = O.knn_rows(q, s, k=opts["k"])
        got = G.rows_as_tuples(rows, True)
    else:
        ranked = case["predicate"] == "bounded_knn_rows"
        rows = O.fixed_radius_neighbors(q, s, radius=opts["radius"], k_max=opts["k_max"], ranked=ranked)
        got = G.rows_as_tuples(rows, ranked)
    assert got == G.expected_rows(case)


def test_oracle_matches_reference_config1_full():
    z = G.load_config1()
    q, s = G.config1_points()
    rows = O.fixed_radius_neighbors(q, s, radius=0.02, k_max=4096, threads=4)
    assert len(rows) == 20911 == len(z["query_id"])
    assert np.array_equal(rows["query_id"], z["query_id"])
    assert np.array_equal(rows["neighbor_id"], z["neighbor_id"])
    assert np.array_equal(rows["distance"].view(np.uint64), z["distance"].view(np.uint64))


@pytest.mark.parametrize("case", G.load_hausdorff(), ids=lambda c: f"copies{c['copies']}")
def test_oracle_hausdorff_matches_reference_app(case):
    a = G.points_columns(case["points_a"], 2)
    b = G.points_columns(case["points_b"], 2)
    for key, (q, s) in (("directed_a_to_b", (a, b)), ("directed_b_to_a", (b, a))):
        got = O.directed_hausdorff(q, s)
        exp = case[key]
        assert got["distance"] == float.fromhex(exp["distance"])
        assert (got["source_id"], got["target_id"], got["row_count"]) == (exp["source_id"], exp["target_id"], exp["row_count"])


def test_oracle_threads_do_not_change_rows():
    rng = np.random.default_rng(7)
    p = rng.random((3000, 3)).astype(np.float32).astype(np.float64)
    b = rng.random((2000, 3)).astype(np.float32).astype(np.float64)
    q = {"id": rng.integers(0, 50, 3000).astype(np.uint32), "x": p[:, 0], "y": p[:, 1], "z": p[:, 2]}
    s = {"id": np.arange(2000, dtype=np.uint32), "x": b[:, 0], "y": b[:, 1], "z": b[:, 2]}
    one = O.fixed_radius_neighbors(q, s, radius=0.08, k_max=5, threads=1)
    many = O.fixed_radius_neighbors(q, s, radius=0.08, k_max=5, threads=8)
    assert G.rows_as_tuples(one, False) == G.rows_as_tuples(many, False)
    k1 = O.knn_rows(q, s, k=7, threads=1)
    k8 = O.knn_rows(q, s, k=7, threads=8)
    assert G.rows_as_tuples(k1, True) == G.rows_as_tuples(k8, True)


@pytest.mark.skipif(not O.reference_library_available(), reason="reference native oracle not built here")
def test_restatement_agrees_with_reference_native_oracle():
    """The reference's own C++ oracle (compiled from its sources into oracle/_ref)
    sorts with a 1e-12 distance tolerance instead of exact ties; on tie-free
    data both must give the same rows."""
    rng = np.random.default_rng(11)
    p = rng.random((800, 3))
    b = rng.random((1500, 3))
    q = {"id": np.arange(800, dtype=np.uint32), "x": p[:, 0], "y": p[:, 1], "z": p[:, 2]}
    s = {"id": np.arange(1500, dtype=np.uint32), "x": b[:, 0], "y": b[:, 1], "z": b[:, 2]}
    ours = O.fixed_radius_neighbors(q, s, radius=0.12, k_max=6)
    ref = O.reference_fixed_radius_neighbors(O.pack_reference_points(q), O.pack_reference_points(s), radius=0.12, k_max=6)
    assert G.rows_as_tuples(ours, False) == G.rows_as_tuples(ref, False)


def _count_cases():
    import json
    from pathlib import Path

    data = json.loads((Path(__file__).parent / "golden" / "count_threshold_2d.json").read_text())
    return data["cases"]


@pytest.mark.parametrize("case", _count_cases(), ids=lambda c: f"{c['name']}-r{c['radius']}-t{c['threshold']}")
def test_oracle_count_threshold_matches_reference_generic_cpu(case):
    """fixed_radius_count_threshold restated from the oracle's exact counts against rows of the
    reference's own generic CPU count (tests/golden/make_count_threshold_golden.py)."""
    q = {k: np.asarray(v, dtype=np.uint32 if k == "id" else np.float64) for k, v in case["query"].items()}
    s = {k: np.asarray(v, dtype=np.uint32 if k == "id" else np.float64) for k, v in case["search"].items()}
    got = O.fixed_radius_count_threshold(q, s, radius=case["radius"], threshold=case["threshold"])
    exp = np.asarray(case["rows"], dtype=np.int64)
    assert np.array_equal(got["query_id"], exp[:, 0])
    assert np.array_equal(got["neighbor_count"], exp[:, 1])
    assert np.array_equal(got["threshold_reached"], exp[:, 2])


def test_python_restatement_matches_reference_config1_prefix():
    """The pure-Python restatement (the timed stand-in for cpu_python_reference) against the reference's
    own config-1 rows, on the first 512 queries (a few seconds of Python)."""
    from oracle import reference_py

    z = G.load_config1()
    q, s = G.config1_points()
    recs = lambda d: np.rec.fromarrays([d["id"], d["x"], d["y"]], names="id,x,y")  # noqa: E731
    rows = reference_py.fixed_radius_neighbors(reference_py.points(recs(q)[:512]), reference_py.points(recs(s)),
                                               radius=0.02, k_max=4096)
    n = int(np.searchsorted(z["query_id"], 512))
    assert len(rows) == n
    assert [r["query_id"] for r in rows] == z["query_id"][:n].tolist()
    assert [r["neighbor_id"] for r in rows] == z["neighbor_id"][:n].tolist()
    assert np.array_equal(np.array([r["distance"] for r in rows]).view(np.uint64), z["distance"][:n].view(np.uint64))


@pytest.mark.parametrize("case", CASES[:12], ids=[c["name"] for c in CASES[:12]])
def test_python_restatement_matches_reference_case(case):
    from oracle import reference_py

    dim = case["dimension"]
    cols = lambda p: G.points_columns(p, dim)  # noqa: E731
    def recs(d):
        names = ["id", "x", "y"] + (["z"] if dim == 3 else [])
        return np.rec.fromarrays([np.asarray(d[n]) for n in names], names=",".join(names))
    q, s = reference_py.points(recs(cols(case["query_points"]))), reference_py.points(recs(cols(case["search_points"])))
    opts = case["options"]
    if case["predicate"] == "knn_rows":
        rows = reference_py.knn_rows(q, s, k=opts["k"])
        got = [(r["query_id"], r["neighbor_id"], r["distance"], r["neighbor_rank"]) for r in rows]
    else:
        ranked = case["predicate"] == "bounded_knn_rows"
        rows = reference_py.fixed_radius_neighbors(q, s, radius=opts["radius"], k_max=opts["k_max"], ranked=ranked)
        got = [(r["query_id"], r["neighbor_id"], r["distance"]) + ((r["neighbor_rank"],) if ranked else ()) for r in rows]
    assert got == G.expected_rows(case)
