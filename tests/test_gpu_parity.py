"""Parity of the CUDA path (through the C ABI) with the reference's outputs.

Small cases compare against the golden fixtures produced by the reference's
own cpu_python_reference (bit-exact rows: ids, ranks, FP64 distances and row
order).  Larger seeded cases compare against the CPU oracle restatement, which
is itself pinned to those fixtures by tests/test_oracle_golden.py.
"""
import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

CASES = G.load_cases()


def _kernel(predicate, dim, **options):
    geometry = rt.Points3D if dim == 3 else rt.Points
    fields = ["query_id", "neighbor_id", "distance"] + ([] if predicate == "fixed_radius_neighbors" else ["neighbor_rank"])

    @rt.kernel(backend="rtdl", precision="float_approx")
    def k():
        q = rt.input("query_points", geometry, role="probe")
        s = rt.input("search_points", geometry, role="build")
        c = rt.traverse(q, s, accel="bvh")
        return rt.emit(rt.refine(c, predicate=getattr(rt, predicate)(**options)), fields=fields)

    return k


def _as_tuples(rows, ranked):
    if ranked:
        return [(r["query_id"], r["neighbor_id"], r["distance"], r["neighbor_rank"]) for r in rows]
    return [(r["query_id"], r["neighbor_id"], r["distance"]) for r in rows]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_run_b200_matches_reference_golden(gpu, case):
    dim = case["dimension"]
    kernel = _kernel(case["predicate"], dim, **case["options"])
    q = G.points_records(case["query_points"], dim)
    s = G.points_records(case["search_points"], dim)
    rows = rt.run_b200(kernel, query_points=q, search_points=s)
    assert _as_tuples(rows, case["predicate"] != "fixed_radius_neighbors") == G.expected_rows(case)


@pytest.mark.parametrize("case", [c for c in CASES if c["predicate"] != "knn_rows"][:12], ids=lambda c: c["name"])
def test_scene_query_matches_golden_with_columns(gpu, case):
    dim = case["dimension"]
    q = rt.pack_points(**{k if k != "id" else "ids": v for k, v in G.points_columns(case["query_points"], dim).items()})
    s = rt.pack_points(**{k if k != "id" else "ids": v for k, v in G.points_columns(case["search_points"], dim).items()})
    ranked = case["predicate"] == "bounded_knn_rows"
    with rt.B200Scene(s) as scene:
        view = scene.query(q, predicate=case["predicate"], radius=case["options"]["radius"], limit=case["options"]["k_max"])
        got = G.rows_as_tuples(view.to_numpy(), ranked)
        view.close()
    assert got == G.expected_rows(case)


def test_config1_full_matches_reference_rows(gpu):
    z = G.load_config1()
    q, s = G.config1_points()
    view = rt.runtime.fixed_radius_neighbors(
        rt.pack_points(ids=q["id"], x=q["x"], y=q["y"]), rt.pack_points(ids=s["id"], x=s["x"], y=s["y"]),
        radius=0.02, k_max=4096)
    a = view.to_numpy()
    view.close()
    assert len(a) == 20911
    assert np.array_equal(a["query_id"], z["query_id"])
    assert np.array_equal(a["neighbor_id"], z["neighbor_id"])
    assert np.array_equal(a["distance"].view(np.uint64), z["distance"].view(np.uint64))


def _clustered(rng, n, centres, sigma=0.01, background=0.1):
    which = rng.integers(0, len(centres), n)
    pts = centres[which] + rng.normal(0.0, sigma, (n, 3))
    bg = rng.random(n) < background
    pts[bg] = rng.random((int(bg.sum()), 3))
    return np.clip(pts, 0.0, 1.0).astype(np.float32).astype(np.float64)


def _cols(pts, ids=None):
    ids = np.arange(len(pts), dtype=np.uint32) if ids is None else ids
    d = {"id": ids, "x": pts[:, 0], "y": pts[:, 1]}
    if pts.shape[1] == 3:
        d["z"] = pts[:, 2]
    return d


def _pack(c):
    return rt.pack_points(ids=c["id"], x=c["x"], y=c["y"], z=c.get("z"))


def _assert_same_rows(a, b, ranked):
    assert len(a) == len(b)
    for f in ("query_id", "neighbor_id") + (("neighbor_rank",) if ranked else ()):
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["distance"].view(np.uint64), b["distance"].view(np.uint64))


@pytest.mark.parametrize("k_max", [1, 8, 32, 64])
def test_clustered_frn_3d_matches_oracle(gpu, k_max):
    rng = np.random.default_rng(100 + k_max)
    centres = rng.random((16, 3))
    s = _cols(_clustered(rng, 40000, centres))
    q = _cols(_clustered(rng, 6000, centres))
    radius = 0.01
    with rt.B200Scene(_pack(s)) as scene:
        view, overflow = scene.query(_pack(q), predicate="fixed_radius_neighbors", radius=radius, limit=k_max,
                                     with_overflow=True)
        got = view.to_numpy()
        view.close()
    exp, counts = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, threads=8, with_counts=True)
    _assert_same_rows(got, exp, False)
    assert np.array_equal(overflow.astype(bool), counts > k_max)
    assert (counts > k_max).any()


@pytest.mark.parametrize("traversal", ["packet", "packet_cube", "lane", "packet_points", "packet_hybrid"])
def test_every_traversal_matches_oracle(gpu, traversal):
    """Each collect traversal of the tuning knob, on FP32-exact clustered
    points and on FP64 inputs (every candidate takes the exact band test)."""
    rng = np.random.default_rng(31)
    centres = rng.random((12, 3))
    s = _cols(_clustered(rng, 30000, centres))
    q = _cols(_clustered(rng, 5000, centres))
    s64 = _cols(0.25 + rng.random((6000, 3)) * 0.5)
    q64 = _cols(0.25 + rng.random((1500, 3)) * 0.5)
    rt.set_tuning(traversal=traversal)
    try:
        for search, query, radius, k_max in ((s, q, 0.01, 64), (s64, q64, 0.05, 12)):
            with rt.B200Scene(_pack(search)) as scene:
                view, overflow = scene.query(_pack(query), predicate="fixed_radius_neighbors", radius=radius,
                                             limit=k_max, with_overflow=True)
                got = view.to_numpy()
                view.close()
            exp, counts = O.fixed_radius_neighbors(query, search, radius=radius, k_max=k_max, threads=8,
                                                   with_counts=True)
            _assert_same_rows(got, exp, False)
            assert np.array_equal(overflow.astype(bool), counts > k_max)
    finally:
        rt.set_tuning()


@pytest.mark.parametrize("traversal", ["packet", "lane"])
def test_knn_walks_match_oracle(gpu, traversal):
    """The nearest-list walk in warp packets of Morton-consecutive queries
    (default: pre-order for k <= 4 and the Hausdorff nearest, nearer child
    first from k = 5) and one thread per query in Morton order ("lane"): KNN rows and the
    Hausdorff nearest, on clustered 3D sets with a query count that leaves a
    partial last warp, and on a 2D lattice whose equal distances are broken
    by id."""
    rng = np.random.default_rng(33)
    centres = rng.random((10, 3))
    s = _cols(_clustered(rng, 25000, centres))
    q = _cols(_clustered(rng, 4001, centres))
    g = np.stack(np.meshgrid(np.arange(60), np.arange(60)), -1).reshape(-1, 2).astype(np.float64) * 0.5
    s2 = {"id": np.arange(len(g), dtype=np.uint32), "x": g[:, 0], "y": g[:, 1]}
    q2 = {"id": np.arange(720, dtype=np.uint32), "x": g[::5, 0][:720] + 0.25, "y": g[::5, 1][:720]}
    rt.set_tuning(traversal=traversal)
    try:
        for search, query in ((s, q), (s2, q2)):
            with rt.B200Scene(_pack(search)) as scene:
                for k in (1, 3, 4, 16, 40):
                    v = scene.query(_pack(query), predicate="knn_rows", limit=k)
                    _assert_same_rows(v.to_numpy(), O.knn_rows(query, search, k=k, threads=8), True)
                    v.close()
                w = scene.directed_hausdorff(_pack(query))
                exp = O.directed_hausdorff(query, search, threads=8)
                assert (w["distance"], w["source_id"], w["target_id"]) == \
                    (exp["distance"], exp["source_id"], exp["target_id"])
    finally:
        rt.set_tuning()


def test_bounded_knn_and_knn_3d_match_oracle(gpu):
    rng = np.random.default_rng(5)
    centres = rng.random((8, 3))
    s = _cols(_clustered(rng, 30000, centres))
    q = _cols(_clustered(rng, 4000, centres))
    with rt.B200Scene(_pack(s)) as scene:
        v = scene.query(_pack(q), predicate="bounded_knn_rows", radius=0.012, limit=16)
        _assert_same_rows(v.to_numpy(), O.fixed_radius_neighbors(q, s, radius=0.012, k_max=16, ranked=True, threads=8), True)
        v.close()
        for k in (1, 4, 16, 64):
            v = scene.query(_pack(q), predicate="knn_rows", limit=k)
            _assert_same_rows(v.to_numpy(), O.knn_rows(q, s, k=k, threads=8), True)
            v.close()


def test_generic_path_large_limits_match_oracle(gpu):
    rng = np.random.default_rng(9)
    centres = rng.random((4, 3))
    s = _cols(_clustered(rng, 5000, centres, sigma=0.02))
    q = _cols(_clustered(rng, 300, centres, sigma=0.02))
    with rt.B200Scene(_pack(s)) as scene:
        v = scene.query(_pack(q), predicate="fixed_radius_neighbors", radius=0.03, limit=300)
        exp = O.fixed_radius_neighbors(q, s, radius=0.03, k_max=300, threads=8)
        _assert_same_rows(v.to_numpy(), exp, False)
        v.close()
        v = scene.query(_pack(q), predicate="knn_rows", limit=100)
        _assert_same_rows(v.to_numpy(), O.knn_rows(q, s, k=100, threads=8), True)
        v.close()


def test_inexact_fp64_inputs_and_large_coordinates(gpu):
    rng = np.random.default_rng(21)
    for offset, radius in ((0.0, 0.04), (1.0e4, 0.004), (-3.0e6, 0.5)):
        s = _cols(offset + rng.random((5000, 3)) * (0.3 if offset else 1.0))
        q = _cols(offset + rng.random((1500, 3)) * (0.3 if offset else 1.0))
        with rt.B200Scene(_pack(s)) as scene:
            v = scene.query(_pack(q), predicate="fixed_radius_neighbors", radius=radius, limit=20)
            _assert_same_rows(v.to_numpy(), O.fixed_radius_neighbors(q, s, radius=radius, k_max=20, threads=8), False)
            v.close()
            v = scene.query(_pack(q), predicate="knn_rows", limit=5)
            _assert_same_rows(v.to_numpy(), O.knn_rows(q, s, k=5, threads=8), True)
            v.close()


def test_duplicates_ties_unsorted_query_ids_2d(gpu):
    rng = np.random.default_rng(33)
    grid = np.stack(np.meshgrid(np.arange(40), np.arange(40)), -1).reshape(-1, 2).astype(np.float64) * 0.25
    s_pts = np.concatenate([grid, grid[:300]])  # coincident duplicates
    s = _cols(s_pts, ids=rng.integers(0, 500, len(s_pts)).astype(np.uint32))  # duplicate ids too
    q_pts = grid[rng.integers(0, len(grid), 700)] + rng.integers(-1, 2, (700, 2)) * 0.125
    q = _cols(q_pts, ids=rng.integers(0, 300, 700).astype(np.uint32))  # unsorted, repeated query ids
    for radius, k_max in ((0.25, 3), (0.5, 7), (0.0, 4), (0.35355339059327373, 64)):
        v = rt.runtime.fixed_radius_neighbors(_pack(q), _pack(s), radius=radius, k_max=k_max)
        _assert_same_rows(v.to_numpy(), O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, threads=8), False)
        v.close()
    v = rt.runtime.knn_rows(_pack(q), _pack(s), k=9)
    _assert_same_rows(v.to_numpy(), O.knn_rows(q, s, k=9, threads=8), True)
    v.close()


def test_tiny_and_single_point_scenes(gpu):
    for ns in (1, 2, 3, 7, 9, 33):
        rng = np.random.default_rng(ns)
        s = _cols(rng.random((ns, 3)))
        q = _cols(rng.random((50, 3)))
        v = rt.runtime.fixed_radius_neighbors(_pack(q), _pack(s), radius=0.4, k_max=5)
        _assert_same_rows(v.to_numpy(), O.fixed_radius_neighbors(q, s, radius=0.4, k_max=5), False)
        v.close()
        v = rt.runtime.knn_rows(_pack(q), _pack(s), k=4)
        _assert_same_rows(v.to_numpy(), O.knn_rows(q, s, k=4), True)
        v.close()


def test_prepared_fixed_radius_3d_matches_direct(gpu):
    rng = np.random.default_rng(4)
    s = _cols(rng.random((20000, 3)).astype(np.float32).astype(np.float64))
    q = _cols(rng.random((3000, 3)).astype(np.float32).astype(np.float64))
    prepared = rt.prepare_b200_fixed_radius_neighbors_3d(_pack(s), max_radius=0.05)
    try:
        for radius in (0.02, 0.05):
            v = prepared.run_raw(_pack(q), radius=radius, k_max=16)
            _assert_same_rows(v.to_numpy(), O.fixed_radius_neighbors(q, s, radius=radius, k_max=16, threads=8), False)
            v.close()
        with pytest.raises(ValueError):
            prepared.run(_pack(q), radius=0.06, k_max=4)
    finally:
        prepared.close()


def test_rt_run_facade_and_raw_mode(gpu):
    case = next(c for c in CASES if c["name"] == "authored_frn_3d")
    kernel = _kernel("fixed_radius_neighbors", 3, **case["options"])
    q = G.points_records(case["query_points"], 3)
    s = G.points_records(case["search_points"], 3)
    result = rt.run(kernel, {"query_points": q, "search_points": s}, execution=rt.ExecutionPolicy(backend="b200"))
    assert _as_tuples(result.rows, False) == G.expected_rows(case)
    assert result.execution_report.accel_kind == "lbvh"
    raw = rt.run_b200(kernel, result_mode="raw", query_points=q, search_points=s)
    try:
        assert raw.to_tuple_rows() == tuple(G.expected_rows(case))
    finally:
        raw.close()
    prepared = rt.prepare_b200(kernel)
    assert prepared.run(query_points=q, search_points=s) == rt.run_b200(kernel, query_points=q, search_points=s)


def test_phase_timings_reported(gpu):
    rng = np.random.default_rng(1)
    s = _cols(rng.random((5000, 3)))
    v = rt.runtime.fixed_radius_neighbors(_pack(s), _pack(s), radius=0.05, k_max=8)
    v.close()
    t = rt.last_phase_timings()
    for phase in ("upload", "build", "traverse", "emit", "download", "total"):
        assert phase in t and t[phase] >= 0.0


def test_lattice_shell_ties_at_the_cut(gpu):
    """Integer points on the shells |v|^2 = 25, 26, 27 around each query give
    groups of exactly equal FP64 distances; with 65..128 candidates per query
    the k_max cut falls inside a tie group, which must be broken by neighbor id
    and then search input order, exactly as the reference sorts."""
    rng = np.random.default_rng(8)
    r = np.arange(-6, 7)
    grid = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    shell = grid[np.isin((grid ** 2).sum(1), (25, 26, 27))].astype(np.float64)
    centres = np.array([[0.0, 0.0, 0.0], [40.0, 0.0, 0.0], [0.0, 40.0, 0.0]])
    pts = np.concatenate([c + shell for c in centres])
    order = rng.permutation(len(pts))
    pts = pts[order]
    s = _cols(pts, ids=(rng.integers(0, 60, len(pts))).astype(np.uint32))  # many duplicate ids
    q = _cols(centres, ids=np.array([7, 3, 5], dtype=np.uint32))
    # radius^2 = 26: 102 candidates per query, 27: 134 (both on the warp-per-query emit)
    for r2, per_query in ((26.0, 102), (27.0, 134)):
        radius = float(np.nextafter(np.sqrt(r2), np.inf))  # radius * radius >= r2 in FP64
        for k_max in (10, 30, 40, 64, 100):
            with rt.B200Scene(_pack(s)) as scene:
                v, overflow = scene.query(_pack(q), predicate="fixed_radius_neighbors", radius=radius,
                                          limit=k_max, with_overflow=True)
                got = v.to_numpy()
                v.close()
            exp, counts = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, with_counts=True)
            assert (counts == per_query).all()
            _assert_same_rows(got, exp, False)
            assert np.array_equal(overflow.astype(bool), counts > k_max)


def test_lattice_ball_generic_path(gpu):
    """All integer points with |v|^2 <= 50 around each query (about 1,500
    candidates, many exactly equal distances): more candidates than the
    per-query slab holds, so the generic path decides the k_max nearest."""
    rng = np.random.default_rng(18)
    r = np.arange(-8, 9)
    grid = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    ball = grid[(grid ** 2).sum(1) <= 50].astype(np.float64)
    centres = np.array([[0.0, 0.0, 0.0], [100.0, 0.0, 0.0]])
    pts = np.concatenate([c + ball for c in centres])[rng.permutation(2 * len(ball))]
    s = _cols(pts, ids=rng.integers(0, 200, len(pts)).astype(np.uint32))
    q = _cols(centres, ids=np.array([1, 0], dtype=np.uint32))
    radius = float(np.nextafter(np.sqrt(50.0), np.inf))
    for k_max in (1, 17, 64):
        v, = [rt.runtime.fixed_radius_neighbors(_pack(q), _pack(s), radius=radius, k_max=k_max)]
        exp, counts = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, with_counts=True)
        assert (counts > 256).all()
        _assert_same_rows(v.to_numpy(), exp, False)
        v.close()


@pytest.mark.parametrize("dim,k_max", [(3, 64), (3, 7), (2, 16), (3, 200)])
def test_device_per_call_entry_matches_oracle(gpu, dim, k_max):
    """rtdl_b200_run_fixed_radius_neighbors_device (build + query in one call on resident records; the
    probe set is prepared beside the build for k_max <= 64): rows, counts and overflow flags."""
    import torch

    from rtdl_b200.runtime import FRN_ROW_DTYPE

    rng = np.random.default_rng(40 + dim + k_max)
    centres = rng.random((12, 3))
    s_pts, q_pts = _clustered(rng, 30000, centres)[:, :dim], _clustered(rng, 5000, centres)[:, :dim]
    # query ids out of order: rows must still come grouped by ascending query id
    s, q = _cols(s_pts), _cols(q_pts, ids=rng.permutation(len(q_pts)).astype(np.uint32) * 3)
    sp, qp = _pack(s), _pack(q)
    d_s = torch.from_numpy(sp.records.view(np.uint8).copy()).cuda()
    d_q = torch.from_numpy(qp.records.view(np.uint8).copy()).cuda()
    radius = 0.012
    n = rt.runtime.fixed_radius_neighbors_device(d_q.data_ptr(), len(q_pts), d_s.data_ptr(), len(s_pts),
                                                 dimension=dim, radius=radius, k_max=k_max, rows_address=None,
                                                 rows_capacity=0)
    rows = torch.empty(max(n, 1) * 16, dtype=torch.uint8, device="cuda")
    flags = torch.empty(len(q_pts), dtype=torch.uint8, device="cuda")
    assert rt.runtime.fixed_radius_neighbors_device(d_q.data_ptr(), len(q_pts), d_s.data_ptr(), len(s_pts),
                                                    dimension=dim, radius=radius, k_max=k_max,
                                                    rows_address=rows.data_ptr(), rows_capacity=n,
                                                    overflow_address=flags.data_ptr()) == n
    got = np.frombuffer(rows.cpu().numpy().tobytes(), dtype=FRN_ROW_DTYPE)[:n]
    exp, counts = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, threads=8, with_counts=True)
    _assert_same_rows(got, exp, False)
    assert np.array_equal(flags.cpu().numpy().astype(bool), counts > k_max)
    # no search points: no rows, flags cleared
    flags.fill_(7)
    assert rt.runtime.fixed_radius_neighbors_device(d_q.data_ptr(), len(q_pts), d_s.data_ptr(), 0, dimension=dim,
                                                    radius=radius, k_max=k_max, rows_address=rows.data_ptr(),
                                                    rows_capacity=n, overflow_address=flags.data_ptr()) == 0
    assert int(flags.max()) == 0


def test_device_rows_path_heavy_and_generic_queries(gpu):
    """Rows into a caller's device buffer take the refinement on device counts: queries with more than
    256 candidates (a dense cluster) and queries no radius separates (400 coincident points) must still
    get the oracle's rows, through the per-call device entry and a resident scene."""
    import torch

    from rtdl_b200.runtime import FRN_ROW_DTYPE

    rng = np.random.default_rng(8)
    dense = rng.normal(0.5, 0.01, (30000, 3))
    same = np.full((400, 3), 0.25)
    s_pts = np.concatenate([dense, same, rng.random((20000, 3))]).astype(np.float32).astype(np.float64)
    q_pts = np.concatenate([rng.normal(0.5, 0.01, (3000, 3)), np.full((7, 3), 0.25),
                            rng.random((2000, 3))]).astype(np.float32).astype(np.float64)
    s, q = _cols(s_pts), _cols(q_pts)
    d_s = torch.from_numpy(_pack(s).records.view(np.uint8).copy()).cuda()
    d_q = torch.from_numpy(_pack(q).records.view(np.uint8).copy()).cuda()
    for radius, k_max in ((0.01, 40), (0.004, 64), (0.02, 5)):
        exp = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, threads=8)
        n = len(exp)
        rows = torch.empty(max(n, 1) * 16, dtype=torch.uint8, device="cuda")
        assert rt.runtime.fixed_radius_neighbors_device(d_q.data_ptr(), len(q_pts), d_s.data_ptr(), len(s_pts),
                                                        dimension=3, radius=radius, k_max=k_max,
                                                        rows_address=rows.data_ptr(), rows_capacity=n) == n
        got = np.frombuffer(rows.cpu().numpy().tobytes(), dtype=FRN_ROW_DTYPE)[:n]
        _assert_same_rows(got, exp, False)
        with rt.B200Scene(_pack(s)) as scene:
            rows.zero_()
            assert scene.query_device(d_q.data_ptr(), len(q_pts), predicate="fixed_radius_neighbors", radius=radius,
                                      limit=k_max, rows_address=rows.data_ptr(), rows_capacity=n) == n
            got = np.frombuffer(rows.cpu().numpy().tobytes(), dtype=FRN_ROW_DTYPE)[:n]
            _assert_same_rows(got, exp, False)


@pytest.mark.parametrize("dim,ranked,k_max", [(3, False, 8), (3, False, 64), (3, True, 16), (2, False, 64), (2, True, 5)])
def test_plain_call_rows_copied_range_by_range(gpu, dim, ranked, k_max):
    """The plain per-call launch with 8,192 queries or more copies its rows to
    the host range by range (eight ranges of queries in output order) while
    later ranges are emitted.  Clustered queries give every emission kind
    (warp lists, 65..kSlab lists, deferred fix-ups, refined heavy queries);
    the first three eighths of the queries lie far from every point, so their
    ranges hold no rows; coincident copies of a few points reach the generic
    path."""
    rng = np.random.default_rng(200 + 7 * k_max + dim)
    centres = rng.random((12, dim if dim == 3 else 3))
    s_pts = _clustered(rng, 60000, centres)[:, :dim]
    s_pts = np.concatenate([s_pts, np.repeat(s_pts[:3], 300, axis=0)])  # 301 copies of three points
    q_pts = _clustered(rng, 24000, centres)[:, :dim]
    q_pts[: 24000 * 3 // 8] += 5.0  # no neighbours
    q_pts[-100:] = s_pts[np.arange(100) % 3]  # queries on the coincident copies
    s, q = _cols(s_pts), _cols(q_pts)
    radius = 0.012
    v = rt.runtime.fixed_radius_neighbors(_pack(q), _pack(s), radius=radius, k_max=k_max, ranked=ranked)
    got = v.to_numpy()
    v.close()
    exp = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, ranked=ranked, threads=8, grid=True)
    _assert_same_rows(got, exp, ranked)
    assert got["query_id"].min() >= 24000 * 3 // 8


@pytest.mark.parametrize("dim,ranked,k_max", [(3, False, 64), (3, True, 12), (2, False, 32)])
def test_plain_call_query_ranges(gpu, dim, ranked, k_max):
    """From 262,144 queries on, the plain per-call launch answers its queries
    in ranges of their input order (here three) and copies each range's rows
    to the host while the next range runs.  Rows must equal the oracle's
    across the range boundaries: ranges of different sizes (the count is not
    a multiple of three), a stretch of queries without neighbours across a
    boundary, dense clusters with list queries and refined heavy queries,
    and queries on coincident points that reach the generic path."""
    rng = np.random.default_rng(314 + k_max + dim)
    centres = rng.random((16, 3))
    s_pts = _clustered(rng, 120000, centres)[:, :dim]
    s_pts = np.concatenate([s_pts, np.repeat(s_pts[:2], 400, axis=0)])  # 401 copies of two points
    nq = 400003
    q_pts = _clustered(rng, nq, centres)[:, :dim]
    q_pts[nq // 4: nq // 2] += 5.0  # no neighbours, across the first range boundary
    q_pts[-50:] = s_pts[np.arange(50) % 2]  # queries on the coincident copies
    s, q = _cols(s_pts), _cols(q_pts)
    radius = 0.01 if dim == 3 else 0.002
    v = rt.runtime.fixed_radius_neighbors(_pack(q), _pack(s), radius=radius, k_max=k_max, ranked=ranked)
    got = v.to_numpy()
    v.close()
    exp = O.fixed_radius_neighbors(q, s, radius=radius, k_max=k_max, ranked=ranked, threads=8, grid=True)
    _assert_same_rows(got, exp, ranked)
