"""Generate golden fixtures by running the reference's own ``cpu_python_reference``.

Run in a container where the rubaolee/rtdl tree is present (located by
``oracle.reference_root()``: ``RTDL_REFERENCE_ROOT``, else the build
container's read-only mount)::

    python tests/golden/make_golden.py

It writes ``cases.json.gz`` (small authored and seeded cases, every float stored as
``float.hex`` so the fixture is bit-exact), ``config1_frn_2d.npz`` (the
4,096 x 4,096 2D fixed-radius case, radius 0.02, seed 0) and ``hausdorff.json``.
The fixtures are what the CPU tests pin the oracle against and what the GPU
tests compare the CUDA backend with; the reference itself is never needed at
test time.

Authored cases come from the reference's own tests:
  tests/goal198_fixed_radius_neighbors_truth_path_test.py:20-101
  tests/goal204_knn_rows_truth_path_test.py
  tests/goal311_v0_5_optix_3d_nn_test.py:41-53
  examples/reference/rtdl_fixed_radius_neighbors_reference.py:23-36
  examples/v2_0/research_benchmarks/hausdorff_xhd/rtdl_hausdorff_distance_app.py:28-54
"""
from __future__ import annotations

import gzip
import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from oracle.oracle import reference_root  # noqa: E402

REF = reference_root()
if REF is None:
    raise SystemExit("the reference tree is not present: set RTDL_REFERENCE_ROOT")
sys.path.insert(0, str(REF / "src"))
sys.path.insert(0, str(REF))

import rtdsl as rt  # noqa: E402

OUT = Path(__file__).resolve().parent


def _kernel(predicate: str, dim: int, **options):
    geometry = rt.Points3D if dim == 3 else rt.Points
    fields = ["query_id", "neighbor_id", "distance"]
    if predicate != "fixed_radius_neighbors":
        fields.append("neighbor_rank")

    @rt.kernel(backend="rtdl", precision="float_approx")
    def golden_kernel():
        q = rt.input("query_points", geometry, role="probe")
        s = rt.input("search_points", geometry, role="build")
        c = rt.traverse(q, s, accel="bvh")
        pred = getattr(rt, predicate)(**options)
        hits = rt.refine(c, predicate=pred)
        return rt.emit(hits, fields=fields)

    return golden_kernel


def _pt(dim, i, x, y, z=0.0):
    if dim == 3:
        return rt.Point3D(id=int(i), x=float(x), y=float(y), z=float(z))
    return rt.Point(id=int(i), x=float(x), y=float(y))


def _enc_points(points, dim):
    out = []
    for p in points:
        row = [int(p.id), float(p.x).hex(), float(p.y).hex()]
        if dim == 3:
            row.append(float(p.z).hex())
        out.append(row)
    return out


def _case(name, predicate, dim, query, search, **options):
    kernel = _kernel(predicate, dim, **options)
    rows = rt.run_cpu_python_reference(kernel, query_points=query, search_points=search)
    enc_rows = []
    for r in rows:
        row = [int(r["query_id"]), int(r["neighbor_id"]), float(r["distance"]).hex()]
        if "neighbor_rank" in r:
            row.append(int(r["neighbor_rank"]))
        enc_rows.append(row)
    print(f"{name}: {len(query)} x {len(search)} -> {len(rows)} rows")
    return {
        "name": name,
        "predicate": predicate,
        "options": options,
        "dimension": dim,
        "query_points": _enc_points(query, dim),
        "search_points": _enc_points(search, dim),
        "rows": enc_rows,
    }


def _clustered(rng, n, dim, centres, sigma, background):
    pts = np.empty((n, dim))
    is_bg = rng.random(n) < background
    which = rng.integers(0, len(centres), n)
    pts[:] = centres[which] + rng.normal(0.0, sigma, (n, dim))
    pts[is_bg] = rng.random((int(is_bg.sum()), dim))
    return np.clip(pts, 0.0, 1.0).astype(np.float32).astype(np.float64)


def main():
    cases = []
    authored_q = (_pt(2, 100, 0.0, 0.0), _pt(2, 101, 3.0, 0.0))
    authored_s = (_pt(2, 1, 0.0, 0.0), _pt(2, 2, 0.3, 0.0), _pt(2, 3, -0.3, 0.0), _pt(2, 4, 3.2, 0.0), _pt(2, 5, 4.0, 0.0))
    cases.append(_case("authored_frn_2d", "fixed_radius_neighbors", 2, authored_q, authored_s, radius=0.5, k_max=3))
    cases.append(_case("authored_knn_2d", "knn_rows", 2, authored_q, authored_s, k=3))
    cases.append(_case("authored_bounded_2d", "bounded_knn_rows", 2, authored_q, authored_s, radius=0.5, k_max=3))
    cases.append(_case("grouped_by_query_id_2d", "fixed_radius_neighbors", 2,
                       (_pt(2, 20, 3.0, 0.0), _pt(2, 10, 0.0, 0.0)), (_pt(2, 1, 0.0, 0.0), _pt(2, 2, 3.0, 0.0)),
                       radius=0.1, k_max=2))
    cases.append(_case("zero_radius_2d", "fixed_radius_neighbors", 2,
                       (_pt(2, 10, 1.0, 1.0),), (_pt(2, 1, 1.0, 1.0), _pt(2, 2, 1.0, 1.0001)), radius=0.0, k_max=4))
    q3 = (_pt(3, 10, 0.0, 0.0, 0.0), _pt(3, 20, 5.0, 0.0, 0.0))
    s3 = (_pt(3, 1, 0.0, 0.0, 0.0), _pt(3, 2, 0.0, 0.0, 0.6), _pt(3, 3, 0.0, 0.8, 0.0), _pt(3, 4, 5.0, 0.0, 0.9))
    cases.append(_case("authored_frn_3d", "fixed_radius_neighbors", 3, q3, s3, radius=1.0, k_max=2))
    cases.append(_case("authored_bounded_3d", "bounded_knn_rows", 3, q3, s3, radius=1.0, k_max=2))
    cases.append(_case("authored_knn_3d", "knn_rows", 3, q3, s3, k=2))
    cases.append(_case("authored_frn_3d_kmax3", "fixed_radius_neighbors", 3, q3, s3, radius=1.0, k_max=3))

    # Ties: equal distances broken by id, duplicate ids broken by input order,
    # coincident points, duplicate query ids out of order.
    tie_s = tuple(_pt(3, i_id, x, y, z) for i_id, (x, y, z) in zip(
        (7, 3, 5, 3, 9, 1, 1, 8),
        ((1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (0, 0, -1), (0.5, 0, 0))))
    tie_q = (_pt(3, 42, 0, 0, 0), _pt(3, 7, 0, 0, 0), _pt(3, 42, 0.5, 0, 0))
    for kmax in (1, 2, 3, 5, 8):
        cases.append(_case(f"ties_frn_3d_k{kmax}", "fixed_radius_neighbors", 3, tie_q, tie_s, radius=1.0, k_max=kmax))
    cases.append(_case("ties_knn_3d_k4", "knn_rows", 3, tie_q, tie_s, k=4))
    cases.append(_case("ties_knn_3d_k20", "knn_rows", 3, tie_q, tie_s, k=20))
    cases.append(_case("ties_bounded_3d_k3", "bounded_knn_rows", 3, tie_q, tie_s, radius=1.0, k_max=3))

    rng = np.random.default_rng(12345)
    # Seeded 2D uniform float64 (config-1 shape, smaller).
    b = rng.random((700, 2)); p = rng.random((600, 2))
    s2 = tuple(_pt(2, i, *b[i]) for i in range(len(b)))
    q2 = tuple(_pt(2, 1000 + i, *p[i]) for i in range(len(p)))
    cases.append(_case("uniform_frn_2d_f64", "fixed_radius_neighbors", 2, q2, s2, radius=0.05, k_max=4096))
    cases.append(_case("uniform_frn_2d_f64_kmax3", "fixed_radius_neighbors", 2, q2, s2, radius=0.05, k_max=3))
    cases.append(_case("uniform_knn_2d_f64_k5", "knn_rows", 2, q2, s2, k=5))

    # Seeded 3D clustered float32 values (config-2 shape, smaller): overflow beyond k_max.
    centres = rng.random((8, 3))
    bs = _clustered(rng, 800, 3, centres, 0.02, 0.1)
    ps = _clustered(rng, 500, 3, centres, 0.02, 0.1)
    s3c = tuple(_pt(3, i, *bs[i]) for i in range(len(bs)))
    q3c = tuple(_pt(3, i, *ps[i]) for i in range(len(ps)))
    cases.append(_case("clustered_frn_3d_f32_k8", "fixed_radius_neighbors", 3, q3c, s3c, radius=0.03, k_max=8))
    cases.append(_case("clustered_frn_3d_f32_k64", "fixed_radius_neighbors", 3, q3c, s3c, radius=0.03, k_max=64))
    cases.append(_case("clustered_bounded_3d_f32_k8", "bounded_knn_rows", 3, q3c, s3c, radius=0.03, k_max=8))
    cases.append(_case("clustered_knn_3d_f32_k16", "knn_rows", 3, q3c, s3c, k=16))
    cases.append(_case("clustered_knn_3d_f32_k1", "knn_rows", 3, q3c, s3c, k=1))

    # Large coordinates with a small radius: the float32 candidate filter must
    # not lose boundary rows (the reference's Goal 229 regression).
    off = 1.0e4
    bl = off + rng.random((400, 3)) * 0.05
    pl = off + rng.random((300, 3)) * 0.05
    cases.append(_case("large_coords_frn_3d_f64", "fixed_radius_neighbors", 3,
                       tuple(_pt(3, i, *pl[i]) for i in range(len(pl))),
                       tuple(_pt(3, i, *bl[i]) for i in range(len(bl))), radius=0.004, k_max=16))
    # Points exactly on the radius (inclusive boundary).
    ring = tuple(_pt(2, i, np.cos(t), np.sin(t)) for i, t in enumerate(np.linspace(0, 2 * np.pi, 24, endpoint=False)))
    axis = (_pt(2, 100, 1.0, 0.0), _pt(2, 101, 0.0, 1.0), _pt(2, 102, -1.0, 0.0), _pt(2, 103, 0.0, -1.0),
            _pt(2, 104, 0.75, 0.0), _pt(2, 105, 0.5, 0.5))
    cases.append(_case("on_radius_2d", "fixed_radius_neighbors", 2, (_pt(2, 0, 0.0, 0.0), _pt(2, 1, 0.25, 0.0)),
                       ring + axis, radius=1.0, k_max=64))
    cases.append(_case("empty_result_2d", "fixed_radius_neighbors", 2, (_pt(2, 0, 10.0, 10.0),), axis, radius=0.1, k_max=4))

    with gzip.open(OUT / "cases.json.gz", "wt") as fh:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, fh, separators=(",", ":"))

    # Config 1 (full size): 4,096 x 4,096 2D, float64 uniform, seed 0, radius 0.02.
    rng0 = np.random.default_rng(0)
    build = rng0.random((4096, 2))
    probe = rng0.random((4096, 2))
    c1 = _case("config1_frn_2d", "fixed_radius_neighbors", 2,
               tuple(_pt(2, i, *probe[i]) for i in range(4096)),
               tuple(_pt(2, i, *build[i]) for i in range(4096)), radius=0.02, k_max=4096)
    rows = c1["rows"]
    np.savez_compressed(
        OUT / "config1_frn_2d.npz",
        query_id=np.array([r[0] for r in rows], dtype=np.uint32),
        neighbor_id=np.array([r[1] for r in rows], dtype=np.uint32),
        distance=np.array([float.fromhex(r[2]) for r in rows], dtype=np.float64),
        seed=np.array(0), radius=np.array(0.02), k_max=np.array(4096), n=np.array(4096),
    )

    # Hausdorff app (authored sets, copies 1 and 3).
    app_path = REF / "examples" / "v2_0" / "research_benchmarks" / "hausdorff_xhd" / "rtdl_hausdorff_distance_app.py"
    spec = importlib.util.spec_from_file_location("rtdl_hausdorff_app", app_path)
    app = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(app)
    hd = []
    for copies in (1, 3):
        result = app.run_app("cpu_python_reference", copies)
        sets = app.make_authored_point_sets(copies=copies)
        hd.append({
            "copies": copies,
            "points_a": _enc_points(sets["points_a"], 2),
            "points_b": _enc_points(sets["points_b"], 2),
            "directed_a_to_b": {k: result["directed_a_to_b"][k] for k in ("distance", "source_id", "target_id", "row_count")},
            "directed_b_to_a": {k: result["directed_b_to_a"][k] for k in ("distance", "source_id", "target_id", "row_count")},
            "hausdorff_distance": result["hausdorff_distance"],
            "witness_direction": result["witness_direction"],
        })
        for key in ("directed_a_to_b", "directed_b_to_a"):
            hd[-1][key]["distance"] = float(hd[-1][key]["distance"]).hex()
        hd[-1]["hausdorff_distance"] = float(hd[-1]["hausdorff_distance"]).hex()
    (OUT / "hausdorff.json").write_text(json.dumps({"generator": "tests/golden/make_golden.py", "cases": hd}, indent=1))


if __name__ == "__main__":
    main()
