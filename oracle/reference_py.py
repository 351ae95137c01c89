"""Pure-Python restatement of the reference's ``cpu_python_reference`` neighbor rows.

TEST INFRASTRUCTURE ONLY: the timed stand-in for the reference's Python
runner on machines where the reference tree is absent (the GPU machines), used
by ``bench.py --workload config1`` and pinned by ``tests/test_oracle_golden.py``
to rows the reference itself produced.  The product never imports it.

It follows ``src/rtdsl/reference.py`` of rubaolee/rtdl line by line in
algorithm and arithmetic, in plain Python loops over point records:

* ``_point_distance_sq`` (``reference.py:882-890``): ``dx = right.x - left.x``
  (search minus query), ``dx*dx + dy*dy + dz*dz`` evaluated left to right in
  FP64, 2D points with z = 0.0;
* ``fixed_radius_neighbors_cpu`` (``reference.py:349-376``): candidates with
  ``d2 <= radius * radius``, sorted by ``(sqrt(d2), id)`` with Python's stable
  sort, the first ``k_max`` kept, then a stable sort of all rows by
  ``query_id``;
* ``knn_rows_cpu`` (``reference.py:379-403``) and ``bounded_knn_rows_cpu``
  (``reference.py:406-434``): the same key, ranks from 1.
"""
from __future__ import annotations

import math
from collections import namedtuple

Point = namedtuple("Point", "id x y")
Point3D = namedtuple("Point3D", "id x y z")


def points(records) -> tuple:
    """Structured numpy records (id, x, y[, z]) -> a tuple of point records."""
    names = records.dtype.names
    ids = records["id"].tolist()
    xs = records["x"].tolist()
    ys = records["y"].tolist()
    if "z" in names:
        return tuple(Point3D(i, x, y, z) for i, x, y, z in zip(ids, xs, ys, records["z"].tolist()))
    return tuple(Point(i, x, y) for i, x, y in zip(ids, xs, ys))


def _distance_sq(left, right) -> float:
    dx = right.x - left.x
    dy = right.y - left.y
    dz = getattr(right, "z", 0.0) - getattr(left, "z", 0.0)
    return dx * dx + dy * dy + dz * dz


def fixed_radius_neighbors(query_points, search_points, *, radius: float, k_max: int, ranked: bool = False) -> list:
    rows = []
    radius_sq = radius * radius
    for q in query_points:
        candidates = []
        for s in search_points:
            d2 = _distance_sq(q, s)
            if d2 > radius_sq:
                continue
            candidates.append((math.sqrt(d2), s.id))
        candidates.sort(key=lambda item: (item[0], item[1]))
        for rank, (distance, nid) in enumerate(candidates[:k_max], start=1):
            row = {"query_id": q.id, "neighbor_id": nid, "distance": distance}
            if ranked:
                row["neighbor_rank"] = rank
            rows.append(row)
    rows.sort(key=lambda row: row["query_id"])
    return rows


def knn_rows(query_points, search_points, *, k: int) -> list:
    rows = []
    for q in query_points:
        candidates = [(math.sqrt(_distance_sq(q, s)), s.id) for s in search_points]
        candidates.sort(key=lambda item: (item[0], item[1]))
        for rank, (distance, nid) in enumerate(candidates[:k], start=1):
            rows.append({"query_id": q.id, "neighbor_id": nid, "distance": distance, "neighbor_rank": rank})
    rows.sort(key=lambda row: row["query_id"])
    return rows
