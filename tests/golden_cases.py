"""Loads the golden fixtures written by tests/golden/make_golden.py (the reference's
own cpu_python_reference output) and converts them to numpy and to records."""
from __future__ import annotations

import gzip
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_cases():
    with gzip.open(GOLDEN / "cases.json.gz", "rt") as fh:
        return json.load(fh)["cases"]


def points_columns(encoded, dim):
    ids = np.array([p[0] for p in encoded], dtype=np.uint32)
    cols = {"id": ids, "x": np.array([float.fromhex(p[1]) for p in encoded]), "y": np.array([float.fromhex(p[2]) for p in encoded])}
    if dim == 3:
        cols["z"] = np.array([float.fromhex(p[3]) for p in encoded])
    return cols


def points_records(encoded, dim):
    import rtdl_b200 as rt

    if dim == 3:
        return tuple(rt.Point3D(id=p[0], x=float.fromhex(p[1]), y=float.fromhex(p[2]), z=float.fromhex(p[3])) for p in encoded)
    return tuple(rt.Point(id=p[0], x=float.fromhex(p[1]), y=float.fromhex(p[2])) for p in encoded)


def expected_rows(case):
    """Rows as tuples (query_id, neighbor_id, distance[, neighbor_rank]) in reference order."""
    out = []
    for r in case["rows"]:
        t = (r[0], r[1], float.fromhex(r[2]))
        if len(r) > 3:
            t = t + (r[3],)
        out.append(t)
    return out


def rows_as_tuples(arr, ranked):
    if ranked:
        return list(zip(arr["query_id"].tolist(), arr["neighbor_id"].tolist(), arr["distance"].tolist(), arr["neighbor_rank"].tolist()))
    return list(zip(arr["query_id"].tolist(), arr["neighbor_id"].tolist(), arr["distance"].tolist()))


def load_config1():
    z = np.load(GOLDEN / "config1_frn_2d.npz")
    return z


def config1_points():
    rng = np.random.default_rng(0)
    build = rng.random((4096, 2))
    probe = rng.random((4096, 2))
    q = {"id": np.arange(4096, dtype=np.uint32), "x": probe[:, 0], "y": probe[:, 1]}
    s = {"id": np.arange(4096, dtype=np.uint32), "x": build[:, 0], "y": build[:, 1]}
    return q, s


def load_hausdorff():
    return json.loads((GOLDEN / "hausdorff.json").read_text())["cases"]
