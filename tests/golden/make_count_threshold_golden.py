"""Writes tests/golden/count_threshold_2d.json with rows from the reference's
own generic CPU count (run here, where the reference tree exists):

    python tests/golden/make_count_threshold_golden.py <reference tree>

The cases are small seeded 2-D sets (a lattice whose spacing puts points
exactly on the radius, duplicates, ids out of order) counted by
``rtdsl.generic_primitives._cpu_fixed_radius_count_threshold_rows`` at
several thresholds.  The oracle restatement (``oracle.fixed_radius_count_threshold``)
is checked against these rows on the CPU, and the CUDA path against the oracle.
"""
import json
import sys
from collections import namedtuple
from pathlib import Path

import numpy as np

P = namedtuple("P", "id x y")


def cases():
    rng = np.random.default_rng(77)
    grid = np.stack(np.meshgrid(np.arange(12), np.arange(12)), -1).reshape(-1, 2).astype(np.float64) * 0.25
    out = []
    # lattice with duplicates: radius 0.25 and 0.5 fall exactly on lattice distances
    s = np.concatenate([grid, grid[:30]])
    s_ids = rng.permutation(len(s)).astype(np.uint32) * 3
    q = grid[rng.integers(0, len(grid), 60)] + rng.integers(-1, 2, (60, 2)) * 0.125
    q_ids = rng.integers(0, 40, 60).astype(np.uint32)
    for radius in (0.25, 0.5, 0.0):
        for threshold in (0, 1, 3, 8):
            out.append(("lattice", s, s_ids, q, q_ids, radius, threshold))
    # uniform points
    s = rng.random((400, 2))
    q = rng.random((120, 2))
    for threshold in (0, 2, 10):
        out.append(("uniform", s, np.arange(400, dtype=np.uint32), q, np.arange(120, dtype=np.uint32) + 1000, 0.07,
                    threshold))
    return out


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from rtdsl.generic_primitives import _cpu_fixed_radius_count_threshold_rows

    result = []
    for name, s, s_ids, q, q_ids, radius, threshold in cases():
        search = [P(int(i), float(x), float(y)) for i, (x, y) in zip(s_ids, s)]
        query = [P(int(i), float(x), float(y)) for i, (x, y) in zip(q_ids, q)]
        rows = _cpu_fixed_radius_count_threshold_rows(query, search, radius=radius, threshold=threshold)
        result.append({
            "name": name, "radius": radius, "threshold": threshold,
            "search": {"id": s_ids.tolist(), "x": s[:, 0].tolist(), "y": s[:, 1].tolist()},
            "query": {"id": q_ids.tolist(), "x": q[:, 0].tolist(), "y": q[:, 1].tolist()},
            "rows": [[r["query_id"], r["neighbor_count"], r["threshold_reached"]] for r in rows],
        })
    out = Path(__file__).resolve().parent / "count_threshold_2d.json"
    out.write_text(json.dumps({"source": "rtdsl/generic_primitives.py:198-227", "cases": result}))
    print(out, len(result))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    else:
        sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
        from oracle.oracle import reference_root

        if reference_root() is None:
            raise SystemExit("give the reference tree as the argument or set RTDL_REFERENCE_ROOT")
        main(str(reference_root()))
