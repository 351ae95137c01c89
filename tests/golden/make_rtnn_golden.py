"""Writes tests/golden/rtnn_ranked_summary_262144.json from the reference's own
published ranked-summary report (run here, where the reference tree exists):

    python tests/golden/make_rtnn_golden.py <reference tree>

For each distribution it keeps the seed and sizes, the aggregate of the
reference's CuPy grid opponent and of its OptiX float32 path, and the median
times of both, as recorded on an RTX A5000.  It also adds the oracle's
aggregate of the same set (regenerated with rtdl_b200.workloads.rtnn_points,
coordinates cast to float32 as the published runs fed them, exact FP64
distances), the value the library must reproduce bit for bit.
"""
import json
import os
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))

REPORT = "docs/reports/goal2920_hausdorff_rtnn_large_probe_pod/rtnn_262144_repeat9.json"


def oracle_aggregate(distribution: str, n: int, seed: int, radius: float, k_max: int) -> dict:
    from oracle import oracle as O
    from rtdl_b200 import workloads

    pts = workloads.rtnn_points(distribution, n, seed)
    for c in ("x", "y", "z"):
        pts[c] = pts[c].astype(np.float32).astype(np.float64)
    _, agg = O.ranked_summaries(pts, pts, radius=radius, k_max=k_max, threads=os.cpu_count() or 1)
    return agg


def main(ref_root: str) -> None:
    src = json.loads((Path(ref_root) / REPORT).read_text())
    out = {"source": REPORT, "radius": src["radius"], "k_max": src["k_max"], "gpu": src.get("gpu"),
           "distributions": {}}
    for row in src["rows"]:
        out["distributions"][row["distribution"]] = {
            "seed": row["generated"]["seed"],
            "point_count": row["generated"]["point_count"],
            "query_count": row["query_count"],
            "exact_aggregate": {k: v for k, v in row["cupy_grid_summary"].items() if k != "row_count"},
            "float32_aggregate": {k: v for k, v in row["rtdl_ranked_aggregate_summary"].items() if k != "row_count"},
            "reference_median_s": row["rtdl_elapsed_sec"],
            "cupy_grid_median_s": row["cupy_grid_elapsed_sec"],
            "reference_mode": row["rtdl_phase_summary"]["modes"],
            "oracle_aggregate": oracle_aggregate(row["distribution"], row["generated"]["point_count"],
                                                 row["generated"]["seed"], src["radius"], src["k_max"]),
        }
    dst = Path(__file__).with_name("rtnn_ranked_summary_262144.json")
    dst.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    else:
        sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
        from oracle.oracle import reference_root

        if reference_root() is None:
            raise SystemExit("give the reference tree as the argument or set RTDL_REFERENCE_ROOT")
        main(str(reference_root()))
