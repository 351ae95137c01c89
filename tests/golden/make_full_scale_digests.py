"""Digests of the full-size benchmark row sets, computed by the oracle on the CPU.

    python tests/golden/make_full_scale_digests.py [--threads N]

Writes ``full_scale_digests.json``, which the GPU tests and ``bench.py`` compare
the CUDA path's complete outputs with (every row of every query, not a sample):

* ``frn_1m``: fixed_radius_neighbors over the 1,048,576 x 1,048,576 3D
  Gaussian-mixture sets (radius 0.00287, k_max 64): row count, SHA-256 of the
  rows (``RtdlFixedRadiusNeighborRow`` bytes, 16 B, final order), SHA-256 of
  the per-query row counts (u32, query input order), the number of queries
  with more than k_max neighbours (overflow), and SHA-256 of each block of
  1,024 queries' rows, so a mismatch can be located;
* ``knn16_1m``: knn_rows with k = 16 on the same sets: SHA-256 of the rows
  packed as (query_id u32, neighbor_id u32, distance f64, neighbor_rank u32),
  20 B per row, without the ABI struct's padding;
* ``hausdorff_4m``: directed A -> B nearest distances over the 4,194,304 x
  4,194,304 2D sets: SHA-256 of the per-query nearest distances (f64) and ids
  (u32) in query input order, and the witness (max by distance, then smaller
  query id, then smaller neighbour id).

The oracle runs with its uniform-grid candidate generator (the same FP64
arithmetic and sort keys as the brute-force restatement, which the CPU tests
check it against); the point sets come from ``rtdl_b200.workloads``, the
generators the benchmark uses.  A few minutes on 8 cores.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from rtdl_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent / "full_scale_digests.json"
RADIUS, K_MAX, K_KNN, BLOCK = 0.00287, 64, 16, 1024

KNN_PACKED = np.dtype({"names": ["query_id", "neighbor_id", "distance", "neighbor_rank"],
                       "formats": ["<u4", "<u4", "<f8", "<u4"], "offsets": [0, 4, 8, 16], "itemsize": 20})


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def frn_digest(rows: np.ndarray, counts: np.ndarray, nq: int) -> dict:
    """Digest of a full fixed-radius row set; rows in final order, counts = rows per query (input order,
    ids = input index so output order is input order)."""
    offsets = np.zeros(nq + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    blocks = [sha(rows[offsets[b]:offsets[min(b + BLOCK, nq)]])[:16] for b in range(0, nq, BLOCK)]
    return {"rows": int(len(rows)), "rows_sha256": sha(rows), "counts_sha256": sha(counts.astype(np.uint32)),
            "block_queries": BLOCK, "block_sha256_16": blocks}


def knn_packed(rows: np.ndarray) -> np.ndarray:
    out = np.zeros(len(rows), dtype=KNN_PACKED)
    for n in KNN_PACKED.names:
        out[n] = rows[n]
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args(argv)
    out = {"generator": "tests/golden/make_full_scale_digests.py",
           "oracle": "oracle/nn_oracle.c (uniform-grid candidates, brute-force arithmetic and keys)"}

    probe, build = workloads.clustered_3d()
    nq = len(probe)
    t = time.time()
    rows, total = O.fixed_radius_neighbors(probe, build, radius=RADIUS, k_max=K_MAX, threads=args.threads,
                                           with_counts=True, grid=True)
    counts = np.minimum(total, K_MAX)
    out["frn_1m"] = {"workload": "clustered_3d 1,048,576 x 1,048,576 (rtdl_b200.workloads.clustered_3d)",
                     "radius": RADIUS, "k_max": K_MAX, "overflow_queries": int((total > K_MAX).sum()),
                     **frn_digest(rows, counts, nq)}
    print(f"frn: {len(rows)} rows in {time.time() - t:.1f} s", flush=True)
    del rows

    t = time.time()
    knn = O.knn_rows(probe, build, k=K_KNN, threads=args.threads, grid=True)
    out["knn16_1m"] = {"workload": "clustered_3d 1,048,576 x 1,048,576", "k": K_KNN, "rows": int(len(knn)),
                       "rows_packed_sha256": sha(knn_packed(knn)),
                       "max_kth_distance": float(knn["distance"].reshape(-1, K_KNN)[:, -1].max())}
    print(f"knn: {len(knn)} rows in {time.time() - t:.1f} s", flush=True)
    del knn

    t = time.time()
    a, b = workloads.hausdorff_2d()
    dist, nid = O.nearest(a, b, threads=args.threads, grid=True)
    qid = np.asarray(a["id"], dtype=np.uint32)
    order = np.lexsort((nid, qid, -dist))  # max distance, then smaller query id, then smaller neighbour id
    w = int(order[0])
    out["hausdorff_4m"] = {"workload": "hausdorff_2d 4,194,304 x 4,194,304 (rtdl_b200.workloads.hausdorff_2d)",
                           "queries": int(len(a)), "nearest_distance_sha256": sha(dist),
                           "nearest_id_sha256": sha(nid),
                           "witness": {"distance": float(dist[w]), "distance_hex": float(dist[w]).hex(),
                                       "source_id": int(qid[w]), "target_id": int(nid[w])}}
    print(f"hausdorff: {len(a)} queries in {time.time() - t:.1f} s", flush=True)
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print(OUT)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
