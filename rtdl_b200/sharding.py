"""Query sharding across GPUs (one process per GPU, no data-path collective).

Rows of one query depend only on that query and the search set
(rubaolee/rtdl ``src/rtdsl/reference.py:358-375``), so every rank holds a
replica of the scene and answers a contiguous range of queries.  Ranges are cut
in *output order* -- queries stably sorted by ``query_id`` -- so concatenating
the ranks' rows in rank order reproduces the single-GPU row order exactly.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [begin, end) of n items for `rank` of `world` (sizes differ by at most 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def output_order(query_ids: np.ndarray) -> np.ndarray:
    """Permutation of queries into output order: stable sort by query_id."""
    return np.argsort(np.asarray(query_ids, dtype=np.uint32), kind="stable")


def shard_queries(query_records: np.ndarray, world: int, rank: int) -> np.ndarray:
    """The structured query records (RtdlPoint / RtdlPoint3D layout) this rank answers."""
    order = output_order(query_records["id"])
    b, e = shard_range(len(order), world, rank)
    return query_records[order[b:e]]


def merge_rows(per_rank_rows: list[np.ndarray]) -> np.ndarray:
    """Concatenates rank results in rank order (already globally ordered), keeping
    the ABI row layout (np.concatenate would drop a structured dtype's padding)."""
    nonempty = [r for r in per_rank_rows if len(r)]
    if not nonempty:
        return per_rank_rows[0][:0] if per_rank_rows else np.zeros(0)
    out = np.empty(sum(len(r) for r in nonempty), dtype=nonempty[0].dtype)
    i = 0
    for r in nonempty:
        out[i: i + len(r)] = r
        i += len(r)
    return out


def merge_directed_hausdorff(per_rank: list[dict]) -> dict:
    """Combines per-rank witnesses with the reference's rule: max by
    (distance, -query_id, -neighbor_id)."""
    best = max(per_rank, key=lambda w: (w["distance"], -w["source_id"], -w["target_id"]))
    out = dict(best)
    out["row_count"] = sum(w["row_count"] for w in per_rank)
    return out
