"""Query sharding over ranks (one process per GPU in production), exercised
with world_size 2 on the gloo backend on CPU.  Each rank answers the queries
of its output-order range; rank 0 concatenates the gathered rows, which must
equal the single-process rows exactly.  The per-rank compute here is the CPU
oracle standing in for a GPU; what is under test is the sharding, the gather
and the merge."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from rtdl_b200 import sharding, workloads


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queries, search, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = sharding.shard_queries(queries, world, rank)
        rows = O.fixed_radius_neighbors(mine, search, radius=0.05, k_max=7)
        witness = O.directed_hausdorff(mine, search)
        gathered = [None] * world
        dist.all_gather_object(gathered, (rows, witness))
        if rank == 0:
            merged = sharding.merge_rows([g[0] for g in gathered])
            hd = sharding.merge_directed_hausdorff([g[1] for g in gathered])
            results.put((merged.tobytes(), hd))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_rank_sharding_reproduces_single_process_rows(world):
    rng = np.random.default_rng(41)
    queries = workloads.records(rng.random((3001, 3)), ids=rng.integers(0, 900, 3001).astype(np.uint32))
    search = workloads.records(rng.random((4000, 3)))
    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, queries, search, results)) for r in range(world)]
    for p in procs:
        p.start()
    merged_bytes, hd = results.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expected = O.fixed_radius_neighbors(queries, search, radius=0.05, k_max=7)
    merged = np.frombuffer(merged_bytes, dtype=expected.dtype)
    for f in ("query_id", "neighbor_id"):
        assert np.array_equal(merged[f], expected[f])
    assert np.array_equal(merged["distance"].view(np.uint64), expected["distance"].view(np.uint64))
    assert hd == O.directed_hausdorff(queries, search)


def test_shard_ranges_cover_everything_once():
    for n in (0, 1, 5, 1000, 1001):
        for world in (1, 2, 3, 8):
            spans = [sharding.shard_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1
