"""Autotuner for the fixed-radius path: picks the kernel configuration per shape class.

The knobs (``rtdl_b200_set_tuning``): the LBVH leaf-bucket size (points per
leaf, the traversal's tile), the collect traversal (``packet``: one warp walks
the tree for 32 neighbouring queries; ``packet_cube``: the same with the
query's bounding cube tested at internal nodes; ``packet_points``: the same
with leaf buckets tested a lane per point, the reaching queries in turn;
``packet_hybrid``, the library default: the one of those two leaf tests that
costs less for each bucket; ``lane``: one thread per query) and the collect
block size.  A shape class is the dimension plus the
log2 buckets of the build size, the query count and the mean in-radius count
(from a sampled query).  :meth:`Autotuner.tune` times every candidate on the
caller's device-resident data with CUDA events (min of ``repeats``), keeps
the fastest, and caches it per class (in memory, and in a JSON file when
``cache_path`` is given); :meth:`Autotuner.apply` sets a class's cached
configuration before a call.  Results do not depend on the configuration
(``tests/test_gpu_autotune.py`` checks the rows of every candidate).
"""
from __future__ import annotations

import itertools
import json
import math
import os
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np

from . import _native
from .runtime import B200Scene, set_tuning

LEAF_SIZES = (8, 16, 24, 32)
TRAVERSALS = ("packet_hybrid", "packet", "packet_cube", "packet_points", "lane")
BLOCK_THREADS = (128, 256)


@dataclass(frozen=True)
class Config:
    leaf_size: int = 0  # 0: the library default (see set_tuning)
    traversal: str = "packet_hybrid"
    block_threads: int = 128

    def apply(self) -> None:
        set_tuning(leaf_size=self.leaf_size, block_threads=self.block_threads, traversal=self.traversal)


DEFAULT = Config()


def shape_class(dimension: int, build_count: int, query_count: int, mean_count: float) -> str:
    """The cache key: dimension and log2 buckets of the sizes and of the mean in-radius count."""
    def b(x: float) -> int:
        return int(round(math.log2(max(x, 1.0))))

    return f"d{dimension}-b{b(build_count)}-q{b(query_count)}-m{b(mean_count + 1.0)}"


class Autotuner:
    def __init__(self, cache_path: str | os.PathLike | None = None, *, repeats: int = 3,
                 leaf_sizes=LEAF_SIZES, traversals=TRAVERSALS, block_threads=BLOCK_THREADS):
        self.cache_path = Path(cache_path) if cache_path else None
        self.repeats = repeats
        self.candidates = [Config(l, t, bt) for l, t, bt in itertools.product(leaf_sizes, traversals, block_threads)]
        self.cache: dict[str, dict] = {}
        if self.cache_path and self.cache_path.exists():
            self.cache = json.loads(self.cache_path.read_text())

    def lookup(self, key: str) -> Config | None:
        entry = self.cache.get(key)
        return Config(**entry["config"]) if entry else None

    def apply(self, key: str) -> Config:
        cfg = self.lookup(key) or DEFAULT
        cfg.apply()
        return cfg

    def _store(self, key: str, cfg: Config, timings: dict) -> None:
        self.cache[key] = {"config": asdict(cfg), "ms": timings}
        if self.cache_path:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            self.cache_path.write_text(json.dumps(self.cache, indent=1, sort_keys=True))

    def tune(self, build_address: int, build_count: int, query_address: int, query_count: int, *, dimension: int,
             radius: float, k_max: int, stream: int | None = None, force: bool = False) -> tuple[str, Config]:
        """Times every candidate on device-resident records (plain build + fixed-radius query, as one call
        would run) and caches the fastest for this shape class; returns (key, config) and applies it."""
        import torch

        mean = self._mean_count(build_address, build_count, query_address, query_count, dimension, radius, k_max,
                                stream)
        key = shape_class(dimension, build_count, query_count, mean)
        if not force and key in self.cache:
            return key, self.apply(key)
        rows = torch.empty(max(query_count * k_max, 1) * 16, dtype=torch.uint8, device="cuda")
        timings = {}
        for cfg in self.candidates:
            cfg.apply()
            best = math.inf
            for _ in range(self.repeats + 1):  # the first run warms the allocator
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                cur = torch.cuda.current_stream()
                a.record(cur)
                self._run(build_address, build_count, query_address, query_count, dimension, radius, k_max,
                          rows.data_ptr(), query_count * k_max, stream)
                b.record(cur)
                b.synchronize()
                best = min(best, a.elapsed_time(b))
            timings[f"{cfg.leaf_size}/{cfg.traversal}/{cfg.block_threads}"] = best
        winner = min(self.candidates, key=lambda c: timings[f"{c.leaf_size}/{c.traversal}/{c.block_threads}"])
        self._store(key, winner, timings)
        winner.apply()
        return key, winner

    def tune_callable(self, key: str, run, *, stream=None, force: bool = False) -> tuple[str, Config]:
        """Times ``run()`` with CUDA events on ``stream`` (a torch stream; default the current one) under
        every candidate, caches the fastest under ``key``, applies it and returns (key, config).  For a
        workload no single plain call stands for, such as one whole problem batch."""
        import torch

        if not force and key in self.cache:
            return key, self.apply(key)
        timings = {}
        for cfg in self.candidates:
            cfg.apply()
            best = math.inf
            for _ in range(self.repeats + 1):  # the first run warms the allocator
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                cur = stream if stream is not None else torch.cuda.current_stream()
                a.record(cur)
                run()
                b.record(cur)
                b.synchronize()
                best = min(best, a.elapsed_time(b))
            timings[f"{cfg.leaf_size}/{cfg.traversal}/{cfg.block_threads}"] = best
        winner = min(self.candidates, key=lambda c: timings[f"{c.leaf_size}/{c.traversal}/{c.block_threads}"])
        self._store(key, winner, timings)
        winner.apply()
        return key, winner

    @staticmethod
    def _run(build_address, build_count, query_address, query_count, dimension, radius, k_max, rows_address,
             capacity, stream):
        scene = B200Scene(None, dimension=dimension, stream=stream, device_points=(build_address, build_count))
        try:
            return scene.query_device(query_address, query_count, predicate="fixed_radius_neighbors", radius=radius,
                                      limit=k_max, rows_address=rows_address, rows_capacity=capacity, stream=stream)
        finally:
            scene.close()

    def _mean_count(self, build_address, build_count, query_address, query_count, dimension, radius, k_max, stream):
        """Mean in-radius count, from the first 4,096 queries (rows counted at k_max = 64)."""
        n = min(query_count, 4096)
        if n == 0:
            return 0.0
        total = self._run(build_address, build_count, query_address, n, dimension, radius, 64, None, 0, stream)
        return total / n


def tune_records(build: np.ndarray, query: np.ndarray, *, radius: float, k_max: int,
                 tuner: Autotuner | None = None, **kw) -> tuple[str, Config]:
    """Convenience: tune on host record arrays (copied to the device once)."""
    import torch

    _native.load_library()
    tuner = tuner or Autotuner()
    d_b = torch.from_numpy(build.view(np.uint8).copy()).cuda()
    d_q = torch.from_numpy(query.view(np.uint8).copy()).cuda()
    dim = 3 if build.dtype.itemsize == 32 else 2
    return tuner.tune(d_b.data_ptr(), len(build), d_q.data_ptr(), len(query), dimension=dim, radius=radius,
                      k_max=k_max, **kw)
