"""A served request loop over resident scenes with continuous batching.

:class:`B200Server` keeps prepared LBVH scenes resident on one GPU and answers
neighbor requests (``fixed_radius_neighbors`` and ``knn_rows``) as they
arrive:

* **admission by device-memory budget** -- every request is charged an
  estimate of the device memory its call needs (query records, the candidate
  slab, row buffer, scratch); a request waits while admitting it would exceed
  the budget (``memory_budget`` minus what the resident scenes hold) and is
  admitted as soon as finishing requests free enough;
* **continuous batching** -- whenever a worker stream is free, the scheduler
  takes the oldest waiting request and, for fixed-radius requests, every other
  waiting fixed-radius request on the same scene (up to ``max_batch_probes``
  probes), and answers the group with ONE launch sequence
  (``rtdl_b200_scene_fixed_radius_neighbors_multi_device``, each request with
  its own radius and k_max); requests that arrive while a group runs join the
  next group;
* **overlap on the device** -- ``streams`` worker threads each own a CUDA
  stream; groups on different workers run concurrently on the GPU (the
  library releases the GIL inside every call);
* **latency accounting** -- each request records its arrival, admission and
  completion time; :meth:`B200Server.stats` reports p50 / p99 latency and
  rows/s.

A request's rows are exactly what the plain per-call path returns for that
request alone (``B200Scene.query``); the served tests check this for every
request of a mixed run.  The reference has no serving layer; its prepared
scenes (``PreparedOptixFixedRadiusNeighbors3D``, ``optix_runtime.py:2315-2419``)
answer one query set per call.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .runtime import FRN_ROW_DTYPE, KNN_ROW_DTYPE, POINT2D_DTYPE, POINT3D_DTYPE, B200Scene

FRN, KNN = "fixed_radius_neighbors", "knn_rows"
_SLAB_BYTES_PER_PROBE = 256 * 8  # candidate slab entries per probe
_SCRATCH_BYTES_PER_PROBE = 160   # per-probe records, lists and orders of one call
_SCENE_BYTES_PER_POINT = 112     # points, exact coordinates, order, codes, nodes


@dataclass
class Request:
    """One neighbor request.  ``rows`` holds the result once ``done`` is set."""

    rid: int
    scene: str
    op: str
    queries: np.ndarray
    radius: float = 0.0
    limit: int = 1
    arrival: float = 0.0
    admitted: float = 0.0
    finished: float = 0.0
    rows: np.ndarray | None = None
    row_count: int = 0
    keep: bool = True  # False: the rows reach pinned host memory but are not kept (load generators)
    error: str | None = None
    batch_size: int = 0  # requests answered by the same launch sequence
    done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_bytes(op: str, probes: int, limit: int, dimension: int) -> int:
    """Device memory one request is charged at admission."""
    rec = 32 if dimension == 3 else 24
    row = 16 if op == FRN else 24
    slab = _SLAB_BYTES_PER_PROBE if op == FRN else 4 * max(limit, 1)
    return probes * (rec + row * max(limit, 1) + slab + _SCRATCH_BYTES_PER_PROBE)


class _Budget:
    def __init__(self, total: int):
        self.total = total
        self.used = 0
        self._lock = threading.Lock()

    def try_take(self, n: int) -> bool:
        with self._lock:
            if self.used + n > self.total:
                return False
            self.used += n
            return True

    def give(self, n: int) -> None:
        with self._lock:
            self.used -= n


class B200Server:
    """Resident scenes, a request queue, and ``streams`` workers on one GPU."""

    def __init__(self, *, memory_budget: int = 120 << 30, streams: int = 4, max_batch_probes: int = 2 << 20,
                 max_batch_requests: int = 256, batching: bool = True, device: int = 0):
        import torch

        self._torch = torch
        self.device = device
        torch.cuda.set_device(device)
        self.budget = _Budget(memory_budget)
        self.max_batch_probes = max_batch_probes
        self.max_batch_requests = max_batch_requests
        self.batching = batching
        self.scenes: dict[str, B200Scene] = {}
        self._scene_bytes: dict[str, int] = {}
        self._pending: collections.deque[Request] = collections.deque()
        self._cv = threading.Condition()
        self._free_workers: collections.deque[int] = collections.deque(range(streams))
        self._work: list[collections.deque] = [collections.deque() for _ in range(streams)]
        self._work_cv = [threading.Condition() for _ in range(streams)]
        self._streams = [torch.cuda.Stream(device=device) for _ in range(streams)]
        # per-worker pinned staging buffers, page-locked once here for the largest group the scheduler
        # forms (page-locking while requests wait would stall them), grown only if a group needs more
        self._pinned: list[dict] = [{} for _ in range(streams)]
        rows_bytes = max(max_batch_probes * 64 * 16, (1 << 20) * 32 * 24)
        for pool in self._pinned:
            self._staging(pool, "queries", max_batch_probes * 32)
            self._staging(pool, "rows", rows_bytes)
        self._threads: list[threading.Thread] = []
        self._running = False
        self._next_id = 0
        self.completed: list[Request] = []
        self._lock = threading.Lock()

    # ---- scenes -------------------------------------------------------------
    def add_scene(self, name: str, points, *, dimension: int | None = None) -> None:
        """Builds the scene's LBVH on the device; it stays resident until close()."""
        scene = B200Scene(points, dimension=dimension)
        nbytes = scene.count * _SCENE_BYTES_PER_POINT
        if not self.budget.try_take(nbytes):
            scene.close()
            raise MemoryError(f"scene {name!r} does not fit the device-memory budget")
        self.scenes[name] = scene
        self._scene_bytes[name] = nbytes

    # ---- requests -----------------------------------------------------------
    def submit(self, scene: str, op: str, queries: np.ndarray, *, radius: float = 0.0, limit: int,
               keep: bool = True) -> Request:
        if scene not in self.scenes:
            raise KeyError(f"unknown scene {scene!r}")
        if op not in (FRN, KNN):
            raise ValueError("op must be 'fixed_radius_neighbors' or 'knn_rows'")
        if op == FRN and not 1 <= limit <= 64:
            raise ValueError("served fixed_radius_neighbors takes k_max in [1, 64]")
        if op == KNN and limit < 1:
            raise ValueError("knn_rows k must be positive")
        dim = self.scenes[scene].dimension
        if queries.dtype != (POINT3D_DTYPE if dim == 3 else POINT2D_DTYPE):
            raise ValueError("queries must be ABI records of the scene's dimension")
        if request_bytes(op, len(queries), limit, dim) > self.budget.total - sum(self._scene_bytes.values()):
            raise MemoryError("request exceeds the device-memory budget left beside the resident scenes")
        with self._cv:
            r = Request(self._next_id, scene, op, queries, float(radius), int(limit), time.perf_counter(),
                        keep=keep)
            self._next_id += 1
            self._pending.append(r)
            self._cv.notify_all()
        return r

    # ---- loop ---------------------------------------------------------------
    def start(self) -> None:
        self._running = True
        self._threads = [threading.Thread(target=self._schedule, daemon=True)]
        self._threads += [threading.Thread(target=self._worker, args=(w,), daemon=True)
                          for w in range(len(self._streams))]
        for t in self._threads:
            t.start()

    def stop(self) -> None:
        self._running = False
        with self._cv:
            self._cv.notify_all()
        for cv in self._work_cv:
            with cv:
                cv.notify_all()
        for t in self._threads:
            t.join(timeout=5)
        self._threads = []

    def close(self) -> None:
        self.stop()
        for name, scene in self.scenes.items():
            scene.close()
            self.budget.give(self._scene_bytes[name])
        self.scenes.clear()
        self._scene_bytes.clear()

    def __enter__(self):
        self.start()
        return self

    def __exit__(self, *exc):
        self.close()

    def _take_group(self) -> tuple[list[Request], int] | None:
        """Called with self._cv held: the oldest waiting request plus, for fixed-radius requests,
        the other waiting fixed-radius requests of its scene that fit; None when nothing fits now."""
        if not self._pending:
            return None
        head = self._pending[0]
        dim = self.scenes[head.scene].dimension
        group = [head]
        probes = len(head.queries)
        if self.batching and head.op == FRN:
            for r in list(self._pending)[1:]:
                if len(group) >= self.max_batch_requests:
                    break
                if r.op == FRN and r.scene == head.scene and probes + len(r.queries) <= self.max_batch_probes:
                    group.append(r)
                    probes += len(r.queries)
        nbytes = sum(request_bytes(r.op, len(r.queries), r.limit, dim) for r in group)
        if not self.budget.try_take(nbytes):
            if len(group) == 1:
                return None
            group = [head]  # the head alone may still fit
            nbytes = request_bytes(head.op, len(head.queries), head.limit, dim)
            if not self.budget.try_take(nbytes):
                return None
        ids = {r.rid for r in group}
        self._pending = collections.deque(r for r in self._pending if r.rid not in ids)
        return group, nbytes

    def _schedule(self) -> None:
        while self._running:
            with self._cv:
                while self._running and (not self._pending or not self._free_workers):
                    self._cv.wait(0.01)
                if not self._running:
                    return
                taken = self._take_group()
                if taken is None:  # waits for memory to free up
                    self._cv.wait(0.001)
                    continue
                w = self._free_workers.popleft()
            now = time.perf_counter()
            for r in taken[0]:
                r.admitted = now
            with self._work_cv[w]:
                self._work[w].append(taken)
                self._work_cv[w].notify()

    def _worker(self, w: int) -> None:
        self._torch.cuda.set_device(self.device)
        stream = self._streams[w]
        while self._running:
            with self._work_cv[w]:
                while self._running and not self._work[w]:
                    self._work_cv[w].wait(0.01)
                if not self._running:
                    return
                group, nbytes = self._work[w].popleft()
            try:
                self._run_group(group, stream, self._pinned[w])
            except Exception as exc:  # reported per request; the loop keeps serving
                for r in group:
                    r.error = str(exc)
            finally:
                self.budget.give(nbytes)
                now = time.perf_counter()
                with self._lock:
                    for r in group:
                        r.finished = now
                        r.batch_size = len(group)
                        self.completed.append(r)
                for r in group:
                    r.done.set()
                with self._cv:
                    self._free_workers.append(w)
                    self._cv.notify_all()

    def _staging(self, pool: dict, name: str, nbytes: int):
        """A pinned host buffer of at least nbytes, kept per worker."""
        buf = pool.get(name)
        if buf is None or buf.numel() < nbytes:
            buf = self._torch.empty(max(nbytes, 1 << 20), dtype=self._torch.uint8, pin_memory=True)
            pool[name] = buf
        return buf

    def _run_group(self, group: list[Request], stream, pool: dict) -> None:
        torch = self._torch
        scene = self.scenes[group[0].scene]
        rec = 32 if scene.dimension == 3 else 24
        counts = [len(r.queries) for r in group]
        qoff = np.zeros(len(group) + 1, dtype=np.uint64)
        qoff[1:] = np.cumsum(counts)
        nq = int(qoff[-1])
        host_q = self._staging(pool, "queries", max(nq * rec, 1))[: max(nq * rec, 1)]
        hq = host_q.numpy()
        for r, a in zip(group, qoff[:-1]):
            hq[int(a) * rec: (int(a) + len(r.queries)) * rec] = r.queries.view(np.uint8)
        with torch.cuda.stream(stream):
            d_q = torch.empty(max(nq * rec, 1), dtype=torch.uint8, device=self.device)
            d_q.copy_(host_q, non_blocking=True)
            if group[0].op == FRN:
                cap = int(sum(n * r.limit for n, r in zip(counts, group)))
                d_rows = torch.empty(max(cap * 16, 16), dtype=torch.uint8, device=self.device)
                offs = scene.fixed_radius_neighbors_multi_device(
                    d_q.data_ptr(), qoff, radius=[r.radius for r in group], k_max=[r.limit for r in group],
                    rows_address=d_rows.data_ptr(), rows_capacity=cap, stream=stream.cuda_stream)
                total, dtype, row = int(offs[-1]), FRN_ROW_DTYPE, 16
            else:
                r = group[0]
                cap = nq * min(r.limit, scene.count)
                d_rows = torch.empty(max(cap * 24, 24), dtype=torch.uint8, device=self.device)
                total = scene.query_device(d_q.data_ptr(), nq, predicate=KNN, limit=r.limit,
                                           rows_address=d_rows.data_ptr(), rows_capacity=cap,
                                           stream=stream.cuda_stream)
                offs = np.array([0, total], dtype=np.uint64)
                dtype, row = KNN_ROW_DTYPE, 24
            host_rows = self._staging(pool, "rows", max(total * row, 1))[: max(total * row, 1)]
            if total:
                host_rows[: total * row].copy_(d_rows[: total * row], non_blocking=True)
            stream.synchronize()
        hr = host_rows.numpy()
        for i, r in enumerate(group):
            a, b = int(offs[i]), int(offs[i + 1])
            r.row_count = b - a
            if r.keep:
                r.rows = np.frombuffer(hr[a * row: b * row].tobytes(), dtype=dtype)

    # ---- reporting ----------------------------------------------------------
    def stats(self) -> dict:
        with self._lock:
            done = [r for r in self.completed if r.error is None]
            failed = len(self.completed) - len(done)
        if not done:
            return {"requests": 0, "failed": failed}
        lat = np.array([r.latency for r in done]) * 1e3
        t0 = min(r.arrival for r in done)
        t1 = max(r.finished for r in done)
        rows = sum(r.row_count for r in done)
        return {
            "requests": len(done), "failed": failed, "rows": rows, "seconds": t1 - t0,
            "rows_per_s": rows / (t1 - t0) if t1 > t0 else None,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "mean_batch": float(np.mean([r.batch_size for r in done])),
        }


def run_plain(scenes: dict[str, B200Scene], requests: list[Request], arrivals: list[float]) -> dict:
    """The plain per-call path on the same trace: one host-buffer call per request, in arrival order,
    on one stream, no batching.  Returns the same statistics as B200Server.stats()."""
    t0 = time.perf_counter()
    done = []
    for r, at in zip(requests, arrivals):
        now = time.perf_counter() - t0
        if now < at:
            time.sleep(at - now)
        view = scenes[r.scene].query(r.queries, predicate=r.op, radius=r.radius, limit=r.limit)
        n = len(view)  # the rows are in host memory (the library's pinned buffer)
        view.close()
        done.append((t0 + at, time.perf_counter(), n))
    lat = np.array([f - a for a, f, _ in done]) * 1e3
    rows = sum(n for _, _, n in done)
    t1 = max(f for _, f, _ in done)
    return {"requests": len(done), "rows": rows, "seconds": t1 - t0, "rows_per_s": rows / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


def replay(server: B200Server, trace: list[tuple[float, str, str, np.ndarray, float, int]],
           keep=None) -> list[Request]:
    """Submits (arrival_s, scene, op, queries, radius, limit) items at their arrival offsets and waits
    for all of them; keep: indices of the trace whose rows are kept (None: all)."""
    t0 = time.perf_counter()
    out = []
    for i, (at, scene, op, q, radius, limit) in enumerate(trace):
        now = time.perf_counter() - t0
        if now < at:
            time.sleep(at - now)
        out.append(server.submit(scene, op, q, radius=radius, limit=limit, keep=keep is None or i in keep))
    for r in out:
        r.done.wait()
    return out


def same_rows(a: np.ndarray, b: np.ndarray) -> bool:
    """Field-by-field equality of two row arrays (FP64 distances by bit pattern)."""
    if a is None or b is None or len(a) != len(b) or a.dtype.names != b.dtype.names:
        return False
    for name in a.dtype.names:
        x, y = a[name], b[name]
        if x.dtype == np.float64:
            x, y = x.view(np.uint64), y.view(np.uint64)
        if not np.array_equal(x, y):
            return False
    return True


__all__ = ["B200Server", "Request", "request_bytes", "run_plain", "replay", "same_rows", "FRN", "KNN"]
