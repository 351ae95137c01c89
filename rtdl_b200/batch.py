"""Problem batches: many independent fixed-radius problems answered together.

A :class:`B200ProblemBatch` holds the search points of P problems in one LBVH
(``rtdl_b200_batch_create``); one call of :meth:`fixed_radius_neighbors`
answers every problem's queries with one launch sequence, each problem with
its own radius and k_max.  The rows of problem p equal what
``rtdl_b200.fixed_radius_neighbors`` (one plain per-call launch) returns for
that problem alone; they come back problem after problem with per-problem
offsets.

The reference answers one problem per call (``rtdl_optix_api.cpp:4076-4150``
through ``optix_runtime.py:15798-15831``); batching many uneven problems into
one launch has no counterpart there.
"""
from __future__ import annotations

import ctypes
from collections.abc import Sequence

import numpy as np

from . import _native
from .runtime import FRN_ROW_DTYPE, PackedPoints, _pack_any


def _concat(sets: Sequence, dimension: int | None) -> tuple[np.ndarray, np.ndarray, int, list]:
    """Packs every problem's points and concatenates them: (records, offsets, dimension, keepalive)."""
    packed = []
    dim = dimension
    for s in sets:
        p = s if isinstance(s, PackedPoints) else None
        if p is None:
            addr, n, d, keep = _pack_any(s, dim)
            p = keep if isinstance(keep, PackedPoints) else None
            if p is None:  # a reference PackedPoints (ctypes records): copy its bytes
                rec = np.ctypeslib.as_array((ctypes.c_uint8 * (n * (32 if d == 3 else 24))).from_address(addr))
                from .runtime import POINT2D_DTYPE, POINT3D_DTYPE

                p = PackedPoints(rec.view(POINT3D_DTYPE if d == 3 else POINT2D_DTYPE).copy(), n, d)
        if dim is None:
            dim = p.dimension
        elif p.dimension != dim:
            raise ValueError("every problem of a batch must have the same dimension")
        packed.append(p)
    if dim is None:
        raise ValueError("a problem batch needs at least one problem")
    offsets = np.zeros(len(packed) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([p.count for p in packed], dtype=np.uint64)
    records = concat_records([p.records[: p.count] for p in packed])
    return records, offsets, dim, packed


def concat_records(arrays: Sequence[np.ndarray]) -> np.ndarray:
    """Concatenates ABI record arrays keeping their padded layout (np.concatenate
    would promote the structured dtype to a packed one, 28 bytes per 3D record)."""
    if not arrays:
        return np.zeros(0, dtype=np.uint8)
    out = np.empty(sum(len(a) for a in arrays), dtype=arrays[0].dtype)
    i = 0
    for a in arrays:
        if a.dtype != out.dtype:
            raise ValueError("every problem of a batch must have the same record layout")
        out[i: i + len(a)] = a
        i += len(a)
    return out


def _per_problem(value, problems: int, dtype, name: str) -> np.ndarray:
    arr = np.asarray(value, dtype=dtype)
    if arr.ndim == 0:
        arr = np.full(problems, arr, dtype=dtype)
    if arr.shape != (problems,):
        raise ValueError(f"{name} must be a scalar or one value per problem")
    return np.ascontiguousarray(arr)


class B200BatchRows:
    """Rows of a batch call: one structured array (``FRN_ROW_DTYPE``) for all
    problems plus ``row_offsets`` (problems + 1 entries)."""

    def __init__(self, rows: np.ndarray, row_offsets: np.ndarray, overflow: np.ndarray | None):
        self.rows = rows
        self.row_offsets = row_offsets
        self.overflow = overflow

    @property
    def problems(self) -> int:
        return len(self.row_offsets) - 1

    def problem(self, p: int) -> np.ndarray:
        return self.rows[int(self.row_offsets[p]): int(self.row_offsets[p + 1])]

    def to_dict_rows(self, p: int) -> tuple[dict, ...]:
        return tuple({"query_id": int(r["query_id"]), "neighbor_id": int(r["neighbor_id"]),
                      "distance": float(r["distance"])} for r in self.problem(p))

    def __len__(self) -> int:
        return len(self.rows)


class B200ProblemBatch:
    """The search points of many problems in one device LBVH."""

    def __init__(self, search_sets: Sequence | None = None, *, dimension: int | None = None,
                 stream: int | None = None, device_points: tuple[int, Sequence[int]] | None = None):
        """search_sets: one points payload per problem (records, PackedPoints, structured arrays).
        device_points: (address of the concatenated records on the device, offsets) instead."""
        lib = _native.load_library()
        self._lib = lib
        self._handle = ctypes.c_void_p()
        err = _native.error_buffer()
        if device_points is not None:
            address, offsets = device_points
            if dimension not in (2, 3):
                raise ValueError("device_points needs an explicit dimension")
            self._offsets = np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
            self.dimension = dimension
            status = lib.rtdl_b200_batch_create(address, self._offsets.ctypes.data, len(self._offsets) - 1,
                                                dimension, 1, stream, ctypes.byref(self._handle), err, len(err))
        else:
            records, self._offsets, self.dimension, keep = _concat(search_sets, dimension)
            status = lib.rtdl_b200_batch_create(records.ctypes.data if len(records) else None,
                                                self._offsets.ctypes.data, len(self._offsets) - 1, self.dimension,
                                                0, stream, ctypes.byref(self._handle), err, len(err))
            del keep, records
        _native.check_status(status, err)
        self.problems = len(self._offsets) - 1
        self._closed = False

    @property
    def handle(self) -> int:
        return self._handle.value or 0

    def fixed_radius_neighbors(self, query_sets: Sequence, *, radius, k_max, with_overflow: bool = False
                               ) -> B200BatchRows:
        """One call for all problems: query_sets[p] against problem p's points with radius[p] / k_max[p]
        (scalars apply to every problem; k_max in [1, 64])."""
        if self._closed:
            raise RuntimeError("batch is closed")
        if len(query_sets) != self.problems:
            raise ValueError("one query set per problem is required")
        records, qoff, _, keep = _concat(query_sets, self.dimension)
        r = _per_problem(radius, self.problems, np.float64, "radius")
        k = _per_problem(k_max, self.problems, np.uint32, "k_max")
        row_offsets = np.zeros(self.problems + 1, dtype=np.uint64)
        nq = int(qoff[-1])
        overflow = np.zeros(nq, dtype=np.uint8) if with_overflow else None
        rows = ctypes.c_void_p()
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_batch_fixed_radius_neighbors(
            self._handle, records.ctypes.data if nq else None, qoff.ctypes.data, r.ctypes.data, k.ctypes.data,
            ctypes.byref(rows), row_offsets.ctypes.data,
            overflow.ctypes.data if overflow is not None and nq else None, err, len(err))
        del keep, records
        _native.check_status(status, err)
        total = int(row_offsets[-1])
        out = np.zeros(total, dtype=FRN_ROW_DTYPE)
        if total:
            ctypes.memmove(out.ctypes.data, rows.value, total * FRN_ROW_DTYPE.itemsize)
        if rows.value:
            self._lib.rtdl_b200_free_rows(rows)
        return B200BatchRows(out, row_offsets, overflow)

    def fixed_radius_neighbors_device(self, query_address: int, query_offsets, *, radius, k_max,
                                      rows_address: int | None, rows_capacity: int,
                                      overflow_address: int | None = None, stream: int | None = None) -> np.ndarray:
        """Device-resident call; returns row_offsets (problems + 1 entries, the last is the total)."""
        qoff = np.ascontiguousarray(np.asarray(query_offsets, dtype=np.uint64))
        if len(qoff) != self.problems + 1:
            raise ValueError("query_offsets needs problems + 1 entries")
        r = _per_problem(radius, self.problems, np.float64, "radius")
        k = _per_problem(k_max, self.problems, np.uint32, "k_max")
        row_offsets = np.zeros(self.problems + 1, dtype=np.uint64)
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_batch_fixed_radius_neighbors_device(
            self._handle, query_address, qoff.ctypes.data, r.ctypes.data, k.ctypes.data, rows_address,
            int(rows_capacity), row_offsets.ctypes.data, overflow_address, stream, err, len(err))
        _native.check_status(status, err)
        return row_offsets

    def close(self) -> None:
        if not self._closed:
            self._lib.rtdl_b200_batch_destroy(self._handle)
            self._closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200ProblemBatchGraph:
    """Every problem of several prepared :class:`B200ProblemBatch` objects
    answered by one captured CUDA graph (``rtdl_b200_batch_graph_create``).

    ``query_address`` holds all problems' device query records back to back
    (problem p at ``query_offsets[p]:query_offsets[p + 1]``, problems numbered
    batch after batch); rows go to the device buffer at ``rows_address``
    (capacity ``rows_capacity`` rows) problem by problem.  Per batch, one
    persistent collect launch takes 32-query packets from a device work queue;
    nothing is read back inside the graph.  Mirrors the reference's captured
    batch graph (``rtdl_optix_api.cpp:4323-4396``), for problem batches.
    """

    def __init__(self, batches: Sequence[B200ProblemBatch], query_address: int, query_offsets, *, radius, k_max,
                 rows_address: int | None, rows_capacity: int):
        lib = _native.load_library()
        self._lib = lib
        self._batches = list(batches)  # kept alive with the graph
        self.problems = sum(b.problems for b in self._batches)
        self._qoff = np.ascontiguousarray(np.asarray(query_offsets, dtype=np.uint64))
        if len(self._qoff) != self.problems + 1:
            raise ValueError("query_offsets needs problems + 1 entries")
        self._radius = _per_problem(radius, self.problems, np.float64, "radius")
        self._kmax = _per_problem(k_max, self.problems, np.uint32, "k_max")
        handles = (ctypes.c_void_p * len(self._batches))(*[b.handle for b in self._batches])
        self._handle = ctypes.c_void_p()
        self._closed = True
        err = _native.error_buffer()
        status = lib.rtdl_b200_batch_graph_create(
            handles, len(self._batches), query_address, self._qoff.ctypes.data, self._radius.ctypes.data,
            self._kmax.ctypes.data, rows_address, int(rows_capacity), ctypes.byref(self._handle), err, len(err))
        _native.check_status(status, err)
        self._closed = False

    def replay(self) -> tuple[np.ndarray, int]:
        """One replay; returns (row_offsets with problems + 1 entries, status bits)."""
        if self._closed:
            raise RuntimeError("graph is closed")
        offsets = np.zeros(self.problems + 1, dtype=np.uint64)
        status = ctypes.c_uint32()
        err = _native.error_buffer()
        st = self._lib.rtdl_b200_batch_graph_replay(self._handle, offsets.ctypes.data, ctypes.byref(status), err,
                                                    len(err))
        _native.check_status(st, err)
        return offsets, int(status.value)

    def launch(self, stream: int | None = None) -> None:
        """Enqueue one replay after `stream`'s work, without waiting."""
        if self._closed:
            raise RuntimeError("graph is closed")
        err = _native.error_buffer()
        _native.check_status(self._lib.rtdl_b200_batch_graph_launch(self._handle, stream, err, len(err)), err)

    def info(self) -> dict:
        problems, kernels, fallbacks = ctypes.c_uint32(), ctypes.c_int(), ctypes.c_ulonglong()
        self._lib.rtdl_b200_batch_graph_info(self._handle, ctypes.byref(problems), ctypes.byref(kernels),
                                             ctypes.byref(fallbacks))
        return {"problems": problems.value, "kernel_nodes": kernels.value, "fallbacks": fallbacks.value}

    def close(self) -> None:
        if not self._closed:
            self._lib.rtdl_b200_batch_graph_destroy(self._handle)
            self._closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
