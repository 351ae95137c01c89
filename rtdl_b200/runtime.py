"""Host runtime of the b200 backend: ``run_b200``, prepared kernels and scenes.

Mirrors the reference's OptiX runtime for the neighbor path
(rubaolee/rtdl ``src/rtdsl/optix_runtime.py``):

* ``run_b200(kernel, *, result_mode="dict"|"raw", **inputs)`` -- ``run_optix``
  (``:1275-1331``): same input validation and messages, same result modes;
* ``prepare_b200(kernel).bind(**inputs).run()/run_raw()`` -- ``prepare_optix``
  (``:865-1000``);
* ``B200RowView`` -- ``OptixRowView`` (``:813-848``): owns the native rows,
  ``close()``, ``to_dict_rows()``, ``to_tuple_rows()``, plus ``to_numpy()``;
* ``PreparedB200FixedRadiusNeighbors3D`` / ``prepare_b200_fixed_radius_neighbors_3d``
  -- ``PreparedOptixFixedRadiusNeighbors3D`` (``:2315-2419, 2962``);
* ``pack_points`` / ``PackedPoints`` -- ``embree_runtime.py:538-542, 987-1037``,
  with a numpy column fast path (no per-point Python loop).

Everything below calls librtdl_b200.so through ctypes; no computation happens
in Python and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from collections.abc import Iterable, Mapping
from dataclasses import dataclass

import numpy as np

from . import _native
from . import dsl
from .lowering import _is_plan, lower_to_b200_plan

NEIGHBOR_PREDICATES = ("fixed_radius_neighbors", "bounded_knn_rows", "knn_rows")
PREDICATE_CODE = {"fixed_radius_neighbors": 0, "bounded_knn_rows": 1, "knn_rows": 2}

POINT2D_DTYPE = np.dtype({"names": ["id", "x", "y"], "formats": ["<u4", "<f8", "<f8"], "offsets": [0, 8, 16], "itemsize": 24})
POINT3D_DTYPE = np.dtype(
    {"names": ["id", "x", "y", "z"], "formats": ["<u4", "<f8", "<f8", "<f8"], "offsets": [0, 8, 16, 24], "itemsize": 32}
)
FRN_ROW_DTYPE = np.dtype(
    {"names": ["query_id", "neighbor_id", "distance"], "formats": ["<u4", "<u4", "<f8"], "offsets": [0, 4, 8], "itemsize": 16}
)
SUMMARY_DTYPE = np.dtype(
    {
        "names": ["query_id", "neighbor_count", "nearest_neighbor_id", "kth_neighbor_id", "nearest_distance",
                  "kth_distance", "sum_distance"],
        "formats": ["<u4", "<u4", "<u4", "<u4", "<f8", "<f8", "<f8"],
        "offsets": [0, 4, 8, 12, 16, 24, 32],
        "itemsize": 40,
    }
)
AGGREGATE_FIELDS = ("query_count", "bounded_neighbor_count", "nearest_id_checksum", "kth_id_checksum", "sum_distance")
COUNT_ROW_DTYPE = np.dtype({"names": ["query_id", "neighbor_count", "threshold_reached"],
                            "formats": ["<u4", "<u4", "<u4"], "offsets": [0, 4, 8], "itemsize": 12})
KNN_ROW_DTYPE = np.dtype(
    {
        "names": ["query_id", "neighbor_id", "distance", "neighbor_rank"],
        "formats": ["<u4", "<u4", "<f8", "<u4"],
        "offsets": [0, 4, 8, 16],
        "itemsize": 24,
    }
)


# ---------------------------------------------------------------------------
# packing
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class PackedPoints:
    """Points in the ABI record layout (RtdlPoint / RtdlPoint3D), held as a numpy array."""

    records: np.ndarray
    count: int
    dimension: int = 2

    @property
    def address(self) -> int:
        return int(self.records.ctypes.data) if self.count else 0


def _record_fields(record, names):
    if isinstance(record, Mapping):
        missing = [n for n in names if n not in record]
        if missing:
            raise ValueError(f"point record is missing fields: {', '.join(missing)}")
        return [record[n] for n in names]
    if all(hasattr(record, n) for n in names):
        return [getattr(record, n) for n in names]
    raise ValueError("point record must be a mapping or dataclass-like object")


def _has_fields(record, names) -> bool:
    if isinstance(record, Mapping):
        return all(n in record for n in names)
    return all(hasattr(record, n) for n in names)


def pack_points(records=None, *, ids=None, x=None, y=None, z=None, dimension: int | None = None) -> PackedPoints:
    """Pack point records or numpy columns into the ABI layout.

    Records follow the reference's coercion (``src/rtdsl/runtime.py:263-336``):
    mappings or objects with ``id, x, y[, z]``.  Columns (``ids``, ``x``, ``y``,
    ``z``) are packed with numpy only.
    """
    if dimension not in (None, 2, 3):
        raise ValueError("points dimension must be one of: 2, 3")
    if records is not None:
        if isinstance(records, PackedPoints):
            return records
        if isinstance(records, np.ndarray) and records.dtype.names is not None:
            names = records.dtype.names
            dim = dimension or (3 if "z" in names else 2)
            return pack_points(ids=records["id"], x=records["x"], y=records["y"],
                               z=records["z"] if dim == 3 else None, dimension=dim)
        if isinstance(records, (str, bytes)) or not isinstance(records, Iterable):
            raise ValueError("points input must be an iterable of records")
        items = list(records)
        dim = dimension
        if dim is None:
            dim = 3 if items and all(_has_fields(r, ("id", "x", "y", "z")) for r in items) else 2
        dtype = POINT3D_DTYPE if dim == 3 else POINT2D_DTYPE
        arr = np.zeros(len(items), dtype=dtype)
        if items:
            names = ("id", "x", "y", "z") if dim == 3 else ("id", "x", "y")
            if dim == 3 and not all(_has_fields(r, names) for r in items):
                raise ValueError("points packed for a 3D layout must provide 3D point records")
            if dim == 2 and any(isinstance(r, dsl.Point3D) or type(r).__name__ == "Point3D" for r in items):
                raise ValueError("points packed for a 2D layout must provide 2D point records")
            cols = list(zip(*(_record_fields(r, names) for r in items)))
            arr["id"] = np.asarray([int(v) for v in cols[0]], dtype=np.int64).astype(np.uint32)
            arr["x"] = np.asarray(cols[1], dtype=np.float64)
            arr["y"] = np.asarray(cols[2], dtype=np.float64)
            if dim == 3:
                arr["z"] = np.asarray(cols[3], dtype=np.float64)
        return PackedPoints(records=arr, count=len(items), dimension=dim)
    if ids is None or x is None or y is None:
        raise ValueError("pack_points needs records or ids/x/y columns")
    dim = dimension or (3 if z is not None else 2)
    ids_a = np.asarray(ids)
    n = len(ids_a)
    if len(x) != n or len(y) != n or (dim == 3 and (z is None or len(z) != n)):
        raise ValueError("packed points arrays must have identical lengths")
    if n and (ids_a.min() < 0 or ids_a.max() > 0xFFFFFFFF):
        raise ValueError("point ids must fit in uint32")
    arr = np.zeros(n, dtype=POINT3D_DTYPE if dim == 3 else POINT2D_DTYPE)  # zeroed padding: deterministic bytes
    arr["id"] = ids_a.astype(np.uint32, copy=False)
    arr["x"] = np.asarray(x, dtype=np.float64)
    arr["y"] = np.asarray(y, dtype=np.float64)
    if dim == 3:
        arr["z"] = np.asarray(z, dtype=np.float64)
    return PackedPoints(records=arr, count=n, dimension=dim)


def _pack_any(payload, dimension: int | None) -> tuple[int, int, int, object]:
    """Returns (address, count, dimension, keepalive) for any supported points payload."""
    cached = getattr(payload, "_rtdl_packed_points", None)
    if cached is not None:
        payload = cached
    if isinstance(payload, PackedPoints):
        if dimension is not None and payload.dimension != dimension:
            raise ValueError("packed points payload dimension does not match the kernel input layout")
        return payload.address, payload.count, payload.dimension, payload
    # The reference's own PackedPoints (ctypes array of _RtdlPoint/_RtdlPoint3D) has the same layout.
    if hasattr(payload, "records") and hasattr(payload, "count") and hasattr(payload, "dimension") \
            and isinstance(getattr(payload, "records"), ctypes.Array):
        if dimension is not None and payload.dimension != dimension:
            raise ValueError("packed points payload dimension does not match the kernel input layout")
        expected = 32 if payload.dimension == 3 else 24
        if ctypes.sizeof(payload.records._type_) != expected:
            raise ValueError("packed points records do not have the RtdlPoint/RtdlPoint3D layout")
        return (ctypes.addressof(payload.records) if payload.count else 0), int(payload.count), int(payload.dimension), payload
    packed = pack_points(records=payload, dimension=dimension)
    return packed.address, packed.count, packed.dimension, packed


# ---------------------------------------------------------------------------
# row views
# ---------------------------------------------------------------------------

@dataclass
class B200RowView:
    """Rows owned by librtdl_b200 (pinned host memory); mirrors ``OptixRowView``."""

    rows_address: int
    row_count: int
    row_dtype: np.dtype
    field_names: tuple
    _closed: bool = False

    def _array(self) -> np.ndarray:
        if self._closed:
            raise RuntimeError("row view is closed")
        if self.row_count == 0:
            return np.zeros(0, dtype=self.row_dtype)
        buf = (ctypes.c_char * (self.row_count * self.row_dtype.itemsize)).from_address(self.rows_address)
        return np.frombuffer(buf, dtype=self.row_dtype)

    def to_numpy(self, copy: bool = True) -> np.ndarray:
        a = self._array()
        if not copy:
            return a
        out = np.empty(len(a), dtype=self.row_dtype)  # a byte copy: padding stays as the library wrote it
        out.view(np.uint8)[:] = a.view(np.uint8)
        return out

    def close(self) -> None:
        if not self._closed:
            if self.rows_address:
                _native.load_library().rtdl_b200_free_rows(ctypes.c_void_p(self.rows_address))
            self._closed = True

    def __len__(self) -> int:
        return self.row_count

    def to_dict_rows(self, fields: tuple | None = None) -> tuple:
        names = tuple(fields or self.field_names)
        a = self._array()
        cols = [a[n].tolist() for n in names]
        return tuple(dict(zip(names, vals)) for vals in zip(*cols)) if self.row_count else ()

    def to_tuple_rows(self, fields: tuple | None = None) -> tuple:
        names = tuple(fields or self.field_names)
        a = self._array()
        cols = [a[n].tolist() for n in names]
        return tuple(zip(*cols)) if self.row_count else ()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _row_view(address: int, count: int, ranked: bool) -> B200RowView:
    if ranked:
        return B200RowView(address, count, KNN_ROW_DTYPE, ("query_id", "neighbor_id", "distance", "neighbor_rank"))
    return B200RowView(address, count, FRN_ROW_DTYPE, ("query_id", "neighbor_id", "distance"))


# ---------------------------------------------------------------------------
# low-level calls (plain per-call launch)
# ---------------------------------------------------------------------------

def fixed_radius_neighbors(query, search, *, radius: float, k_max: int, dimension: int | None = None,
                           ranked: bool = False) -> B200RowView:
    """One plain per-call launch (``rtdl_b200_run_fixed_radius_neighbors[_3d]`` or
    ``rtdl_b200_run_bounded_knn_rows[_3d]`` when ``ranked``)."""
    lib = _native.load_library()
    qa, qn, qd, qk = _pack_any(query, dimension)
    sa, sn, sd, sk = _pack_any(search, dimension or qd)
    if qd != sd:
        raise ValueError("query and search points must have the same dimension")
    name = ("rtdl_b200_run_bounded_knn_rows" if ranked else "rtdl_b200_run_fixed_radius_neighbors") + ("_3d" if qd == 3 else "")
    rows = ctypes.c_void_p()
    count = ctypes.c_size_t()
    err = _native.error_buffer()
    status = getattr(lib, name)(qa, qn, sa, sn, float(radius), int(k_max), ctypes.byref(rows), ctypes.byref(count), err, len(err))
    _native.check_status(status, err)
    del qk, sk
    return _row_view(rows.value or 0, count.value, ranked)


def fixed_radius_neighbors_device(query_address: int, query_count: int, search_address: int, search_count: int, *,
                                  dimension: int, radius: float, k_max: int, rows_address: int | None,
                                  rows_capacity: int, overflow_address: int | None = None,
                                  stream: int | None = None) -> int:
    """One plain per-call launch on device-resident records (``rtdl_b200_run_fixed_radius_neighbors_device``):
    builds the scene, writes the rows (``rows_address`` None: counts only); returns the row count."""
    count = ctypes.c_size_t()
    err = _native.error_buffer()
    status = _native.load_library().rtdl_b200_run_fixed_radius_neighbors_device(
        query_address, int(query_count), search_address, int(search_count), int(dimension), float(radius),
        int(k_max), rows_address, int(rows_capacity), ctypes.byref(count), overflow_address, stream, err, len(err))
    _native.check_status(status, err)
    return int(count.value)


def knn_rows(query, search, *, k: int, dimension: int | None = None) -> B200RowView:
    """One plain per-call launch of ``rtdl_b200_run_k_closest_hits[_3d]``."""
    lib = _native.load_library()
    qa, qn, qd, qk = _pack_any(query, dimension)
    sa, sn, sd, sk = _pack_any(search, dimension or qd)
    if qd != sd:
        raise ValueError("query and search points must have the same dimension")
    name = "rtdl_b200_run_k_closest_hits" + ("_3d" if qd == 3 else "")
    rows = ctypes.c_void_p()
    count = ctypes.c_size_t()
    err = _native.error_buffer()
    status = getattr(lib, name)(qa, qn, sa, sn, int(k), ctypes.byref(rows), ctypes.byref(count), err, len(err))
    _native.check_status(status, err)
    del qk, sk
    return _row_view(rows.value or 0, count.value, True)


# ---------------------------------------------------------------------------
# kernels: run_b200 / prepare_b200
# ---------------------------------------------------------------------------

def _resolve_kernel(kernel_fn_or_compiled):
    if hasattr(kernel_fn_or_compiled, "refine_op") and hasattr(kernel_fn_or_compiled, "inputs"):
        return kernel_fn_or_compiled
    if callable(kernel_fn_or_compiled):
        return kernel_fn_or_compiled()
    raise TypeError("expected an @rt.kernel function or a CompiledKernel")


def _validate_kernel(compiled) -> None:
    # same checks and messages as src/rtdsl/runtime.py:145-149
    if compiled.precision != "float_approx":
        raise ValueError("RTDL CPU simulator currently supports only precision='float_approx'")
    if compiled.candidates is None or compiled.refine_op is None or compiled.emit_op is None:
        raise ValueError("RTDL CPU simulator requires a fully compiled kernel with traverse/refine/emit")


def _check_inputs(expected, inputs, label="RTDL b200"):
    missing = [n for n in expected if n not in inputs]
    unexpected = [n for n in inputs if n not in expected]
    if missing:
        raise ValueError(f"missing {label} inputs: {', '.join(sorted(missing))}")
    if unexpected:
        raise ValueError(f"unexpected {label} inputs: {', '.join(sorted(unexpected))}")


def _call_plan(plan, packed: dict) -> B200RowView:
    """Executes a lowered plan: the plan's query/search binding, predicate and options reach the C ABI."""
    query = packed[plan.query_input]
    search = packed[plan.search_input]
    opts = plan.predicate_options
    if plan.predicate == "knn_rows":
        return knn_rows(query, search, k=int(opts["k"]))
    return fixed_radius_neighbors(query, search, radius=float(opts["radius"]), k_max=int(opts["k_max"]),
                                  ranked=plan.predicate == "bounded_knn_rows")


def _lower(kernel_fn_or_compiled_or_plan):
    """A B200ExecutionPlan for a kernel function, a compiled kernel or a plan
    (the reference's RTExecutionPlan or this backend's); kernels are checked
    with the runner's messages first (src/rtdsl/runtime.py:145-149)."""
    if _is_plan(kernel_fn_or_compiled_or_plan):
        return lower_to_b200_plan(kernel_fn_or_compiled_or_plan)
    compiled = _resolve_kernel(kernel_fn_or_compiled_or_plan)
    _validate_kernel(compiled)
    pred = compiled.refine_op.predicate.name
    if pred not in NEIGHBOR_PREDICATES:
        raise ValueError(f"unsupported predicate for b200 backend: {pred!r}")
    return lower_to_b200_plan(compiled)


class PreparedB200Kernel:
    """Compiled-once handle; mirrors ``PreparedOptixKernel`` for the neighbor predicates.  It holds the
    kernel's B200ExecutionPlan (``.plan``), which every run executes."""

    def __init__(self, kernel_fn_or_compiled):
        self.plan = _lower(kernel_fn_or_compiled)
        self.compiled = None if _is_plan(kernel_fn_or_compiled) else _resolve_kernel(kernel_fn_or_compiled)
        self.expected_inputs = {name: self.plan.dimension for name in self.plan.input_names}
        self.predicate_name = self.plan.predicate
        _native.load_library()

    def bind(self, **inputs) -> "PreparedB200Execution":
        _check_inputs(self.expected_inputs, inputs)
        packed = {}
        for name, payload in inputs.items():
            _addr, _n, _d, keep = _pack_any(payload, self.expected_inputs[name])
            packed[name] = keep
        return PreparedB200Execution(self.plan, packed)

    def run(self, **inputs) -> tuple:
        return self.bind(**inputs).run()


@dataclass
class PreparedB200Execution:
    plan: object
    packed_inputs: dict

    def run_raw(self) -> B200RowView:
        return _call_plan(self.plan, self.packed_inputs)

    def run(self) -> tuple:
        view = self.run_raw()
        try:
            return _project(self.plan.emit_fields, view)
        finally:
            view.close()


def _project(fields, view: B200RowView) -> tuple:
    fields = tuple(fields)
    missing = [f for f in fields if f not in view.field_names]
    if missing:
        raise ValueError("b200 row is missing emitted fields: " + ", ".join(missing))
    return view.to_dict_rows(fields)


def prepare_b200(kernel_fn_or_compiled) -> PreparedB200Kernel:
    return PreparedB200Kernel(kernel_fn_or_compiled)


def run_b200(kernel_fn_or_compiled, *, result_mode: str = "dict", **inputs):
    """Execute a neighbor kernel on the B200 backend (mirrors ``run_optix``).

    Takes an ``@rt.kernel`` function, a compiled kernel, or an execution plan
    (the reference's ``RTExecutionPlan`` or a ``B200ExecutionPlan``); a kernel
    is lowered to its plan first and the plan executes.
    ``result_mode="dict"`` returns ``tuple[dict, ...]`` projected onto the
    kernel's emitted fields; ``"raw"`` returns a ``B200RowView`` the caller
    closes.
    """
    plan = _lower(kernel_fn_or_compiled)
    _check_inputs({name: None for name in plan.input_names}, inputs)
    if result_mode not in {"dict", "raw"}:
        raise ValueError("b200 result_mode must be 'dict' or 'raw'")
    execution = PreparedB200Kernel(plan).bind(**inputs)
    return execution.run_raw() if result_mode == "raw" else execution.run()


# ---------------------------------------------------------------------------
# scenes (resident LBVH)
# ---------------------------------------------------------------------------

class B200Scene:
    """An LBVH built on the device over search points; serves FRN, bounded KNN,
    KNN and Hausdorff calls until ``close()``."""

    def __init__(self, search_points, *, dimension: int | None = None, stream: int | None = None,
                 device_points: tuple[int, int] | None = None):
        lib = _native.load_library()
        self._lib = lib
        self._handle = ctypes.c_void_p()
        err = _native.error_buffer()
        if device_points is not None:
            address, count = device_points
            if dimension not in (2, 3):
                raise ValueError("device_points needs an explicit dimension")
            self.dimension, self.count = dimension, int(count)
            status = lib.rtdl_b200_scene_create(address, self.count, dimension, 1, stream, ctypes.byref(self._handle), err, len(err))
        else:
            addr, n, dim, keep = _pack_any(search_points, dimension)
            self.dimension, self.count = dim, n
            status = lib.rtdl_b200_scene_create(addr, n, dim, 0, stream, ctypes.byref(self._handle), err, len(err))
            del keep
        _native.check_status(status, err)
        self._closed = False

    @property
    def handle(self) -> int:
        return self._handle.value or 0

    def query(self, query_points, *, predicate: str, radius: float = 0.0, limit: int, with_overflow: bool = False):
        if self._closed:
            raise RuntimeError("scene is closed")
        code = PREDICATE_CODE[predicate]
        addr, n, dim, keep = _pack_any(query_points, self.dimension)
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        overflow = np.zeros(n, dtype=np.uint8) if with_overflow else None
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_query(
            self._handle, addr, n, code, float(radius), int(limit), ctypes.byref(rows), ctypes.byref(count),
            overflow.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if overflow is not None else None, err, len(err))
        del keep
        _native.check_status(status, err)
        view = _row_view(rows.value or 0, count.value, code != 0)
        return (view, overflow) if with_overflow else view

    def query_device(self, query_address: int, query_count: int, *, predicate: str, radius: float = 0.0, limit: int,
                     rows_address: int, rows_capacity: int, overflow_address: int | None = None,
                     stream: int | None = None) -> int:
        """Device-resident call; returns the total row count."""
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_query_device(
            self._handle, query_address, int(query_count), PREDICATE_CODE[predicate], float(radius), int(limit),
            rows_address, int(rows_capacity), ctypes.byref(count), overflow_address, stream, err, len(err))
        _native.check_status(status, err)
        return count.value

    def fixed_radius_neighbors_multi_device(self, query_address: int, query_offsets, *, radius, k_max,
                                            rows_address: int | None, rows_capacity: int,
                                            overflow_address: int | None = None,
                                            stream: int | None = None) -> np.ndarray:
        """Several fixed_radius_neighbors requests (query ranges given by query_offsets, one radius and
        k_max each) in one launch sequence; returns row_offsets (requests + 1 entries)."""
        qoff = np.ascontiguousarray(np.asarray(query_offsets, dtype=np.uint64))
        m = len(qoff) - 1
        r = np.ascontiguousarray(np.broadcast_to(np.asarray(radius, dtype=np.float64), (m,)))
        k = np.ascontiguousarray(np.broadcast_to(np.asarray(k_max, dtype=np.uint32), (m,)))
        row_offsets = np.zeros(m + 1, dtype=np.uint64)
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_fixed_radius_neighbors_multi_device(
            self._handle, query_address, qoff.ctypes.data, m, r.ctypes.data, k.ctypes.data, rows_address,
            int(rows_capacity), row_offsets.ctypes.data, overflow_address, stream, err, len(err))
        _native.check_status(status, err)
        return row_offsets

    def ranked_summaries_device(self, query_address: int, query_count: int, *, radius: float, k_max: int,
                                summaries_address: int | None = None, stream: int | None = None) -> dict:
        """fixed_radius_neighbors reduced to per-query ranked summaries (written to summaries_address,
        SUMMARY_DTYPE, query order, when given) and their aggregate, which is returned."""
        agg = _native.RtdlFixedRadiusRankedNeighborAggregate()
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_ranked_summaries_device(
            self._handle, query_address, int(query_count), float(radius), int(k_max), summaries_address,
            ctypes.byref(agg), stream, err, len(err))
        _native.check_status(status, err)
        return {f: (float(getattr(agg, f)) if f == "sum_distance" else int(getattr(agg, f))) for f in AGGREGATE_FIELDS}

    def ranked_summaries_prepared(self, queries: B200Queries, *, radius: float, k_max: int,
                                  summaries_address: int | None = None, stream: int | None = None) -> dict:
        """ranked_summaries_device for a prepared query set."""
        agg = _native.RtdlFixedRadiusRankedNeighborAggregate()
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_ranked_summaries_prepared_device(
            self._handle, queries.handle, float(radius), int(k_max), summaries_address, ctypes.byref(agg), stream,
            err, len(err))
        _native.check_status(status, err)
        return {f: (float(getattr(agg, f)) if f == "sum_distance" else int(getattr(agg, f))) for f in AGGREGATE_FIELDS}

    def query_prepared_device(self, queries: B200Queries, *, radius: float, k_max: int, rows_address: int | None,
                              rows_capacity: int, overflow_address: int | None = None,
                              stream: int | None = None) -> int:
        """fixed_radius_neighbors rows (k_max <= 64) of a prepared query set; returns the total row count."""
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_query_prepared_device(
            self._handle, queries.handle, float(radius), int(k_max), rows_address, int(rows_capacity),
            ctypes.byref(count), overflow_address, stream, err, len(err))
        _native.check_status(status, err)
        return count.value

    def directed_hausdorff(self, query_points, *, with_nearest: bool = False):
        if self._closed:
            raise RuntimeError("scene is closed")
        addr, n, dim, keep = _pack_any(query_points, self.dimension)
        dist = ctypes.c_double()
        src = ctypes.c_uint32()
        tgt = ctypes.c_uint32()
        nd = np.zeros(n, dtype=np.float64) if with_nearest else None
        ni = np.zeros(n, dtype=np.uint32) if with_nearest else None
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_directed_hausdorff(
            self._handle, addr, n, ctypes.byref(dist), ctypes.byref(src), ctypes.byref(tgt),
            nd.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if nd is not None else None,
            ni.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if ni is not None else None, err, len(err))
        del keep
        _native.check_status(status, err)
        result = {"distance": dist.value, "source_id": int(src.value), "target_id": int(tgt.value), "row_count": n}
        return (result, nd, ni) if with_nearest else result

    def directed_hausdorff_device(self, query_address: int, query_count: int, *, nearest_distance_address=None,
                                  nearest_id_address=None, stream: int | None = None) -> dict:
        """Device-resident directed Hausdorff; per-query outputs stay in device memory."""
        dist = ctypes.c_double()
        src = ctypes.c_uint32()
        tgt = ctypes.c_uint32()
        err = _native.error_buffer()
        status = self._lib.rtdl_b200_scene_directed_hausdorff_device(
            self._handle, query_address, int(query_count), nearest_distance_address, nearest_id_address,
            ctypes.byref(dist), ctypes.byref(src), ctypes.byref(tgt), stream, err, len(err))
        _native.check_status(status, err)
        return {"distance": dist.value, "source_id": int(src.value), "target_id": int(tgt.value),
                "row_count": int(query_count)}

    def close(self) -> None:
        if not getattr(self, "_closed", True):
            self._lib.rtdl_b200_scene_destroy(self._handle)
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


class B200Queries:
    """A query set prepared once on the device (records, FP32 points, processing and output order) for
    repeated fixed-radius calls against resident scenes (``rtdl_b200_queries_create``)."""

    def __init__(self, query_points=None, *, dimension: int | None = None, stream: int | None = None,
                 device_points: tuple[int, int] | None = None):
        lib = _native.load_library()
        self._lib = lib
        self._handle = ctypes.c_void_p()
        self._closed = False
        err = _native.error_buffer()
        if device_points is not None:
            address, count = device_points
            if dimension not in (2, 3):
                raise ValueError("device_points needs an explicit dimension")
            self.dimension, self.count = dimension, int(count)
            status = lib.rtdl_b200_queries_create(address, self.count, dimension, 1, stream,
                                                  ctypes.byref(self._handle), err, len(err))
        else:
            addr, n, dim, keep = _pack_any(query_points, dimension)
            self.dimension, self.count = dim, n
            status = lib.rtdl_b200_queries_create(addr, n, dim, 0, stream, ctypes.byref(self._handle), err, len(err))
            del keep
        _native.check_status(status, err)

    @property
    def handle(self) -> int:
        return self._handle.value or 0

    @property
    def closed(self) -> bool:
        return self._closed

    def close(self) -> None:
        if not self._closed:
            self._lib.rtdl_b200_queries_destroy(self._handle)
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


class PreparedB200FixedRadiusQueryPoints3D(B200Queries):
    """Prepared 3-D query points; mirrors ``PreparedOptixFixedRadiusQueryPoints3D``
    (``optix_runtime.py:1843-1910``)."""

    def __init__(self, query_points):
        addr, n, dim, keep = _pack_any(query_points, 3)
        if dim != 3:
            raise ValueError("prepare_b200_fixed_radius_query_points_3d requires 3-D points")
        super().__init__(query_points, dimension=3)


class PreparedB200FixedRadiusNeighbors3D:
    """Prepared 3-D fixed-radius scene; mirrors ``PreparedOptixFixedRadiusNeighbors3D``
    (``optix_runtime.py:2315-2419``) on top of the C ABI's prepared entry points."""

    def __init__(self, search_points, *, max_radius: float):
        if max_radius <= 0:
            raise ValueError("max_radius must be positive")
        addr, n, dim, keep = _pack_any(search_points, 3)
        if dim != 3:
            raise ValueError("prepare_b200_fixed_radius_neighbors_3d requires 3-D points")
        self._keep = keep
        self._count = n
        self._max_radius = float(max_radius)
        self._handle = ctypes.c_void_p()
        self._closed = False
        if n == 0:
            return
        lib = _native.load_library()
        err = _native.error_buffer()
        status = lib.rtdl_b200_prepare_fixed_radius_neighbors_3d(addr, n, ctypes.c_double(self._max_radius),
                                                                 ctypes.byref(self._handle), err, len(err))
        _native.check_status(status, err)

    @property
    def max_radius(self) -> float:
        return self._max_radius

    @property
    def closed(self) -> bool:
        return self._closed

    def run_raw(self, query_points, *, radius: float, k_max: int) -> B200RowView:
        if self._closed:
            raise RuntimeError("prepared b200 fixed-radius-neighbor 3D handle is closed")
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > self._max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if k_max <= 0:
            raise ValueError("k_max must be positive")
        addr, n, dim, keep = _pack_any(query_points, 3)
        if dim != 3:
            raise ValueError("PreparedB200FixedRadiusNeighbors3D.run_raw requires 3-D points")
        if n == 0 or self._count == 0:
            return _row_view(0, 0, False)
        lib = _native.load_library()
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = lib.rtdl_b200_run_prepared_fixed_radius_neighbors_3d(
            self._handle, addr, n, ctypes.c_double(float(radius)), ctypes.c_size_t(int(k_max)),
            ctypes.byref(rows), ctypes.byref(count), err, len(err))
        del keep
        _native.check_status(status, err)
        return _row_view(rows.value or 0, count.value, False)

    def run(self, query_points, *, radius: float, k_max: int) -> tuple:
        view = self.run_raw(query_points, radius=radius, k_max=k_max)
        try:
            return view.to_dict_rows()
        finally:
            view.close()

    def _summary_checks(self, query_points, radius: float, k_max: int, what: str):
        if self._closed:
            raise RuntimeError("prepared b200 fixed-radius-neighbor 3D handle is closed")
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > self._max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if k_max <= 0:
            raise ValueError("k_max must be positive")
        if k_max > 64:
            raise ValueError(f"PreparedB200FixedRadiusNeighbors3D.{what} currently supports k_max <= 64")
        addr, n, dim, keep = _pack_any(query_points, 3)
        if dim != 3:
            raise ValueError(f"PreparedB200FixedRadiusNeighbors3D.{what} requires 3-D points")
        return addr, n, keep

    def run_ranked_summary_raw(self, query_points, *, radius: float, k_max: int) -> B200RowView:
        """One ranked summary per query (``optix_runtime.py:2541-2609``)."""
        addr, n, keep = self._summary_checks(query_points, radius, k_max, "run_ranked_summary_raw")
        if n == 0 or self._count == 0:
            return B200RowView(0, 0, SUMMARY_DTYPE, SUMMARY_DTYPE.names)
        lib = _native.load_library()
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = lib.rtdl_b200_run_prepared_ranked_fixed_radius_neighbor_summaries_3d(
            self._handle, addr, n, float(radius), int(k_max), ctypes.byref(rows), ctypes.byref(count), err, len(err))
        del keep
        _native.check_status(status, err)
        return B200RowView(rows.value or 0, count.value, SUMMARY_DTYPE, SUMMARY_DTYPE.names)

    def run_ranked_summary(self, query_points, *, radius: float, k_max: int) -> tuple:
        view = self.run_ranked_summary_raw(query_points, radius=radius, k_max=k_max)
        try:
            return view.to_dict_rows()
        finally:
            view.close()

    def aggregate_ranked_summary_prepared_queries(self, prepared_queries: B200Queries, *, radius: float, k_max: int,
                                                  precision: str = "float32") -> dict:
        """Aggregate over a prepared query set (``optix_runtime.py:2689-2750``); exact FP64 distances
        whatever ``precision`` names."""
        if prepared_queries.closed:
            raise RuntimeError("prepared b200 fixed-radius query handle is closed")
        if precision not in {"float64", "float32"}:
            raise ValueError("precision must be 'float64' or 'float32'")
        if self._closed:
            raise RuntimeError("prepared b200 fixed-radius-neighbor 3D handle is closed")
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > self._max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if k_max <= 0:
            raise ValueError("k_max must be positive")
        if k_max > 64:
            raise ValueError("PreparedB200FixedRadiusNeighbors3D.aggregate_ranked_summary_prepared_queries "
                             "currently supports k_max <= 64")
        if prepared_queries.count == 0 or self._count == 0:
            return {"query_count": int(prepared_queries.count), "bounded_neighbor_count": 0,
                    "nearest_id_checksum": 0, "kth_id_checksum": 0, "sum_distance": 0.0}
        agg = _native.RtdlFixedRadiusRankedNeighborAggregate()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d(
            self._handle, prepared_queries.handle, float(radius), int(k_max), ctypes.byref(agg), err, len(err))
        _native.check_status(status, err)
        return {f: (float(getattr(agg, f)) if f == "sum_distance" else int(getattr(agg, f))) for f in AGGREGATE_FIELDS}

    def aggregate_ranked_summary(self, query_points, *, radius: float, k_max: int,
                                 precision: str = "float64") -> dict:
        """The aggregate over all queries (``optix_runtime.py:2618-2687``); the distances are exact
        FP64 whatever ``precision`` names."""
        if precision not in {"float64", "float32"}:
            raise ValueError("precision must be 'float64' or 'float32'")
        addr, n, keep = self._summary_checks(query_points, radius, k_max, "aggregate_ranked_summary")
        if n == 0 or self._count == 0:
            return {"query_count": int(n), "bounded_neighbor_count": 0, "nearest_id_checksum": 0,
                    "kth_id_checksum": 0, "sum_distance": 0.0}
        agg = _native.RtdlFixedRadiusRankedNeighborAggregate()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_aggregate_prepared_ranked_fixed_radius_neighbor_summaries_3d(
            self._handle, addr, n, float(radius), int(k_max), ctypes.byref(agg), err, len(err))
        del keep
        _native.check_status(status, err)
        return {f: (float(getattr(agg, f)) if f == "sum_distance" else int(getattr(agg, f))) for f in AGGREGATE_FIELDS}

    def prepare_ranked_summary_prepared_queries_batch_graph(
            self, prepared_queries: B200Queries, requests, *,
            precision: str = "float32") -> "PreparedB200FixedRadiusRankedSummaryAggregateBatchGraph3D":
        """A captured CUDA graph of ranked-summary aggregates for several (radius, k_max)
        requests over one prepared query set (``optix_runtime.py:2838-2856``)."""
        if self._closed:
            raise RuntimeError("prepared b200 fixed-radius-neighbor 3D handle is closed")
        if prepared_queries.closed:
            raise RuntimeError("prepared b200 fixed-radius query handle is closed")
        return PreparedB200FixedRadiusRankedSummaryAggregateBatchGraph3D(self, prepared_queries, requests,
                                                                          precision=precision)

    def close(self) -> None:
        if not self._closed:
            if self._handle.value:
                _native.load_library().rtdl_b200_destroy_prepared_fixed_radius_neighbors_3d(self._handle)
            self._closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _normalize_graph_requests(owner: PreparedB200FixedRadiusNeighbors3D, requests) -> tuple:
    """Request checks of the reference's graph (``optix_runtime.py:2292-2312``)."""
    normalized = tuple(dict(r) for r in requests)
    if not normalized:
        raise ValueError("prepared fixed-radius aggregate graph requires at least one request")
    out = []
    for r in normalized:
        radius = float(r["radius"])
        k_max = int(r["k_max"])
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > owner.max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if k_max <= 0:
            raise ValueError("k_max must be positive")
        if k_max > 64:
            raise ValueError("PreparedB200FixedRadiusNeighbors3D prepared query aggregate graph currently supports "
                             "k_max <= 64")
        out.append({"radius": radius, "k_max": k_max})
    return tuple(out)


class _DeviceArray:
    """A raw device buffer exposed through ``__cuda_array_interface__`` (read by torch.as_tensor)."""

    def __init__(self, address: int, nbytes: int, stream: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (address, False),
                                         "version": 3, "stream": stream or None}


class PreparedB200FixedRadiusRankedSummaryAggregateBatchGraph3D:
    """Captured CUDA graph of prepared-query ranked-summary aggregates; mirrors
    ``PreparedOptixFixedRadiusRankedSummaryAggregateBatchGraph3D`` (``optix_runtime.py:1912-2289``).

    The graph holds the whole fixed-radius path of every request (collect, refinement of heavy
    queries, emit, summary, aggregate) over buffers allocated once, and runs on its own stream.
    The aggregates are exact (FP64 distances) whatever ``precision`` names; requests whose heavy
    queries the captured refinement leaves unresolved are recomputed by the plain call."""

    def __init__(self, owner: PreparedB200FixedRadiusNeighbors3D, prepared_queries: B200Queries, requests, *,
                 precision: str = "float32"):
        if precision not in {"float32", "float64"}:
            raise ValueError("precision must be 'float32' or 'float64'")
        if owner.closed:
            raise RuntimeError("prepared b200 fixed-radius-neighbor 3D handle is closed")
        if prepared_queries.closed:
            raise RuntimeError("prepared b200 fixed-radius query handle is closed")
        self._owner = owner
        self._prepared_queries = prepared_queries
        self._requests = _normalize_graph_requests(owner, requests)
        self._precision = precision
        self._handle = ctypes.c_void_p()
        self._closed = False
        self._request_buffer_update_count = 0
        self._empty = prepared_queries.count == 0 or owner._count == 0
        if self._empty:
            return
        self._call("rtdl_b200_prepare_fixed_radius_ranked_summary_aggregate_batch_graph_3d", owner._handle,
                   prepared_queries.handle, *self._request_arrays(self._requests), ctypes.byref(self._handle))

    @staticmethod
    def _request_arrays(requests):
        n = len(requests)
        radii = (ctypes.c_double * n)(*[r["radius"] for r in requests])
        k_values = (ctypes.c_size_t * n)(*[r["k_max"] for r in requests])
        return radii, k_values, ctypes.c_size_t(n)

    @staticmethod
    def _call(name, *args):
        err = _native.error_buffer()
        status = getattr(_native.load_library(), name)(*args, err, len(err))
        _native.check_status(status, err)

    def _check_open(self):
        if self._closed:
            raise RuntimeError("prepared fixed-radius aggregate graph handle is closed")
        if self._owner.closed:
            raise RuntimeError("prepared b200 fixed-radius-neighbor 3D handle is closed")
        if self._prepared_queries.closed:
            raise RuntimeError("prepared b200 fixed-radius query handle is closed")

    @property
    def closed(self) -> bool:
        return self._closed

    @property
    def request_buffer_update_count(self) -> int:
        return self._request_buffer_update_count

    @property
    def fallback_count(self) -> int:
        """Requests recomputed by the plain call so far (heavy queries the refinement left)."""
        if self._empty:
            return 0
        fb = ctypes.c_uint64()
        self._call("rtdl_b200_fixed_radius_ranked_summary_aggregate_batch_graph_status_device_3d", self._handle,
                   None, ctypes.byref(fb))
        return int(fb.value)

    def _result(self, index: int, agg: dict, **extra) -> dict:
        out = {
            "query_count": int(agg["query_count"]),
            "bounded_neighbor_count": int(agg["bounded_neighbor_count"]),
            "nearest_id_checksum": int(agg["nearest_id_checksum"]),
            "kth_id_checksum": int(agg["kth_id_checksum"]),
            "sum_distance": float(agg["sum_distance"]),
            "precision": self._precision,
            "query_resident": True,
            "request_index": index,
            "radius": float(self._requests[index]["radius"]),
            "k_max": int(self._requests[index]["k_max"]),
            "cuda_graph_replay": True,
            "request_buffer_update_count": self._request_buffer_update_count,
        }
        out.update(extra)
        return out

    def _empty_results(self, **extra) -> tuple:
        zero = {"query_count": int(self._prepared_queries.count), "bounded_neighbor_count": 0,
                "nearest_id_checksum": 0, "kth_id_checksum": 0, "sum_distance": 0.0}
        return tuple(self._result(i, zero, **extra) for i in range(len(self._requests)))

    def update_requests(self, requests) -> None:
        """New (radius, k_max) requests, same count; the graph is captured again."""
        self._check_open()
        normalized = _normalize_graph_requests(self._owner, requests)
        if len(normalized) != len(self._requests):
            raise ValueError("prepared fixed-radius aggregate graph request updates must keep request_count unchanged")
        if not self._empty:
            self._call("rtdl_b200_update_fixed_radius_ranked_summary_aggregate_batch_graph_3d", self._handle,
                       *self._request_arrays(normalized))
        self._requests = normalized
        self._request_buffer_update_count += 1

    def replay(self) -> tuple:
        self._check_open()
        if self._empty:
            return self._empty_results()
        aggs = (_native.RtdlFixedRadiusRankedNeighborAggregate * len(self._requests))()
        self._call("rtdl_b200_replay_fixed_radius_ranked_summary_aggregate_batch_graph_3d", self._handle, aggs)
        return tuple(self._result(i, {f: getattr(a, f) for f in AGGREGATE_FIELDS}) for i, a in enumerate(aggs))

    def launch_device_partials(self) -> tuple[int, int, int, int, int]:
        """Enqueues one replay without waiting; returns (partials device address, partial count,
        request count, query blocks per request, the graph's CUDA stream handle)."""
        self._check_open()
        if self._empty:
            raise RuntimeError("an empty prepared handle has no graph to launch")
        ptr, count, reqs, blocks, stream = (ctypes.c_uint64(), ctypes.c_size_t(), ctypes.c_size_t(),
                                            ctypes.c_size_t(), ctypes.c_uint64())
        self._call("rtdl_b200_launch_fixed_radius_ranked_summary_aggregate_batch_graph_device_partials_3d",
                   self._handle, ctypes.byref(ptr), ctypes.byref(count), ctypes.byref(reqs), ctypes.byref(blocks),
                   ctypes.byref(stream))
        n_req, n_blk = int(reqs.value), int(blocks.value)
        if n_req != len(self._requests) or int(count.value) != n_req * n_blk:
            raise RuntimeError("native fixed-radius graph returned inconsistent partial counts")
        return int(ptr.value), int(count.value), n_req, n_blk, int(stream.value)

    def replay_same_stream_device_partials_summary(self) -> dict:
        """Enqueues a replay and reduces the device partials with a torch consumer on the graph's
        stream (no host read between the graph and the consumer); the reference's CuPy consumer
        (``optix_runtime.py:2098-2270``) in torch.  Requests whose status word is nonzero are then
        recomputed by the plain aggregate call."""
        import torch

        self._check_open()
        if self._empty:
            return {"aggregates": self._empty_results(same_stream_partner_reduced=False),
                    "metadata": {"backend": "b200", "empty_graph_path": True,
                                 "same_stream_partner_consumer_executed": False}}
        ptr, count, n_req, n_blk, stream = self.launch_device_partials()
        status_ptr = ctypes.c_uint64()
        self._call("rtdl_b200_fixed_radius_ranked_summary_aggregate_batch_graph_status_device_3d", self._handle,
                   ctypes.byref(status_ptr), None)
        ext = torch.cuda.ExternalStream(stream)
        with torch.cuda.stream(ext):
            raw = torch.as_tensor(_DeviceArray(ptr, count * 40, stream), device="cuda")
            words = raw.view(torch.int64).view(n_req, n_blk, 5)
            ints = words[:, :, :4].sum(dim=1)
            sums = words[:, :, 4].view(torch.float64).sum(dim=1)
            status = torch.as_tensor(_DeviceArray(int(status_ptr.value), n_req * 4, stream),
                                     device="cuda").view(torch.int32).clone()
            ints_h, sums_h, status_h = ints.cpu(), sums.cpu(), status.cpu()  # waits on the graph's stream
        aggregates = []
        recomputed = 0
        for i in range(n_req):
            if int(status_h[i]) != 0:
                agg = self._owner.aggregate_ranked_summary_prepared_queries(
                    self._prepared_queries, radius=self._requests[i]["radius"], k_max=self._requests[i]["k_max"])
                recomputed += 1
            else:
                agg = dict(zip(AGGREGATE_FIELDS[:4], (int(v) for v in ints_h[i].tolist())))
                agg["sum_distance"] = float(sums_h[i])
            aggregates.append(self._result(i, agg, same_stream_partner_reduced=int(status_h[i]) == 0))
        return {"aggregates": tuple(aggregates),
                "metadata": {"backend": "b200", "native_symbol":
                             "rtdl_b200_launch_fixed_radius_ranked_summary_aggregate_batch_graph_device_partials_3d",
                             "producer_consumer_stream_ordering": "same_cuda_stream",
                             "producer_host_synchronization_used": False,
                             "bounded_partner_consumer": "torch",
                             "partial_row_size_bytes": 40, "partial_count": count,
                             "request_count": n_req, "query_block_count": n_blk,
                             "requests_recomputed_by_plain_call": recomputed}}

    # the reference's name for the same-stream consumer (its consumer is CuPy, this one is torch)
    replay_same_stream_device_partials_summary_cupy = replay_same_stream_device_partials_summary

    def close(self) -> None:
        if self._closed:
            return
        handle = self._handle
        self._handle = ctypes.c_void_p()
        self._closed = True
        if handle.value:
            _native.load_library().rtdl_b200_destroy_fixed_radius_ranked_summary_aggregate_batch_graph_3d(handle)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_address(obj) -> int:
    """Device address of a partner buffer: a torch tensor, an object exposing
    ``__cuda_array_interface__``, or an int address."""
    if obj is None:
        return 0
    if isinstance(obj, int):
        return obj
    if hasattr(obj, "data_ptr"):
        return int(obj.data_ptr())
    cai = getattr(obj, "__cuda_array_interface__", None)
    if cai is not None:
        return int(cai["data"][0])
    raise TypeError("expected a CUDA tensor, a __cuda_array_interface__ object or a device address")


def _count_rows(view: B200RowView) -> tuple:
    try:
        return tuple({"query_id": int(r["query_id"]), "neighbor_count": int(r["neighbor_count"]),
                      "threshold_reached": int(r["threshold_reached"])} for r in view.to_numpy())
    finally:
        view.close()


def fixed_radius_count_threshold_2d(query_points, search_points=None, *, radius: float,
                                    threshold: int = 0) -> tuple:
    """One row per query: its in-radius count, stopped at ``threshold`` when positive, and whether it was
    reached; mirrors ``fixed_radius_count_threshold_2d_optix`` (``optix_runtime.py:1430-1492``)."""
    if radius < 0:
        raise ValueError("radius must be non-negative")
    if threshold < 0:
        raise ValueError("threshold must be non-negative")
    qa, qn, qd, qk = _pack_any(query_points, 2)
    sa, sn, sd, sk = (qa, qn, qd, qk) if search_points is None else _pack_any(search_points, 2)
    rows = ctypes.c_void_p()
    count = ctypes.c_size_t()
    err = _native.error_buffer()
    status = _native.load_library().rtdl_b200_run_fixed_radius_count_threshold(
        qa, qn, sa, sn, float(radius), int(threshold), ctypes.byref(rows), ctypes.byref(count), err, len(err))
    del qk, sk
    _native.check_status(status, err)
    return _count_rows(B200RowView(rows.value or 0, count.value, COUNT_ROW_DTYPE, COUNT_ROW_DTYPE.names))


class PreparedB200FixedRadiusCountThreshold2D:
    """Prepared 2-D fixed-radius count-threshold scene; mirrors ``PreparedOptixFixedRadiusCountThreshold2D``
    (``optix_runtime.py:1495-1842``)."""

    def __init__(self, search_points, *, max_radius: float):
        if max_radius < 0:
            raise ValueError("max_radius must be non-negative")
        addr, n, dim, keep = _pack_any(search_points, 2)
        if dim != 2:
            raise ValueError("prepare_b200_fixed_radius_count_threshold_2d requires 2-D points")
        self._count = n
        self._max_radius = float(max_radius)
        self._handle = ctypes.c_void_p()
        self._closed = False
        self._search_scene_true_zero_copy = False
        if n == 0:
            return
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_prepare_fixed_radius_count_threshold_2d(
            addr, n, ctypes.c_double(self._max_radius), ctypes.byref(self._handle), err, len(err))
        del keep
        _native.check_status(status, err)

    @classmethod
    def from_device_columns(cls, search_point_columns: dict, *, max_radius: float):
        """From partner-owned device columns ``ids`` (u32), ``x``, ``y`` (f64); mirrors
        ``prepare_optix_fixed_radius_count_threshold_2d_device_search_columns`` (``optix_runtime.py:4215-4270``)."""
        if max_radius < 0:
            raise ValueError("max_radius must be non-negative")
        self = cls.__new__(cls)
        n = int(search_point_columns.get("count", len(search_point_columns["ids"])))
        self._count = n
        self._max_radius = float(max_radius)
        self._handle = ctypes.c_void_p()
        self._closed = False
        self._search_scene_true_zero_copy = True
        if n == 0:
            return self
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_prepare_fixed_radius_count_threshold_2d_device_search_columns(
            _device_address(search_point_columns["ids"]), _device_address(search_point_columns["x"]),
            _device_address(search_point_columns["y"]), n, ctypes.c_double(self._max_radius),
            ctypes.byref(self._handle), err, len(err))
        _native.check_status(status, err)
        return self

    @property
    def max_radius(self) -> float:
        return self._max_radius

    @property
    def closed(self) -> bool:
        return self._closed

    def _checks(self, radius: float, threshold: int = 0):
        if self._closed:
            raise RuntimeError("prepared b200 fixed-radius count handle is closed")
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > self._max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if threshold < 0:
            raise ValueError("threshold must be non-negative")

    def _queries(self, query_points, what: str):
        addr, n, dim, keep = _pack_any(query_points, 2)
        if dim != 2:
            raise ValueError(f"PreparedB200FixedRadiusCountThreshold2D.{what} requires 2-D points")
        return addr, n, keep

    def run(self, query_points, *, radius: float, threshold: int = 0) -> tuple:
        self._checks(radius, threshold)
        addr, n, keep = self._queries(query_points, "run")
        if n == 0 or self._count == 0:
            return ()
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_run_prepared_fixed_radius_count_threshold_2d(
            self._handle, addr, n, float(radius), int(threshold), ctypes.byref(rows), ctypes.byref(count), err,
            len(err))
        del keep
        _native.check_status(status, err)
        return _count_rows(B200RowView(rows.value or 0, count.value, COUNT_ROW_DTYPE, COUNT_ROW_DTYPE.names))

    def count_threshold_reached(self, query_points, *, radius: float, threshold: int = 0) -> int:
        """How many queries reached ``threshold`` (the scalar path, no rows)."""
        self._checks(radius, threshold)
        addr, n, keep = self._queries(query_points, "count_threshold_reached")
        if n == 0 or self._count == 0:
            return 0
        out = ctypes.c_size_t()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_count_prepared_fixed_radius_threshold_reached_2d(
            self._handle, addr, n, float(radius), int(threshold), ctypes.byref(out), err, len(err))
        del keep
        _native.check_status(status, err)
        return int(out.value)

    def nearest_witness_rows(self, query_points, *, radius: float) -> tuple:
        """One row per query: its nearest in-radius point (neighbor_id 0xFFFFFFFF, distance FLT_MAX when none)."""
        self._checks(radius)
        addr, n, keep = self._queries(query_points, "nearest_witness_rows")
        if n == 0 or self._count == 0:
            return ()
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_run_prepared_fixed_radius_nearest_witness_2d(
            self._handle, addr, n, float(radius), ctypes.byref(rows), ctypes.byref(count), err, len(err))
        del keep
        _native.check_status(status, err)
        view = _row_view(rows.value or 0, count.value, False)
        try:
            return view.to_dict_rows()
        finally:
            view.close()

    def write_device_count_threshold_columns(self, query_point_columns: dict, *, radius: float, threshold: int,
                                             query_ids_out, neighbor_counts_out, threshold_flags_out) -> dict:
        """Device query columns (``ids``, ``x``, ``y``) in, device output columns out; needs a scene prepared
        from device columns (``from_device_columns``)."""
        self._checks(radius, threshold)
        if not self._search_scene_true_zero_copy:
            raise RuntimeError("write_device_count_threshold_columns requires a device-search-column prepared scene")
        n = int(query_point_columns.get("count", len(query_point_columns["ids"])))
        meta = {"backend": "b200", "query_count": n, "radius": float(radius), "threshold": int(threshold)}
        if n == 0 or self._count == 0:
            return {"metadata": meta}
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_write_prepared_fixed_radius_count_threshold_2d_device_query_columns(
            self._handle, _device_address(query_point_columns["ids"]), _device_address(query_point_columns["x"]),
            _device_address(query_point_columns["y"]), n, float(radius), int(threshold),
            _device_address(query_ids_out), _device_address(neighbor_counts_out), _device_address(threshold_flags_out),
            err, len(err))
        _native.check_status(status, err)
        return {"metadata": meta}

    def close(self) -> None:
        if not self._closed:
            if self._handle.value:
                _native.load_library().rtdl_b200_destroy_prepared_fixed_radius_count_threshold_2d(self._handle)
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


class PreparedB200FixedRadiusCountThreshold3D:
    """Prepared 3-D fixed-radius count-threshold scene; mirrors ``PreparedOptixFixedRadiusCountThreshold3D``
    (``optix_runtime.py:2974-3110``): host query records in, caller-owned device columns out."""

    def __init__(self, search_points, *, max_radius: float):
        if max_radius <= 0:
            raise ValueError("max_radius must be positive")
        addr, n, dim, keep = _pack_any(search_points, 3)
        if dim != 3:
            raise ValueError("prepare_b200_fixed_radius_count_threshold_3d requires 3-D points")
        self._count = n
        self._max_radius = float(max_radius)
        self._handle = ctypes.c_void_p()
        self._closed = False
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_prepare_fixed_radius_count_threshold_3d(
            addr, n, ctypes.c_double(self._max_radius), ctypes.byref(self._handle), err, len(err))
        del keep
        _native.check_status(status, err)

    @property
    def max_radius(self) -> float:
        return self._max_radius

    @property
    def closed(self) -> bool:
        return self._closed

    def write_device_count_threshold_columns(self, query_points, *, radius: float, threshold: int,
                                             query_ids_out, neighbor_counts_out, threshold_flags_out) -> dict:
        if self._closed:
            raise RuntimeError("prepared b200 fixed-radius count-threshold 3D handle is closed")
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > self._max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if threshold < 0:
            raise ValueError("threshold must be non-negative")
        addr, n, dim, keep = _pack_any(query_points, 3)
        if dim != 3:
            raise ValueError("write_device_count_threshold_columns requires 3-D query points")
        meta = {"backend": "b200", "query_count": n, "search_count": self._count, "radius": float(radius),
                "threshold": int(threshold), "materializes_neighbor_rows": False}
        if n == 0:
            return {"metadata": meta}
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_write_prepared_fixed_radius_count_threshold_3d_device_outputs(
            self._handle, addr, n, float(radius), int(threshold), _device_address(query_ids_out),
            _device_address(neighbor_counts_out), _device_address(threshold_flags_out), err, len(err))
        del keep
        _native.check_status(status, err)
        return {"metadata": meta}

    def close(self) -> None:
        if not self._closed:
            if self._handle.value:
                _native.load_library().rtdl_b200_destroy_prepared_fixed_radius_count_threshold_3d(self._handle)
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


POINT_GROUP_DTYPE = np.dtype({"names": ["id", "point_offset", "point_count", "min_x", "min_y", "max_x", "max_y"],
                              "formats": ["<u4", "<u4", "<u4", "<f8", "<f8", "<f8", "<f8"],
                              "offsets": [0, 4, 8, 16, 24, 32, 40], "itemsize": 48})


def pack_point_groups(groups) -> np.ndarray:
    """Groups (mappings or objects with id, point_offset, point_count, min_x, min_y, max_x, max_y, or a
    structured array) as ``RtdlPointGroupBounds2D`` records."""
    if isinstance(groups, np.ndarray) and groups.dtype.names:
        out = np.zeros(len(groups), dtype=POINT_GROUP_DTYPE)
        for f in POINT_GROUP_DTYPE.names:
            out[f] = groups[f]
        return out
    rows = tuple(groups)
    out = np.zeros(len(rows), dtype=POINT_GROUP_DTYPE)
    for i, g in enumerate(rows):
        for f in POINT_GROUP_DTYPE.names:
            out[f][i] = g[f] if isinstance(g, Mapping) else getattr(g, f)
    return out


class PreparedB200PointGroupNearestWitness2D:
    """Prepared 2-D point-group scene; mirrors ``PreparedOptixPointGroupNearestWitness2D``
    (``optix_runtime.py:4284-4540``): threshold coverage and one nearest in-radius witness per query over
    search points that belong to groups whose box is within radius."""

    def __init__(self, search_points, groups, *, max_radius: float):
        if max_radius < 0:
            raise ValueError("max_radius must be non-negative")
        addr, n, dim, keep = _pack_any(search_points, 2)
        if dim != 2:
            raise ValueError("prepare_b200_point_group_nearest_witness_2d requires 2-D points")
        self._groups = pack_point_groups(groups)
        self._count = n
        self._group_count = len(self._groups)
        self._max_radius = float(max_radius)
        self._handle = ctypes.c_void_p()
        self._closed = False
        if n == 0 or self._group_count == 0:
            return
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_prepare_point_group_nearest_witness_2d(
            addr, n, self._groups.ctypes.data, self._group_count, ctypes.c_double(self._max_radius),
            ctypes.byref(self._handle), err, len(err))
        del keep
        _native.check_status(status, err)

    @property
    def max_radius(self) -> float:
        return self._max_radius

    @property
    def closed(self) -> bool:
        return self._closed

    def _checks(self, radius: float, threshold: int = 0):
        if self._closed:
            raise RuntimeError("prepared b200 point-group handle is closed")
        if radius < 0:
            raise ValueError("radius must be non-negative")
        if radius > self._max_radius:
            raise ValueError("radius must be less than or equal to prepared max_radius")
        if threshold < 0:
            raise ValueError("threshold must be non-negative")

    def _queries(self, query_points, what: str):
        addr, n, dim, keep = _pack_any(query_points, 2)
        if dim != 2:
            raise ValueError(f"PreparedB200PointGroupNearestWitness2D.{what} requires 2-D points")
        return addr, n, keep

    @property
    def _empty(self) -> bool:
        return self._count == 0 or self._group_count == 0

    def count_threshold_reached(self, query_points, *, radius: float, threshold: int = 0) -> int:
        self._checks(radius, threshold)
        addr, n, keep = self._queries(query_points, "count_threshold_reached")
        if n == 0 or self._empty:
            return 0
        out = ctypes.c_size_t()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_count_prepared_point_group_threshold_reached_2d(
            self._handle, addr, n, float(radius), int(threshold), ctypes.byref(out), err, len(err))
        del keep
        _native.check_status(status, err)
        return int(out.value)

    def threshold_flags(self, query_points, *, radius: float, threshold: int = 0) -> np.ndarray:
        """One uint32 threshold-reached flag per query point."""
        self._checks(radius, threshold)
        addr, n, keep = self._queries(query_points, "threshold_flags")
        if n == 0:
            return np.asarray([], dtype=np.uint32)
        if self._empty:
            return np.full(n, 1 if int(threshold) == 0 else 0, dtype=np.uint32)
        flags = np.zeros(n, dtype=np.uint32)
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_write_prepared_point_group_threshold_flags_2d(
            self._handle, addr, n, float(radius), int(threshold), flags.ctypes.data, err, len(err))
        del keep
        _native.check_status(status, err)
        return flags

    def nearest_witness_rows(self, query_points, *, radius: float) -> tuple:
        self._checks(radius)
        addr, n, keep = self._queries(query_points, "nearest_witness_rows")
        if n == 0 or self._empty:
            return ()
        rows = ctypes.c_void_p()
        count = ctypes.c_size_t()
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_run_prepared_point_group_nearest_witness_2d(
            self._handle, addr, n, float(radius), ctypes.byref(rows), ctypes.byref(count), err, len(err))
        del keep
        _native.check_status(status, err)
        view = _row_view(rows.value or 0, count.value, False)
        try:
            return view.to_dict_rows()
        finally:
            view.close()

    def nearest_max_distance_row(self, query_points, *, radius: float) -> dict:
        """The witness row of largest distance, reduced on the device."""
        self._checks(radius)
        addr, n, keep = self._queries(query_points, "nearest_max_distance_row")
        if n == 0 or self._empty:
            return {"query_id": 0xFFFFFFFF, "neighbor_id": 0xFFFFFFFF, "distance": float("inf")}
        row = np.zeros(1, dtype=FRN_ROW_DTYPE)
        err = _native.error_buffer()
        status = _native.load_library().rtdl_b200_reduce_prepared_point_group_nearest_max_distance_2d(
            self._handle, addr, n, float(radius), row.ctypes.data, err, len(err))
        del keep
        _native.check_status(status, err)
        return {"query_id": int(row["query_id"][0]), "neighbor_id": int(row["neighbor_id"][0]),
                "distance": float(row["distance"][0])}

    def close(self) -> None:
        if not self._closed:
            if self._handle.value:
                _native.load_library().rtdl_b200_destroy_prepared_point_group_nearest_witness_2d(self._handle)
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


def prepare_b200_point_group_nearest_witness_2d(search_points, groups, *, max_radius: float):
    return PreparedB200PointGroupNearestWitness2D(search_points, groups, max_radius=max_radius)


def prepare_b200_fixed_radius_count_threshold_2d(search_points, *, max_radius: float):
    return PreparedB200FixedRadiusCountThreshold2D(search_points, max_radius=max_radius)


def prepare_b200_fixed_radius_count_threshold_2d_device_search_columns(search_point_columns: dict, *,
                                                                       max_radius: float):
    return PreparedB200FixedRadiusCountThreshold2D.from_device_columns(search_point_columns, max_radius=max_radius)


def prepare_b200_fixed_radius_count_threshold_3d(search_points, *, max_radius: float):
    return PreparedB200FixedRadiusCountThreshold3D(search_points, max_radius=max_radius)


def prepare_b200_fixed_radius_neighbors_3d(search_points, *, max_radius: float) -> PreparedB200FixedRadiusNeighbors3D:
    return PreparedB200FixedRadiusNeighbors3D(search_points, max_radius=max_radius)


def directed_hausdorff(query_points, search_points, *, dimension: int | None = None) -> dict:
    """Directed Hausdorff witness (max over queries of the exact nearest distance,
    ties to the smaller query id then neighbor id), reduced on the device."""
    with B200Scene(search_points, dimension=dimension) as scene:
        return scene.directed_hausdorff(query_points)


def hausdorff_distance(points_a, points_b, *, dimension: int | None = None) -> dict:
    """Undirected Hausdorff as the reference app reports it
    (``rtdl_hausdorff_distance_app.py:152``): both directions, the larger wins
    with the direction name as the tie-break."""
    ab = directed_hausdorff(points_a, points_b, dimension=dimension)
    ba = directed_hausdorff(points_b, points_a, dimension=dimension)
    direction, best = max((("a_to_b", ab), ("b_to_a", ba)), key=lambda item: (float(item[1]["distance"]), item[0]))
    return {
        "directed_a_to_b": ab,
        "directed_b_to_a": ba,
        "hausdorff_distance": float(best["distance"]),
        "witness_direction": direction,
    }


def set_tuning(*, leaf_size: int = 0, block_threads: int = 128, traversal: str = "packet_hybrid") -> None:
    """Set the kernel tuning knobs (see ``rtdl_b200_set_tuning``); ``leaf_size`` 0 keeps the default
    leaf bucket size (32 points)."""
    modes = {"packet": 0, "lane": 1, "packet_cube": 2, "packet_points": 3, "packet_hybrid": 4}
    if traversal not in modes:
        raise ValueError("traversal must be 'packet', 'lane', 'packet_cube', 'packet_points' or 'packet_hybrid'")
    status = _native.load_library().rtdl_b200_set_tuning(int(leaf_size), int(block_threads), modes[traversal])
    if status != 0:
        raise ValueError("leaf_size must be in [0, 32] and block_threads one of 64, 128, 256")


def set_device(device: int) -> None:
    if _native.load_library().rtdl_b200_set_device(int(device)) != 0:
        raise RuntimeError(f"cannot select CUDA device {device}")
