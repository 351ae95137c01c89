"""ctypes wrapper over the CPU restatement in ``nn_oracle.c`` (test infrastructure).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  It is the checker, never the product: the CUDA backend
(``rtdl_b200``) does not import it.

The semantics restate ``src/rtdsl/reference.py:349-434`` and ``:882-890`` of
rubaolee/rtdl (see the header of ``nn_oracle.c`` for the line-by-line mapping).
Inputs are numpy columns; outputs are numpy structured arrays whose dtypes
match the reference ABI rows ``RtdlFixedRadiusNeighborRow`` {u32, u32, f64}
and ``RtdlKnnNeighborRow`` {u32, u32, f64, u32}
(``src/native/optix/rtdl_optix_prelude.h:254-295``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libnn_oracle.so"
REF_LIB_PATH = HERE / "_ref" / "librtdl_oracle.so"

FRN_ROW_DTYPE = np.dtype(
    {"names": ["query_id", "neighbor_id", "distance"], "formats": ["<u4", "<u4", "<f8"], "offsets": [0, 4, 8], "itemsize": 16}
)
KNN_ROW_DTYPE = np.dtype(
    {
        "names": ["query_id", "neighbor_id", "distance", "neighbor_rank"],
        "formats": ["<u4", "<u4", "<f8", "<u4"],
        "offsets": [0, 4, 8, 16],
        "itemsize": 24,
    }
)

_lib = None


# Where the reference tree is read from (test infrastructure only: fixture
# generation, the cross-checks of the CPU tests, and compiling the reference's
# own oracle).  RTDL_REFERENCE_ROOT names it; when unset, the read-only mount of
# the build container is tried.  Nothing run on a GPU machine reads it.
_DEFAULT_REFERENCE_MOUNT = "/root/reference"


def reference_root() -> Path | None:
    """The reference tree, or None when it is not present on this machine."""
    root = Path(os.environ.get("RTDL_REFERENCE_ROOT") or _DEFAULT_REFERENCE_MOUNT)
    return root if (root / "src" / "rtdsl").is_dir() else None


def build() -> Path:
    """Compile ``libnn_oracle.so`` (and the reference's own oracle when its tree is present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    ref_root = reference_root()
    if ref_root is not None and (ref_root / "src" / "native" / "rtdl_oracle.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_ROOT={ref_root}"], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    u32p = ctypes.POINTER(ctypes.c_uint32)
    f64p = ctypes.POINTER(ctypes.c_double)
    lib.nn_oracle_rows.argtypes = [
        u32p, f64p, f64p, f64p, ctypes.c_size_t,
        u32p, f64p, f64p, f64p, ctypes.c_size_t,
        ctypes.c_int, ctypes.c_double, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
        ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t), u32p,
    ]
    lib.nn_oracle_rows.restype = ctypes.c_int
    lib.nn_oracle_nearest.argtypes = [
        u32p, f64p, f64p, f64p, ctypes.c_size_t,
        u32p, f64p, f64p, f64p, ctypes.c_size_t,
        ctypes.c_int, f64p, u32p,
    ]
    lib.nn_oracle_nearest.restype = ctypes.c_int
    lib.nn_oracle_rows_grid.argtypes = lib.nn_oracle_rows.argtypes
    lib.nn_oracle_rows_grid.restype = ctypes.c_int
    lib.nn_oracle_nearest_grid.argtypes = lib.nn_oracle_nearest.argtypes
    lib.nn_oracle_nearest_grid.restype = ctypes.c_int
    lib.nn_oracle_free.argtypes = [ctypes.c_void_p]
    lib.nn_oracle_free.restype = None
    _lib = lib
    return lib


def _columns(points):
    """Accepts an (n, 2|3) float array plus ids, or a dict with id/x/y[/z]."""
    ids = np.ascontiguousarray(points["id"], dtype=np.uint32)
    x = np.ascontiguousarray(points["x"], dtype=np.float64)
    y = np.ascontiguousarray(points["y"], dtype=np.float64)
    z = points.get("z") if isinstance(points, dict) else (points["z"] if "z" in points.dtype.names else None)
    z = None if z is None else np.ascontiguousarray(z, dtype=np.float64)
    return ids, x, y, z


def _ptr(a, ctype):
    if a is None:
        return ctypes.cast(None, ctypes.POINTER(ctype))
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _call_rows(query, search, mode, radius, k, ranked, threads, want_counts, grid=False):
    lib = _load()
    fn = lib.nn_oracle_rows_grid if grid else lib.nn_oracle_rows
    qid, qx, qy, qz = _columns(query)
    sid, sx, sy, sz = _columns(search)
    if (qz is None) != (sz is None):
        raise ValueError("query and search sets must have the same dimension")
    rows_ptr = ctypes.c_void_p()
    count = ctypes.c_size_t()
    counts = np.zeros(len(qid), dtype=np.uint32) if want_counts else None
    status = fn(
        _ptr(qid, ctypes.c_uint32), _ptr(qx, ctypes.c_double), _ptr(qy, ctypes.c_double), _ptr(qz, ctypes.c_double), len(qid),
        _ptr(sid, ctypes.c_uint32), _ptr(sx, ctypes.c_double), _ptr(sy, ctypes.c_double), _ptr(sz, ctypes.c_double), len(sid),
        mode, float(radius), int(k), int(ranked), int(threads),
        ctypes.byref(rows_ptr), ctypes.byref(count), _ptr(counts, ctypes.c_uint32),
    )
    if status != 0:
        raise RuntimeError("nn_oracle_rows failed (out of memory)")
    dtype = KNN_ROW_DTYPE if ranked else FRN_ROW_DTYPE
    n = count.value
    try:
        if n:
            buf = (ctypes.c_char * (n * dtype.itemsize)).from_address(rows_ptr.value)
            rows = np.frombuffer(buf, dtype=dtype).copy()
        else:
            rows = np.zeros(0, dtype=dtype)
    finally:
        lib.nn_oracle_free(rows_ptr)
    return (rows, counts) if want_counts else rows


def fixed_radius_neighbors(query, search, *, radius, k_max, threads=1, ranked=False, with_counts=False, grid=False):
    """FRN rows (``reference.py:349-376``); ``ranked=True`` gives bounded_knn_rows (``:406-434``).
    ``grid=True`` takes the candidates from a uniform grid over the search set instead of every
    search point (same arithmetic and keys, the same rows; for the full-size sets)."""
    return _call_rows(query, search, 0, radius, k_max, ranked, threads, with_counts, grid)


COUNT_ROW_DTYPE = np.dtype({"names": ["query_id", "neighbor_count", "threshold_reached"],
                            "formats": ["<u4", "<u4", "<u4"], "offsets": [0, 4, 8], "itemsize": 12})


def fixed_radius_count_threshold(query, search, *, radius, threshold, threads=1):
    """The reference's generic count (``src/rtdsl/generic_primitives.py:198-227``): per query, in input
    order, its points within radius counted until a positive threshold is reached (threshold 0 counts
    them all); ``threshold_reached`` is 1 when a positive threshold was reached.  Restated from the
    oracle's exact in-radius counts: the stopped count is min(count, threshold)."""
    _, counts = _call_rows(query, search, 0, radius, 1, False, threads, True)
    thr = int(threshold)
    out = np.zeros(len(counts), dtype=COUNT_ROW_DTYPE)
    out["query_id"] = np.asarray(query["id"], dtype=np.uint32)
    out["neighbor_count"] = np.minimum(counts, thr) if thr > 0 else counts
    out["threshold_reached"] = (counts >= thr) if thr > 0 else 0
    return out


def nearest_witness(query, search, *, radius, threads=1):
    """Nearest in-radius neighbour of each query, in input order (the reference's prepared nearest
    witness, ``rtdl_optix_core.cpp:6043-6090``: smaller distance, then smaller id); queries without
    one get neighbor_id 0xFFFFFFFF and distance FLT_MAX.  Restated from the k_max = 1 rows, which
    come grouped by query id, stable in input order."""
    rows, counts = _call_rows(query, search, 0, radius, 1, False, threads, True)
    ids = np.asarray(query["id"], dtype=np.uint32)
    out = np.zeros(len(ids), dtype=FRN_ROW_DTYPE)
    out["query_id"] = ids
    out["neighbor_id"] = 0xFFFFFFFF
    out["distance"] = 3.4028234663852886e38
    order = np.argsort(ids, kind="stable")
    hit = order[counts[order] > 0]
    out["neighbor_id"][hit] = rows["neighbor_id"]
    out["distance"][hit] = rows["distance"]
    return out


def point_group_witness(query, search, groups, *, radius, threshold=0):
    """The reference's prepared point-group kernels (``rtdl_optix_core.cpp:6119-6358``) restated in FP64
    (numpy, small cases): a search point takes part for a query when it and its group's box are within
    radius (inclusive), once per group holding it.  Returns (stopped counts, flags, witness rows, max row):
    counting stops at a positive threshold; the flag is 1 when it was reached; the witness is the nearest
    such point by distance then smaller id (0xFFFFFFFF / FLT_MAX when none); the max row is the witness of
    largest distance, then smaller query id, then smaller neighbour id, a missing witness counting as
    infinitely far."""
    qx = np.asarray(query["x"], dtype=np.float64)
    qy = np.asarray(query["y"], dtype=np.float64)
    qid = np.asarray(query["id"], dtype=np.uint32)
    sx = np.asarray(search["x"], dtype=np.float64)
    sy = np.asarray(search["y"], dtype=np.float64)
    sid = np.asarray(search["id"], dtype=np.uint32)
    r2 = float(radius) * float(radius)
    nq = len(qid)
    counts = np.zeros(nq, dtype=np.int64)
    best_d2 = np.full(nq, np.inf)
    best_id = np.full(nq, 0xFFFFFFFF, dtype=np.int64)
    for g in groups:
        lo, n = int(g["point_offset"]), int(g["point_count"])
        dxb = np.where(qx < g["min_x"], g["min_x"] - qx, np.where(qx > g["max_x"], qx - g["max_x"], 0.0))
        dyb = np.where(qy < g["min_y"], g["min_y"] - qy, np.where(qy > g["max_y"], qy - g["max_y"], 0.0))
        ok = (dxb * dxb + dyb * dyb) <= r2
        if n == 0 or not ok.any():
            continue
        qi = np.flatnonzero(ok)
        dx = sx[None, lo:lo + n] - qx[qi, None]
        dy = sy[None, lo:lo + n] - qy[qi, None]
        d2 = dx * dx + dy * dy
        inr = d2 <= r2
        counts[qi] += inr.sum(axis=1)
        d2m = np.where(inr, d2, np.inf)
        ids = sid[lo:lo + n].astype(np.int64)
        for row, q in enumerate(qi):
            m = d2m[row]
            if not np.isfinite(m).any():
                continue
            mn = m.min()
            cand = ids[m == mn].min()
            if mn < best_d2[q] or (mn == best_d2[q] and cand < best_id[q]):
                best_d2[q] = mn
                best_id[q] = cand
    thr = int(threshold)
    stopped = np.minimum(counts, thr) if thr > 0 else counts
    flags = (counts >= thr).astype(np.uint32) if thr > 0 else np.zeros(nq, dtype=np.uint32)
    rows = np.zeros(nq, dtype=FRN_ROW_DTYPE)
    rows["query_id"] = qid
    found = np.isfinite(best_d2)
    rows["neighbor_id"] = np.where(found, best_id, 0xFFFFFFFF).astype(np.uint32)
    rows["distance"] = np.where(found, np.sqrt(np.where(found, best_d2, 0.0)), 3.4028234663852886e38)
    key = np.where(found, rows["distance"], np.inf)
    order = np.lexsort((rows["neighbor_id"], rows["query_id"], -key))
    top = order[0] if nq else None
    max_row = {"query_id": 0xFFFFFFFF, "neighbor_id": 0xFFFFFFFF, "distance": float("inf")} if top is None else {
        "query_id": int(rows["query_id"][top]), "neighbor_id": int(rows["neighbor_id"][top]),
        "distance": float(key[top])}
    return stopped.astype(np.uint32), flags, rows, max_row


SUMMARY_DTYPE = np.dtype(
    {
        "names": ["query_id", "neighbor_count", "nearest_neighbor_id", "kth_neighbor_id", "nearest_distance",
                  "kth_distance", "sum_distance"],
        "formats": ["<u4", "<u4", "<u4", "<u4", "<f8", "<f8", "<f8"],
        "offsets": [0, 4, 8, 12, 16, 24, 32],
        "itemsize": 40,
    }
)


def ranked_summaries(query, search, *, radius, k_max, threads=1):
    """Per-query ranked summaries (query input order) and their aggregate, restated from the FRN rows.

    Semantics of the reference's exact summary kernel (``src/native/optix/rtdl_optix_core.cpp:5215-5296``:
    the k_max nearest by (distance, id), first and last of them, their distances added in rank order)
    and of its aggregate (``:5377-5431``: sums of the counts, of the first and last ids, of the distance
    sums).  The rows are the oracle's fixed_radius_neighbors rows, so rank order is (distance, id).  The
    per-query sum is a left-to-right sequential sum (``np.cumsum``); the aggregate's distance sum adds the
    per-query sums in query order.
    """
    rows, counts = fixed_radius_neighbors(query, search, radius=radius, k_max=k_max, threads=threads,
                                          with_counts=True)
    n = len(counts)
    qid = np.asarray(query["id"], dtype=np.uint32)
    kept = np.minimum(counts.astype(np.int64), int(k_max))
    order = np.argsort(qid, kind="stable")  # rows are grouped by query id, stable in input order
    starts = np.zeros(n + 1, dtype=np.int64)
    starts[1:] = np.cumsum(kept[order])
    out = np.zeros(n, dtype=SUMMARY_DTYPE)
    out["query_id"] = qid
    out["nearest_neighbor_id"] = 0xFFFFFFFF
    out["kth_neighbor_id"] = 0xFFFFFFFF
    for j, i in enumerate(order):
        a, b = starts[j], starts[j + 1]
        out[i]["neighbor_count"] = b - a
        if b > a:
            seg = rows[a:b]
            out[i]["nearest_neighbor_id"] = seg["neighbor_id"][0]
            out[i]["kth_neighbor_id"] = seg["neighbor_id"][-1]
            out[i]["nearest_distance"] = seg["distance"][0]
            out[i]["kth_distance"] = seg["distance"][-1]
            out[i]["sum_distance"] = np.cumsum(seg["distance"])[-1]
    agg = {
        "query_count": n,
        "bounded_neighbor_count": int(kept.sum()),
        "nearest_id_checksum": int(out["nearest_neighbor_id"].astype(np.uint64).sum()) % (1 << 64),
        "kth_id_checksum": int(out["kth_neighbor_id"].astype(np.uint64).sum()) % (1 << 64),
        "sum_distance": float(np.cumsum(out["sum_distance"])[-1]) if n else 0.0,
    }
    return out, agg


def knn_rows(query, search, *, k, threads=1, grid=False):
    """KNN rows (``reference.py:379-403``); ``grid`` as for fixed_radius_neighbors."""
    return _call_rows(query, search, 1, 0.0, k, True, threads, False, grid)


def nearest(query, search, *, threads=1, grid=False):
    """Per-query nearest (distance, neighbor_id) in query-input order (knn_rows with k=1)."""
    lib = _load()
    fn = lib.nn_oracle_nearest_grid if grid else lib.nn_oracle_nearest
    qid, qx, qy, qz = _columns(query)
    sid, sx, sy, sz = _columns(search)
    dist = np.zeros(len(qid), dtype=np.float64)
    nid = np.zeros(len(qid), dtype=np.uint32)
    status = fn(
        _ptr(qid, ctypes.c_uint32), _ptr(qx, ctypes.c_double), _ptr(qy, ctypes.c_double), _ptr(qz, ctypes.c_double), len(qid),
        _ptr(sid, ctypes.c_uint32), _ptr(sx, ctypes.c_double), _ptr(sy, ctypes.c_double), _ptr(sz, ctypes.c_double), len(sid),
        int(threads), _ptr(dist, ctypes.c_double), _ptr(nid, ctypes.c_uint32),
    )
    if status != 0:
        raise RuntimeError("nn_oracle_nearest failed")
    return dist, nid


def directed_hausdorff(query, search, *, threads=1):
    """Directed Hausdorff witness: max over queries of (distance, -query_id, -neighbor_id).

    Follows ``examples/v2_0/research_benchmarks/hausdorff_xhd/rtdl_hausdorff_distance_app.py:108-130``.
    """
    dist, nid = nearest(query, search, threads=threads)
    qid = np.asarray(query["id"], dtype=np.uint32)
    order = np.lexsort((nid.astype(np.int64), qid.astype(np.int64), -dist))
    best = order[0]
    return {"distance": float(dist[best]), "source_id": int(qid[best]), "target_id": int(nid[best]), "row_count": int(len(qid))}


# --- the reference's own native oracle (compiled from its sources into _ref/) ---------------

class _RefPoint3D(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint32), ("x", ctypes.c_double), ("y", ctypes.c_double), ("z", ctypes.c_double)]


class _RefPoint2D(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint32), ("x", ctypes.c_double), ("y", ctypes.c_double)]


def reference_library_available() -> bool:
    return REF_LIB_PATH.exists()


_ref_lib = None


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        lib = ctypes.CDLL(str(REF_LIB_PATH))
        for name in ("rtdl_oracle_run_fixed_radius_neighbors_3d", "rtdl_oracle_run_fixed_radius_neighbors"):
            fn = getattr(lib, name)
            fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double,
                           ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                           ctypes.c_char_p, ctypes.c_size_t]
            fn.restype = ctypes.c_int
        for name in ("rtdl_oracle_run_k_closest_hits_3d", "rtdl_oracle_run_k_closest_hits"):
            fn = getattr(lib, name)
            fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                           ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p, ctypes.c_size_t]
            fn.restype = ctypes.c_int
        lib.rtdl_oracle_free_rows.argtypes = [ctypes.c_void_p]
        lib.rtdl_oracle_free_rows.restype = None
        _ref_lib = lib
    return _ref_lib


def pack_reference_points(points):
    """numpy columns -> ctypes array of the reference's RtdlPoint / RtdlPoint3D."""
    ids, x, y, z = _columns(points)
    if z is None:
        arr = (_RefPoint2D * len(ids))()
        view = np.frombuffer(arr, dtype=np.dtype({"names": ["id", "x", "y"], "formats": ["<u4", "<f8", "<f8"], "offsets": [0, 8, 16], "itemsize": 24}))
        view["id"], view["x"], view["y"] = ids, x, y
    else:
        arr = (_RefPoint3D * len(ids))()
        view = np.frombuffer(arr, dtype=np.dtype({"names": ["id", "x", "y", "z"], "formats": ["<u4", "<f8", "<f8", "<f8"], "offsets": [0, 8, 16, 24], "itemsize": 32}))
        view["id"], view["x"], view["y"], view["z"] = ids, x, y, z
    return arr, len(ids), z is not None


def reference_fixed_radius_neighbors(packed_query, packed_search, *, radius, k_max):
    """One call of the reference's native ``rtdl_oracle_run_fixed_radius_neighbors[_3d]``
    (``src/native/oracle/rtdl_oracle_api.cpp:900-1023``).  Releases the GIL (ctypes)."""
    lib = _load_ref()
    qarr, nq, is3d = packed_query
    sarr, ns, _ = packed_search
    fn = lib.rtdl_oracle_run_fixed_radius_neighbors_3d if is3d else lib.rtdl_oracle_run_fixed_radius_neighbors
    rows = ctypes.c_void_p()
    count = ctypes.c_size_t()
    err = ctypes.create_string_buffer(4096)
    status = fn(ctypes.addressof(qarr), nq, ctypes.addressof(sarr), ns, float(radius), int(k_max),
                ctypes.byref(rows), ctypes.byref(count), err, len(err))
    if status != 0:
        raise RuntimeError(err.value.decode())
    try:
        n = count.value
        out = np.frombuffer((ctypes.c_char * (n * 16)).from_address(rows.value), dtype=FRN_ROW_DTYPE).copy() if n else np.zeros(0, FRN_ROW_DTYPE)
    finally:
        lib.rtdl_oracle_free_rows(rows)
    return out
