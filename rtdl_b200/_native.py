"""ctypes binding of librtdl_b200.so (the C ABI in include/rtdl_b200.h).

The binding mirrors how RTDL binds its OptiX library
(rubaolee/rtdl src/rtdsl/optix_runtime.py:15957-16010 loader,
:17508-17540 argtypes, :18524-18540 status check): one process-wide handle,
explicit argtypes, a 4,096-byte error buffer per call and ``RuntimeError`` on
a non-zero status.  There is no fallback: if the library is missing or fails
to load, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

PKG = Path(__file__).resolve().parent
DEFAULT_LIB = PKG / "librtdl_b200.so"

_lock = threading.Lock()
_lib = None


class RtdlPoint(ctypes.Structure):
    """``RtdlPoint`` {u32 id; f64 x, y} -- rtdl_optix_prelude.h:103-106 (24 B)."""

    _fields_ = [("id", ctypes.c_uint32), ("x", ctypes.c_double), ("y", ctypes.c_double)]


class RtdlPoint3D(ctypes.Structure):
    """``RtdlPoint3D`` {u32 id; f64 x, y, z} -- rtdl_optix_prelude.h:138-141 (32 B)."""

    _fields_ = [("id", ctypes.c_uint32), ("x", ctypes.c_double), ("y", ctypes.c_double), ("z", ctypes.c_double)]


class RtdlFixedRadiusNeighborRow(ctypes.Structure):
    """``RtdlFixedRadiusNeighborRow`` {u32, u32, f64} -- rtdl_optix_prelude.h:254-260 (16 B)."""

    _fields_ = [("query_id", ctypes.c_uint32), ("neighbor_id", ctypes.c_uint32), ("distance", ctypes.c_double)]


class RtdlKnnNeighborRow(ctypes.Structure):
    """``RtdlKnnNeighborRow`` {u32, u32, f64, u32} -- rtdl_optix_prelude.h:289-295 (24 B)."""

    _fields_ = [
        ("query_id", ctypes.c_uint32),
        ("neighbor_id", ctypes.c_uint32),
        ("distance", ctypes.c_double),
        ("neighbor_rank", ctypes.c_uint32),
    ]


class RtdlB200Witness(ctypes.Structure):
    """Result record of rtdl_b200_scene_directed_hausdorff_noalloc (24 B)."""

    _fields_ = [
        ("distance", ctypes.c_double),
        ("source_id", ctypes.c_uint32),
        ("target_id", ctypes.c_uint32),
        ("status", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class RtdlFixedRadiusRankedNeighborSummary(ctypes.Structure):
    """Per-query ranked summary -- rtdl_optix_prelude.h:300-316 (40 B)."""

    _fields_ = [
        ("query_id", ctypes.c_uint32),
        ("neighbor_count", ctypes.c_uint32),
        ("nearest_neighbor_id", ctypes.c_uint32),
        ("kth_neighbor_id", ctypes.c_uint32),
        ("nearest_distance", ctypes.c_double),
        ("kth_distance", ctypes.c_double),
        ("sum_distance", ctypes.c_double),
    ]


class RtdlFixedRadiusRankedNeighborAggregate(ctypes.Structure):
    """Aggregate of the summaries -- rtdl_optix_prelude.h:318-329 (40 B)."""

    _fields_ = [
        ("query_count", ctypes.c_size_t),
        ("bounded_neighbor_count", ctypes.c_size_t),
        ("nearest_id_checksum", ctypes.c_uint64),
        ("kth_id_checksum", ctypes.c_uint64),
        ("sum_distance", ctypes.c_double),
    ]


assert ctypes.sizeof(RtdlFixedRadiusRankedNeighborSummary) == 40
assert ctypes.sizeof(RtdlFixedRadiusRankedNeighborAggregate) == 40
assert ctypes.sizeof(RtdlPoint) == 24 and ctypes.sizeof(RtdlPoint3D) == 32
assert ctypes.sizeof(RtdlFixedRadiusNeighborRow) == 16 and ctypes.sizeof(RtdlKnnNeighborRow) == 24

# Every symbol the header declares, with (restype, argtypes).
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_cp = ctypes.c_char_p
_d = ctypes.c_double
_i = ctypes.c_int
_u32p = ctypes.POINTER(ctypes.c_uint32)
_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vpp = ctypes.POINTER(ctypes.c_void_p)
_szp = ctypes.POINTER(ctypes.c_size_t)

SIGNATURES = {
    "rtdl_b200_get_version": (_i, [ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "rtdl_b200_set_device": (_i, [_i]),
    "rtdl_b200_run_fixed_radius_neighbors": (_i, [_vp, _sz, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_run_fixed_radius_neighbors_device": (_i, [_vp, _sz, _vp, _sz, _i, _d, _sz, _vp, _sz, _szp, _vp, _vp,
                                                         _cp, _sz]),
    "rtdl_b200_run_fixed_radius_neighbors_3d": (_i, [_vp, _sz, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_run_bounded_knn_rows": (_i, [_vp, _sz, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_run_bounded_knn_rows_3d": (_i, [_vp, _sz, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_run_k_closest_hits": (_i, [_vp, _sz, _vp, _sz, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_run_k_closest_hits_3d": (_i, [_vp, _sz, _vp, _sz, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_free_rows": (None, [_vp]),
    "rtdl_b200_prepare_fixed_radius_neighbors_3d": (_i, [_vp, _sz, _d, _vpp, _cp, _sz]),
    "rtdl_b200_run_prepared_fixed_radius_neighbors_3d": (_i, [_vp, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_destroy_prepared_fixed_radius_neighbors_3d": (None, [_vp]),
    "rtdl_b200_scene_create": (_i, [_vp, _sz, _i, _i, _vp, _vpp, _cp, _sz]),
    "rtdl_b200_scene_destroy": (None, [_vp]),
    "rtdl_b200_scene_query": (_i, [_vp, _vp, _sz, _i, _d, _sz, _vpp, _szp, _u8p, _cp, _sz]),
    "rtdl_b200_scene_query_device": (_i, [_vp, _vp, _sz, _i, _d, _sz, _vp, _sz, _szp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_scene_directed_hausdorff": (_i, [_vp, _vp, _sz, _dp, _u32p, _u32p, _dp, _u32p, _cp, _sz]),
    "rtdl_b200_scene_directed_hausdorff_device": (_i, [_vp, _vp, _sz, _vp, _vp, _dp, _u32p, _u32p, _vp, _cp, _sz]),
    "rtdl_b200_scene_directed_hausdorff_noalloc": (_i, [_vp, _vp, _sz, _vp, _vp, _vp, _vp, _cp, _sz]),
    # batch arrays (offsets, radius, k_max, row offsets) are passed as addresses of numpy buffers
    "rtdl_b200_batch_create": (_i, [_vp, _vp, ctypes.c_uint32, _i, _i, _vp, _vpp, _cp, _sz]),
    "rtdl_b200_batch_destroy": (None, [_vp]),
    "rtdl_b200_batch_graph_create": (_i, [_vp, ctypes.c_uint32, _vp, _vp, _vp, _vp, _vp, _sz, _vpp, _cp, _sz]),
    "rtdl_b200_batch_graph_replay": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32), _cp, _sz]),
    "rtdl_b200_batch_graph_launch": (_i, [_vp, _vp, _cp, _sz]),
    "rtdl_b200_batch_graph_info": (_i, [_vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(_i),
                                        ctypes.POINTER(ctypes.c_ulonglong)]),
    "rtdl_b200_batch_graph_destroy": (None, [_vp]),
    "rtdl_b200_batch_fixed_radius_neighbors": (_i, [_vp, _vp, _vp, _vp, _vp, _vpp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_batch_fixed_radius_neighbors_device": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp,
                                                           _cp, _sz]),
    "rtdl_b200_scene_fixed_radius_neighbors_multi_device": (_i, [_vp, _vp, _vp, ctypes.c_uint32, _vp, _vp, _vp, _sz,
                                                                  _vp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_run_prepared_ranked_fixed_radius_neighbor_summaries_3d": (_i, [_vp, _vp, _sz, _d, _sz, _vpp, _szp,
                                                                               _cp, _sz]),
    "rtdl_b200_aggregate_prepared_ranked_fixed_radius_neighbor_summaries_3d": (_i, [_vp, _vp, _sz, _d, _sz, _vp, _cp,
                                                                                     _sz]),
    "rtdl_b200_scene_ranked_summaries_device": (_i, [_vp, _vp, _sz, _d, _sz, _vp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_queries_create": (_i, [_vp, _sz, _i, _i, _vp, _vpp, _cp, _sz]),
    "rtdl_b200_queries_destroy": (None, [_vp]),
    "rtdl_b200_prepare_fixed_radius_query_points_3d": (_i, [_vp, _sz, _vpp, _cp, _sz]),
    "rtdl_b200_destroy_prepared_fixed_radius_query_points_3d": (None, [_vp]),
    "rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d": (_i, [_vp, _vp, _d, _sz, _vp,
                                                                                           _cp, _sz]),
    "rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d_f32": (_i, [_vp, _vp, _d, _sz, _vp,
                                                                                               _cp, _sz]),
    "rtdl_b200_scene_ranked_summaries_prepared_device": (_i, [_vp, _vp, _d, _sz, _vp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_scene_query_prepared_device": (_i, [_vp, _vp, _d, _sz, _vp, _sz, _szp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_prepare_fixed_radius_ranked_summary_aggregate_batch_graph_3d": (
        _i, [_vp, _vp, _dp, ctypes.POINTER(_sz), _sz, _vpp, _cp, _sz]),
    "rtdl_b200_replay_fixed_radius_ranked_summary_aggregate_batch_graph_3d": (_i, [_vp, _vp, _cp, _sz]),
    "rtdl_b200_launch_fixed_radius_ranked_summary_aggregate_batch_graph_device_partials_3d": (
        _i, [_vp, ctypes.POINTER(ctypes.c_uint64), _szp, _szp, _szp, ctypes.POINTER(ctypes.c_uint64), _cp, _sz]),
    "rtdl_b200_fixed_radius_ranked_summary_aggregate_batch_graph_status_device_3d": (
        _i, [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), _cp, _sz]),
    "rtdl_b200_update_fixed_radius_ranked_summary_aggregate_batch_graph_3d": (
        _i, [_vp, _dp, ctypes.POINTER(_sz), _sz, _cp, _sz]),
    "rtdl_b200_destroy_fixed_radius_ranked_summary_aggregate_batch_graph_3d": (None, [_vp]),
    "rtdl_b200_run_fixed_radius_count_threshold": (_i, [_vp, _sz, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_prepare_fixed_radius_count_threshold_2d": (_i, [_vp, _sz, _d, _vpp, _cp, _sz]),
    "rtdl_b200_prepare_fixed_radius_count_threshold_2d_device_search_columns": (
        _i, [_vp, _vp, _vp, _sz, _d, _vpp, _cp, _sz]),
    "rtdl_b200_run_prepared_fixed_radius_count_threshold_2d": (_i, [_vp, _vp, _sz, _d, _sz, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_write_prepared_fixed_radius_count_threshold_2d_device_query_columns": (
        _i, [_vp, _vp, _vp, _vp, _sz, _d, _sz, _vp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_count_prepared_fixed_radius_threshold_reached_2d": (_i, [_vp, _vp, _sz, _d, _sz, _szp, _cp, _sz]),
    "rtdl_b200_run_prepared_fixed_radius_nearest_witness_2d": (_i, [_vp, _vp, _sz, _d, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_destroy_prepared_fixed_radius_count_threshold_2d": (None, [_vp]),
    "rtdl_b200_prepare_fixed_radius_count_threshold_3d": (_i, [_vp, _sz, _d, _vpp, _cp, _sz]),
    "rtdl_b200_write_prepared_fixed_radius_count_threshold_3d_device_outputs": (
        _i, [_vp, _vp, _sz, _d, _sz, _vp, _vp, _vp, _cp, _sz]),
    "rtdl_b200_destroy_prepared_fixed_radius_count_threshold_3d": (None, [_vp]),
    "rtdl_b200_prepare_point_group_nearest_witness_2d": (_i, [_vp, _sz, _vp, _sz, _d, _vpp, _cp, _sz]),
    "rtdl_b200_count_prepared_point_group_threshold_reached_2d": (_i, [_vp, _vp, _sz, _d, _sz, _szp, _cp, _sz]),
    "rtdl_b200_write_prepared_point_group_threshold_flags_2d": (_i, [_vp, _vp, _sz, _d, _sz, _vp, _cp, _sz]),
    "rtdl_b200_run_prepared_point_group_nearest_witness_2d": (_i, [_vp, _vp, _sz, _d, _vpp, _szp, _cp, _sz]),
    "rtdl_b200_reduce_prepared_point_group_nearest_max_distance_2d": (_i, [_vp, _vp, _sz, _d, _vp, _cp, _sz]),
    "rtdl_b200_destroy_prepared_point_group_nearest_witness_2d": (None, [_vp]),
    "rtdl_b200_get_last_phase_timings": (_i, [ctypes.POINTER(ctypes.c_char_p), _dp, _i]),
    "rtdl_b200_set_tuning": (_i, [_i, _i, _i]),
    "rtdl_b200_get_launch_count": (_i, [ctypes.POINTER(ctypes.c_ulonglong)]),
    "rtdl_b200_get_last_query_stats": (_i, [ctypes.POINTER(ctypes.c_ulonglong), _i]),
}


def library_path() -> Path:
    env = os.environ.get("RTDL_B200_LIB")
    return Path(env) if env else DEFAULT_LIB


def load_library(build_if_missing: bool = True):
    """Load librtdl_b200.so once per process (building it in-tree if it is missing)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not path.exists() and build_if_missing and "RTDL_B200_LIB" not in os.environ:
            from . import build as _build

            _build.build()
        if not path.exists():
            raise RuntimeError(f"librtdl_b200.so not found at {path}; run `python -m rtdl_b200.build`")
        lib = ctypes.CDLL(str(path))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def check_status(status: int, error) -> None:
    """Raise like the reference's ``_check_status`` (optix_runtime.py:18524-18540)."""
    if status == 0:
        return
    msg = error.value.decode("utf-8", errors="replace").strip() if error is not None else ""
    raise RuntimeError(msg or f"b200 backend call failed with status {status}")


def error_buffer():
    return ctypes.create_string_buffer(4096)


def launch_count() -> int:
    """Kernels launched by librtdl_b200 in this process so far."""
    v = ctypes.c_ulonglong()
    load_library().rtdl_b200_get_launch_count(ctypes.byref(v))
    return int(v.value)


STAT_NAMES = ("nodes", "leaf_points", "in_radius", "inserts", "shifts", "band_checks", "max_count",
              "generic_queries", "large_queries", "leaf_pairs", "emit_fixups", "refined_queries")


def last_query_stats() -> dict[str, int]:
    """Traversal counters of this thread's last query (RTDL_B200_STATS must be set)."""
    vals = (ctypes.c_ulonglong * 16)()
    n = load_library().rtdl_b200_get_last_query_stats(vals, 16)
    return {STAT_NAMES[i]: int(vals[i]) for i in range(min(n, len(STAT_NAMES)))}


def last_phase_timings() -> dict[str, float]:
    """Phase timings (ms, CUDA events) of this thread's last call."""
    lib = load_library()
    names = (ctypes.c_char_p * 32)()
    vals = (ctypes.c_double * 32)()
    n = lib.rtdl_b200_get_last_phase_timings(names, vals, 32)
    return {names[i].decode(): float(vals[i]) for i in range(min(n, 32))}
