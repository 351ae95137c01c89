"""CPU-only checks of the C ABI library and the host-side mirror (no GPU work)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import rtdl_b200 as rt
from rtdl_b200 import _native

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "rtdl_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(rtdl_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_native.library_path()))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert sorted(_native.SIGNATURES) == declared_symbols()


def test_abi_struct_layouts_match_reference():
    assert ctypes.sizeof(_native.RtdlPoint) == 24
    assert ctypes.sizeof(_native.RtdlPoint3D) == 32
    assert _native.RtdlFixedRadiusNeighborRow.distance.offset == 8
    assert ctypes.sizeof(_native.RtdlFixedRadiusNeighborRow) == 16
    assert _native.RtdlKnnNeighborRow.neighbor_rank.offset == 16
    assert ctypes.sizeof(_native.RtdlKnnNeighborRow) == 24
    assert rt.runtime.POINT3D_DTYPE.itemsize == 32 and rt.runtime.POINT2D_DTYPE.itemsize == 24


def _call_frn3d(radius, k_max, nq=1, ns=1, null_out=False):
    lib = _native.load_library()
    q = (_native.RtdlPoint3D * max(nq, 1))()
    s = (_native.RtdlPoint3D * max(ns, 1))()
    rows = ctypes.c_void_p()
    count = ctypes.c_size_t(123)
    err = _native.error_buffer()
    status = lib.rtdl_b200_run_fixed_radius_neighbors_3d(
        q, nq, s, ns, radius, k_max, None if null_out else ctypes.byref(rows), ctypes.byref(count), err, len(err))
    return status, err.value.decode(), rows.value, count.value


def test_validation_messages_match_reference_before_any_gpu_work():
    # messages of rtdl_optix_api.cpp:4115-4127
    assert _call_frn3d(-1.0, 4)[:2] == (1, "fixed_radius_neighbors radius must be non-negative")
    assert _call_frn3d(1.0, 0)[:2] == (1, "fixed_radius_neighbors k_max must be positive")
    assert _call_frn3d(1.0, 2**32)[:2] == (1, "fixed_radius_neighbors k_max exceeds uint32 limit")
    assert _call_frn3d(1.0, 4, null_out=True)[:2] == (1, "output pointers must not be null")


def test_empty_inputs_return_zero_rows_without_gpu():
    status, msg, rows, count = _call_frn3d(1.0, 4, nq=0, ns=5)
    assert (status, rows, count) == (0, None, 0)
    status, msg, rows, count = _call_frn3d(1.0, 4, nq=3, ns=0)
    assert (status, rows, count) == (0, None, 0)


def test_knn_validation():
    lib = _native.load_library()
    q = (_native.RtdlPoint * 1)()
    rows = ctypes.c_void_p()
    count = ctypes.c_size_t()
    err = _native.error_buffer()
    assert lib.rtdl_b200_run_k_closest_hits(q, 1, q, 1, 0, ctypes.byref(rows), ctypes.byref(count), err, len(err)) == 1
    assert err.value.decode() == "knn_rows k must be positive"


def test_prepare_validation():
    lib = _native.load_library()
    h = ctypes.c_void_p()
    err = _native.error_buffer()
    assert lib.rtdl_b200_prepare_fixed_radius_neighbors_3d(None, 0, 0.0, ctypes.byref(h), err, len(err)) == 1
    assert err.value.decode() == "fixed_radius_neighbors_3d max_radius must be positive"


def test_batch_graph_validation_before_any_gpu_work():
    lib = _native.load_library()
    g = ctypes.c_void_p()
    err = _native.error_buffer()
    qoff = (ctypes.c_ulonglong * 2)(0, 0)
    radius = (ctypes.c_double * 1)(0.1)
    kmax = (ctypes.c_uint32 * 1)(8)
    assert lib.rtdl_b200_batch_graph_create(None, 1, None, qoff, radius, kmax, None, 0, None, err, len(err)) == 1
    assert err.value.decode() == "graph_out must not be null"
    assert lib.rtdl_b200_batch_graph_create(None, 1, None, qoff, radius, kmax, None, 0, ctypes.byref(g), err,
                                            len(err)) == 1
    assert err.value.decode() == "batches must not be null"
    batches = (ctypes.c_void_p * 1)(None)
    assert lib.rtdl_b200_batch_graph_create(batches, 0, None, qoff, radius, kmax, None, 0, ctypes.byref(g), err,
                                            len(err)) == 1
    assert err.value.decode() == "a batch graph needs at least one problem batch"
    assert lib.rtdl_b200_batch_graph_create(batches, 1, None, qoff, radius, kmax, None, 0, ctypes.byref(g), err,
                                            len(err)) == 1
    assert err.value.decode() == "batch graph inputs must be problem batch handles"
    assert g.value is None
    assert lib.rtdl_b200_batch_graph_replay(None, None, None, err, len(err)) == 1
    assert err.value.decode() == "graph must not be null"
    assert lib.rtdl_b200_batch_graph_launch(None, None, err, len(err)) == 1
    assert lib.rtdl_b200_batch_graph_info(None, None, None, None) == 1
    lib.rtdl_b200_batch_graph_destroy(None)  # no-op


def test_set_tuning_bounds():
    with pytest.raises(ValueError):
        rt.set_tuning(leaf_size=-1, block_threads=128)
    with pytest.raises(ValueError):
        rt.set_tuning(leaf_size=33, block_threads=128)
    with pytest.raises(ValueError):
        rt.set_tuning(leaf_size=8, block_threads=96)
    with pytest.raises(ValueError, match="traversal"):
        rt.set_tuning(traversal="packet_pairs")
    from rtdl_b200 import _native as nat
    assert nat.load_library().rtdl_b200_set_tuning(0, 128, 5) != 0  # traversal codes are 0..4
    for mode in ("packet", "lane", "packet_cube", "packet_points", "packet_hybrid"):
        rt.set_tuning(traversal=mode)
    rt.set_tuning(leaf_size=8, block_threads=128)
    rt.set_tuning()  # back to the defaults: leaf size by the scene's use


# ---- DSL mirror ---------------------------------------------------------------

def _frn_kernel(radius=0.5, k_max=3, geometry=None):
    geometry = geometry or rt.Points

    @rt.kernel(backend="rtdl", precision="float_approx")
    def k():
        q = rt.input("query_points", geometry, role="probe")
        s = rt.input("search_points", geometry, role="build")
        c = rt.traverse(q, s, accel="bvh")
        h = rt.refine(c, predicate=rt.fixed_radius_neighbors(radius=radius, k_max=k_max))
        return rt.emit(h, fields=["query_id", "neighbor_id", "distance"])

    return k


def test_dsl_compiles_like_reference():
    compiled = rt.compile_kernel(_frn_kernel())
    assert compiled.refine_op.predicate.name == "fixed_radius_neighbors"
    assert compiled.refine_op.predicate.options == {"radius": 0.5, "k_max": 3}
    assert compiled.candidates.left.name == "query_points"
    assert compiled.candidates.right.name == "search_points"
    assert compiled.emit_op.fields == ("query_id", "neighbor_id", "distance")


def test_predicate_validation_messages():
    with pytest.raises(ValueError, match="fixed_radius_neighbors radius must be non-negative"):
        rt.fixed_radius_neighbors(radius=-1.0, k_max=1)
    with pytest.raises(ValueError, match="fixed_radius_neighbors k_max must be positive"):
        rt.fixed_radius_neighbors(radius=1.0, k_max=0)
    with pytest.raises(ValueError, match="knn_rows k must be positive"):
        rt.knn_rows(k=0)
    with pytest.raises(ValueError, match="bounded_knn_rows k_max must be positive"):
        rt.bounded_knn_rows(radius=1.0, k_max=0)
    with pytest.raises(RuntimeError, match="must run inside"):
        rt.input("x", rt.Points)


def test_run_b200_input_validation():
    k = _frn_kernel()
    with pytest.raises(ValueError, match="missing RTDL b200 inputs: search_points"):
        rt.run_b200(k, query_points=())
    with pytest.raises(ValueError, match="unexpected RTDL b200 inputs: extra"):
        rt.run_b200(k, query_points=(), search_points=(), extra=())
    with pytest.raises(ValueError, match="result_mode"):
        rt.run_b200(k, query_points=(), search_points=(), result_mode="columns")


def test_execution_policy_has_no_fallback():
    with pytest.raises(ValueError):
        rt.ExecutionPolicy(backend="b200", allow_fallback=True)
    with pytest.raises(ValueError):
        rt.ExecutionPolicy(backend="optix")


def test_pack_points_columns_and_records_agree():
    recs = (rt.Point3D(id=3, x=1.0, y=2.0, z=3.0), rt.Point3D(id=9, x=-1.5, y=0.25, z=7.0))
    a = rt.pack_points(records=recs)
    b = rt.pack_points(ids=[3, 9], x=[1.0, -1.5], y=[2.0, 0.25], z=[3.0, 7.0])
    assert a.dimension == b.dimension == 3
    assert a.records.tobytes() == b.records.tobytes()
    c = (_native.RtdlPoint3D * 2)(_native.RtdlPoint3D(3, 1.0, 2.0, 3.0), _native.RtdlPoint3D(9, -1.5, 0.25, 7.0))
    assert bytes(c) == a.records.tobytes()
    m = rt.pack_points(records=[{"id": 1, "x": 0.5, "y": 0.25}])
    assert m.dimension == 2 and m.records["x"][0] == 0.5
    with pytest.raises(ValueError):
        rt.pack_points(records=recs, dimension=2)


def test_register_with_reference_dispatch(monkeypatch):
    import importlib
    import os
    import sys

    from oracle.oracle import reference_root

    ref = reference_root()
    if ref is None:
        pytest.skip("reference tree not present")
    monkeypatch.syspath_prepend(str(Path(ref) / "src"))
    rtdsl = importlib.import_module("rtdsl")
    from rtdl_b200 import execution as ex

    calls = []

    def fake_run_b200(kernel, *, result_mode="dict", **inputs):
        calls.append((kernel, result_mode, sorted(inputs)))
        return ({"query_id": 1, "neighbor_id": 2, "distance": 0.0},)

    monkeypatch.setattr(ex, "run_b200", fake_run_b200)
    ex.register_with_rtdsl(rtdsl)
    policy = rtdsl.ExecutionPolicy(backend="b200")
    k = _frn_kernel()
    result = rtdsl.run(k, {"query_points": (), "search_points": ()}, execution=policy)
    assert result.rows == ({"query_id": 1, "neighbor_id": 2, "distance": 0.0},)
    assert calls and calls[0][1] == "dict"
    assert result.execution_report.selected_backend == "b200"
    # other backends still route to the reference's own runners
    rows = rtdsl.run(k, {"query_points": (), "search_points": ()}, execution=rtdsl.ExecutionPolicy(backend="cpu_python_reference")).rows
    assert rows == ()
    sys.modules.pop("rtdsl", None)


def test_autotune_shape_classes_and_cache(tmp_path):
    from rtdl_b200.autotune import Autotuner, Config, shape_class

    assert shape_class(3, 1 << 20, 1 << 20, 31.0) == "d3-b20-q20-m5"
    assert shape_class(2, 1000, 0, 0.0) == "d2-b10-q0-m0"
    t = Autotuner(tmp_path / "c.json")
    t._store("d3-b20-q20-m5", Config(16, "lane", 256), {"16/lane/256": 1.0})
    assert Autotuner(tmp_path / "c.json").lookup("d3-b20-q20-m5") == Config(16, "lane", 256)
    assert t.lookup("missing") is None


def test_autotune_callable_picks_caches_and_applies_the_fastest(tmp_path, monkeypatch):
    """tune_callable's host logic without a GPU: CUDA events are replaced by a
    clock that charges each run the time the active candidate costs; the
    fastest candidate must win, be cached under the key (file included), be
    applied last, and a second call must come from the cache without runs."""
    import rtdl_b200.autotune as at

    applied = []
    monkeypatch.setattr(at.Config, "apply", lambda self: applied.append(self))
    cost = {c: 10.0 + i for i, c in enumerate(at.Autotuner().candidates)}
    fastest = at.Config(24, "packet", 256)
    cost[fastest] = 1.0

    class FakeEvent:
        clock = 0.0

        def __init__(self, enable_timing=False):
            self.t = None

        def record(self, stream=None):
            self.t = FakeEvent.clock

        def synchronize(self):
            pass

        def elapsed_time(self, end):
            return end.t - self.t

    runs = []

    def run():
        runs.append(applied[-1])
        FakeEvent.clock += cost[applied[-1]]

    import torch

    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    tuner = at.Autotuner(tmp_path / "t.json", repeats=2)
    key, cfg = tuner.tune_callable("problem batch 0 of 1", run, stream=object())
    assert (key, cfg) == ("problem batch 0 of 1", fastest)
    assert applied[-1] == fastest
    assert len(runs) == 3 * len(tuner.candidates)  # one warm-up run and two timed runs each
    assert tuner.cache[key]["ms"]["24/packet/256"] == 1.0
    assert at.Autotuner(tmp_path / "t.json").lookup(key) == fastest
    n_runs = len(runs)
    assert tuner.tune_callable(key, run, stream=object()) == (key, fastest)
    assert len(runs) == n_runs and applied[-1] == fastest
