"""Execution plans and the drop-in path, on the CPU.

* A kernel lowers to a B200ExecutionPlan that records the predicate, its
  options, the reference's role choice (build/probe) and the runners' binding
  (query = candidates.left, search = candidates.right), with
  ``accel_kind="lbvh"``.
* With the reference tree present, kernels compiled by the real ``rtdsl``
  (the reference's own example and goal311 kernels) and the reference's own
  ``RTExecutionPlan`` of them go through ``rtdsl.run(..., backend="b200")``.
  The native row call is replaced by the oracle restatement, so what is
  checked is everything on the host side of the C ABI: which inputs reach the
  ABI as query and search set, the predicate options, the packing, and the
  projection of rows into dicts -- against ``cpu_python_reference`` on the same
  kernel and inputs.
"""
from __future__ import annotations

import importlib
import importlib.util
import sys
from dataclasses import dataclass

import numpy as np
import pytest

import rtdl_b200 as rt
from oracle import oracle as O
from rtdl_b200 import runtime as R
from rtdl_b200.lowering import B200ExecutionPlan, lower_to_b200_plan


@rt.kernel(backend="rtdl", precision="float_approx")
def _frn3d():
    q = rt.input("query_points", rt.Points3D, role="probe")
    s = rt.input("search_points", rt.Points3D, role="build")
    return rt.emit(rt.refine(rt.traverse(q, s, accel="bvh"), predicate=rt.fixed_radius_neighbors(radius=0.25, k_max=5)),
                   fields=["query_id", "neighbor_id", "distance"])


@rt.kernel(backend="rtdl", precision="float_approx")
def _knn_swapped_roles():
    a = rt.input("a", rt.Points, role="build")
    b = rt.input("b", rt.Points, role="probe")
    return rt.emit(rt.refine(rt.traverse(a, b, accel="bvh"), predicate=rt.knn_rows(k=3)),
                   fields=["query_id", "neighbor_id", "distance", "neighbor_rank"])


def test_plan_of_mirror_kernel():
    plan = lower_to_b200_plan(_frn3d)
    assert isinstance(plan, B200ExecutionPlan)
    assert plan.accel_kind == "lbvh" and plan.backend == "b200"
    assert plan.predicate == plan.workload_kind == "fixed_radius_neighbors"
    assert plan.predicate_options == {"radius": 0.25, "k_max": 5}
    assert (plan.query_input, plan.search_input) == ("query_points", "search_points")
    assert (plan.probe_input.name, plan.build_input.name) == ("query_points", "search_points")
    assert plan.dimension == 3 and plan.entry_point == "rtdl_b200_run_fixed_radius_neighbors_3d"
    assert plan.output_record[0] == "RtdlFixedRadiusNeighborRow"
    d = plan.to_dict()
    assert d["accel_kind"] == "lbvh" and d["launch_params"][0][0] == "query_points"


def test_plan_keeps_runner_binding_when_roles_are_swapped():
    plan = lower_to_b200_plan(_knn_swapped_roles)
    # the reference's role rule makes `a` the build side ...
    assert plan.build_input.name == "a" and plan.probe_input.name == "b"
    # ... but its runners answer candidates.left as the query set
    assert (plan.query_input, plan.search_input) == ("a", "b")
    assert plan.entry_point == "rtdl_b200_run_k_closest_hits"


def test_lowering_rejects_what_the_reference_rejects():
    @rt.kernel(backend="rtdl", precision="float_approx")
    def not_bvh():
        q = rt.input("q", rt.Points)
        s = rt.input("s", rt.Points)
        return rt.emit(rt.refine(rt.traverse(q, s, accel="grid"), predicate=rt.knn_rows(k=1)),
                       fields=["query_id", "neighbor_id"])

    with pytest.raises(ValueError, match="accel='bvh'"):
        lower_to_b200_plan(not_bvh)


# ---- the host side of the ABI, with the oracle standing in for the library ----

@dataclass
class _OracleView:
    rows: np.ndarray
    field_names: tuple

    def to_dict_rows(self, fields=None):
        names = tuple(fields or self.field_names)
        return tuple({n: self.rows[n][i].item() for n in names} for i in range(len(self.rows)))

    def close(self):
        pass


@pytest.fixture
def abi_calls(monkeypatch):
    """Replaces the two native row calls by the oracle and records what reached them."""
    calls = []

    def frn(query, search, *, radius, k_max, dimension=None, ranked=False):
        calls.append(("fixed_radius_neighbors", query.records["id"].tolist(), search.records["id"].tolist(),
                      {"radius": radius, "k_max": k_max, "ranked": ranked}))
        rows = O.fixed_radius_neighbors(query.records, search.records, radius=radius, k_max=k_max, ranked=ranked)
        names = ("query_id", "neighbor_id", "distance") + (("neighbor_rank",) if ranked else ())
        return _OracleView(rows, names)

    def knn(query, search, *, k, dimension=None):
        calls.append(("knn_rows", query.records["id"].tolist(), search.records["id"].tolist(), {"k": k}))
        rows = O.knn_rows(query.records, search.records, k=k)
        return _OracleView(rows, ("query_id", "neighbor_id", "distance", "neighbor_rank"))

    monkeypatch.setattr(R, "fixed_radius_neighbors", frn)
    monkeypatch.setattr(R, "knn_rows", knn)
    return calls


@pytest.fixture
def rtdsl(monkeypatch):
    ref = O.reference_root()
    if ref is None:
        pytest.skip("reference tree not present")
    monkeypatch.syspath_prepend(str(ref))
    monkeypatch.syspath_prepend(str(ref / "src"))
    saved = {k: v for k, v in sys.modules.items() if k == "rtdsl" or k.startswith("rtdsl.")}
    mod = importlib.import_module("rtdsl")
    from rtdl_b200.execution import register_with_rtdsl

    register_with_rtdsl(mod)
    yield mod, ref
    for k in [k for k in sys.modules if k == "rtdsl" or k.startswith("rtdsl.")]:
        del sys.modules[k]
    sys.modules.update(saved)


def _reference_example(ref, relpath, name):
    spec = importlib.util.spec_from_file_location(f"_ref_example_{name}", ref / relpath)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _goal311_kernels(rt_ref):
    # the kernels of the reference's tests/goal311_v0_5_optix_3d_nn_test.py:12-35, written with the real rtdsl
    @rt_ref.kernel(backend="rtdl", precision="float_approx")
    def fixed_radius_neighbors_3d():
        query_points = rt_ref.input("query_points", rt_ref.Points3D, role="probe")
        search_points = rt_ref.input("search_points", rt_ref.Points3D, role="build")
        candidates = rt_ref.traverse(query_points, search_points, accel="bvh")
        hits = rt_ref.refine(candidates, predicate=rt_ref.fixed_radius_neighbors(radius=1.0, k_max=2))
        return rt_ref.emit(hits, fields=["query_id", "neighbor_id", "distance"])

    @rt_ref.kernel(backend="rtdl", precision="float_approx")
    def bounded_knn_rows_3d():
        query_points = rt_ref.input("query_points", rt_ref.Points3D, role="probe")
        search_points = rt_ref.input("search_points", rt_ref.Points3D, role="build")
        candidates = rt_ref.traverse(query_points, search_points, accel="bvh")
        hits = rt_ref.refine(candidates, predicate=rt_ref.bounded_knn_rows(radius=1.0, k_max=2))
        return rt_ref.emit(hits, fields=["query_id", "neighbor_id", "distance", "neighbor_rank"])

    @rt_ref.kernel(backend="rtdl", precision="float_approx")
    def knn_rows_3d():
        query_points = rt_ref.input("query_points", rt_ref.Points3D, role="probe")
        search_points = rt_ref.input("search_points", rt_ref.Points3D, role="build")
        candidates = rt_ref.traverse(query_points, search_points, accel="bvh")
        hits = rt_ref.refine(candidates, predicate=rt_ref.knn_rows(k=2))
        return rt_ref.emit(hits, fields=["query_id", "neighbor_id", "distance", "neighbor_rank"])

    case = {
        "query_points": (rt_ref.Point3D(id=10, x=0.0, y=0.0, z=0.0), rt_ref.Point3D(id=20, x=5.0, y=0.0, z=0.0)),
        "search_points": (rt_ref.Point3D(id=1, x=0.0, y=0.0, z=0.0), rt_ref.Point3D(id=2, x=0.0, y=0.0, z=0.6),
                          rt_ref.Point3D(id=3, x=0.0, y=0.8, z=0.0), rt_ref.Point3D(id=4, x=5.0, y=0.0, z=0.9)),
    }
    return (fixed_radius_neighbors_3d, bounded_knn_rows_3d, knn_rows_3d), case


def _assert_same_rows(got, exp):
    assert len(got) == len(exp)
    for g, e in zip(got, exp):
        assert g == e


def test_reference_compiled_kernels_through_rtdsl_run(rtdsl, abi_calls):
    rt_ref, ref = rtdsl
    kernels, case = _goal311_kernels(rt_ref)
    frn_ex = _reference_example(ref, "examples/reference/rtdl_fixed_radius_neighbors_reference.py", "frn")
    knn_ex = _reference_example(ref, "examples/reference/rtdl_knn_rows_reference.py", "knn")
    runs = [(k, case) for k in kernels]
    runs.append((frn_ex.fixed_radius_neighbors_reference, frn_ex.make_fixed_radius_neighbors_authored_case()))
    runs.append((knn_ex.knn_rows_reference, knn_ex.make_knn_rows_authored_case()))
    b200 = rt_ref.ExecutionPolicy(backend="b200")
    cpu = rt_ref.ExecutionPolicy(backend="cpu_python_reference")
    for kernel, inputs in runs:
        compiled = rt_ref.compile_kernel(kernel) if not hasattr(kernel, "refine_op") else kernel
        pred = compiled.refine_op.predicate
        abi_calls.clear()
        got = rt_ref.run(kernel, inputs, execution=b200)
        assert got.execution_report.selected_backend == "b200"
        exp = rt_ref.run(kernel, inputs, execution=cpu).rows
        _assert_same_rows(got.rows, exp)
        # what reached the ABI: the left input as queries, the right as search points, the kernel's options
        (name, qids, sids, opts), = abi_calls
        assert name == ("knn_rows" if pred.name == "knn_rows" else "fixed_radius_neighbors")
        assert qids == [p.id for p in inputs[compiled.candidates.left.name]]
        assert sids == [p.id for p in inputs[compiled.candidates.right.name]]
        if pred.name == "knn_rows":
            assert opts == {"k": pred.options["k"]}
        else:
            assert opts == {"radius": pred.options["radius"], "k_max": pred.options["k_max"],
                            "ranked": pred.name == "bounded_knn_rows"}


def test_reference_plan_lowers_and_runs(rtdsl, abi_calls):
    rt_ref, _ref = rtdsl
    kernels, case = _goal311_kernels(rt_ref)
    for kernel in kernels:
        compiled = rt_ref.compile_kernel(kernel)
        ref_plan = rt_ref.lower_to_execution_plan(compiled)
        from_kernel = lower_to_b200_plan(compiled)
        from_plan = lower_to_b200_plan(ref_plan)  # options read from the plan itself
        with_kernel = lower_to_b200_plan(ref_plan, compiled=compiled)
        for p in (from_kernel, from_plan, with_kernel):
            assert p.accel_kind == "lbvh"
            assert p.predicate == ref_plan.predicate == compiled.refine_op.predicate.name
            assert p.predicate_options == from_kernel.predicate_options
            assert (p.query_input, p.search_input) == ("query_points", "search_points")
            assert p.build_input.name == ref_plan.build_input.name
            assert p.probe_input.name == ref_plan.probe_input.name
            assert tuple(p.emit_fields) == tuple(ref_plan.emit_fields)
        assert from_plan.source_plan is ref_plan
        exp = rt_ref.run(kernel, case, execution=rt_ref.ExecutionPolicy(backend="cpu_python_reference")).rows
        _assert_same_rows(rt.run_b200(ref_plan, **case), exp)
        _assert_same_rows(rt.run_b200(from_kernel, **case), exp)


def test_swapped_roles_answer_like_the_reference_runner(rtdsl, abi_calls):
    """Explicit roles that put the build side on the left change the plan's
    build/probe choice but not the rows: the reference's runner still answers
    the left input as queries, and so does this backend."""
    rt_ref, _ref = rtdsl

    @rt_ref.kernel(backend="rtdl", precision="float_approx")
    def swapped():
        a = rt_ref.input("a", rt_ref.Points, role="build")
        b = rt_ref.input("b", rt_ref.Points, role="probe")
        return rt_ref.emit(rt_ref.refine(rt_ref.traverse(a, b, accel="bvh"),
                                         predicate=rt_ref.fixed_radius_neighbors(radius=0.3, k_max=4)),
                           fields=["query_id", "neighbor_id", "distance"])

    rng = np.random.default_rng(5)
    a = tuple(rt_ref.Point(id=int(i), x=float(x), y=float(y)) for i, (x, y) in enumerate(rng.random((20, 2))))
    b = tuple(rt_ref.Point(id=100 + int(i), x=float(x), y=float(y)) for i, (x, y) in enumerate(rng.random((30, 2))))
    got = rt_ref.run(swapped, {"a": a, "b": b}, execution=rt_ref.ExecutionPolicy(backend="b200")).rows
    exp = rt_ref.run(swapped, {"a": a, "b": b}, execution=rt_ref.ExecutionPolicy(backend="cpu_python_reference")).rows
    assert len(exp) > 0
    _assert_same_rows(got, exp)
    plan = lower_to_b200_plan(rt_ref.compile_kernel(swapped))
    assert plan.build_input.name == "a" and plan.query_input == "a"
