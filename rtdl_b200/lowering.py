"""Execution plans of the neighbor predicates for the b200 backend.

RTDL lowers a ``CompiledKernel`` to an ``RTExecutionPlan``
(rubaolee/rtdl ``src/rtdsl/lowering.py:41-90``; the three neighbor lowerings
at ``:435-626``; the plan type at ``src/rtdsl/ir.py:132-180``).  This module
gives the b200 backend the same step:

* :func:`lower_to_b200_plan` takes an ``@rt.kernel`` function, a compiled
  kernel (the reference's or this package's mirror), or a plan the reference
  lowered, and returns a :class:`B200ExecutionPlan`: the reference plan's
  fields with this backend's values (``accel_kind="lbvh"``, the C entry point
  and its arguments, the CUDA kernels that run) plus the predicate's options.
* :func:`run_b200` (in ``runtime.py``) executes every kernel through such a
  plan, so the predicate, its options and the query/search binding that reach
  the C ABI are the plan's.

Validation follows the reference lowering (same checks, same messages):
backend ``rtdl``/``rayjoin``, a complete kernel, ``accel="bvh"``,
``precision="float_approx"``, point inputs on both sides.

Roles.  ``build_input`` / ``probe_input`` are chosen by the reference's rule
(``lowering.py:976-1007``).  The rows, however, are defined by the reference's
runners, which always answer ``candidates.left`` as the query set and
``candidates.right`` as the search set, whatever the roles say
(``src/rtdsl/runtime.py:223-242``, ``optix_runtime.py:15800-15801``).  The plan
therefore records the runners' binding in ``query_input`` / ``search_input``,
and that binding is what executes; the two agree whenever the kernel's roles
are unset or say probe = left, build = right.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import Any

NEIGHBOR_PREDICATES = ("fixed_radius_neighbors", "knn_rows", "bounded_knn_rows")

# emitted field -> C type, as in the reference lowering's table (lowering.py:12-38)
_EMIT_FIELD_TYPES = {"query_id": "uint32_t", "neighbor_id": "uint32_t", "distance": "double",
                     "neighbor_rank": "uint32_t"}
_RECORD_NAMES = {"fixed_radius_neighbors": "RtdlFixedRadiusNeighborRow", "knn_rows": "RtdlKnnNeighborRow",
                 "bounded_knn_rows": "RtdlKnnNeighborRow"}
_ENTRY_POINTS = {
    ("fixed_radius_neighbors", 2): "rtdl_b200_run_fixed_radius_neighbors",
    ("fixed_radius_neighbors", 3): "rtdl_b200_run_fixed_radius_neighbors_3d",
    ("bounded_knn_rows", 2): "rtdl_b200_run_bounded_knn_rows",
    ("bounded_knn_rows", 3): "rtdl_b200_run_bounded_knn_rows_3d",
    ("knn_rows", 2): "rtdl_b200_run_k_closest_hits",
    ("knn_rows", 3): "rtdl_b200_run_k_closest_hits_3d",
}
_EXACT_MODE = "fp32_traversal_fp64_band_recheck"


@dataclass(frozen=True)
class B200ExecutionPlan:
    """The reference ``RTExecutionPlan``'s fields, with this backend's values,
    plus the predicate options and the runners' query/search binding."""

    kernel_name: str
    workload_kind: str
    backend: str
    precision: str
    build_input: Any
    probe_input: Any
    accel_kind: str
    predicate: str
    exact_refine_mode: str
    emit_fields: tuple[str, ...]
    launch_params: tuple[tuple[str, str, str], ...]  # (name, C type, role) of the entry point's arguments
    host_steps: tuple[str, ...]
    device_programs: tuple[str, ...]
    output_record: tuple[str, tuple[tuple[str, str], ...]]  # record name, (field, C type) pairs
    bvh_policy: str
    predicate_options: dict = field(default_factory=dict)
    query_input: str = ""
    search_input: str = ""
    dimension: int = 2
    entry_point: str = ""
    input_names: tuple[str, ...] = ()
    source_plan: Any = None  # the reference's RTExecutionPlan when lowered from one

    def to_dict(self) -> dict[str, object]:
        def geometry(g):
            return {"name": g.name, "geometry": g.geometry.name, "layout": g.layout.name, "role": g.role}

        return {
            "kernel_name": self.kernel_name,
            "workload_kind": self.workload_kind,
            "backend": self.backend,
            "precision": self.precision,
            "build_input": geometry(self.build_input),
            "probe_input": geometry(self.probe_input),
            "accel_kind": self.accel_kind,
            "predicate": self.predicate,
            "predicate_options": dict(self.predicate_options),
            "exact_refine_mode": self.exact_refine_mode,
            "emit_fields": list(self.emit_fields),
            "query_input": self.query_input,
            "search_input": self.search_input,
            "dimension": self.dimension,
            "entry_point": self.entry_point,
            "launch_params": [list(p) for p in self.launch_params],
            "host_steps": list(self.host_steps),
            "device_programs": list(self.device_programs),
            "output_record": {"name": self.output_record[0], "fields": [list(f) for f in self.output_record[1]]},
            "bvh_policy": self.bvh_policy,
        }


def _is_plan(obj) -> bool:
    return hasattr(obj, "workload_kind") and hasattr(obj, "build_input") and hasattr(obj, "probe_input")


def _resolve_compiled(kernel_fn_or_compiled):
    if hasattr(kernel_fn_or_compiled, "refine_op") and hasattr(kernel_fn_or_compiled, "inputs"):
        return kernel_fn_or_compiled
    if callable(kernel_fn_or_compiled):
        return kernel_fn_or_compiled()
    raise TypeError("expected an @rt.kernel function, a CompiledKernel or an execution plan")


def choose_roles(candidates):
    """(build, probe) by the reference's rule for two point inputs (lowering.py:976-1007)."""
    left, right = candidates.left, candidates.right
    if left.role is not None and left.role == right.role:
        raise ValueError("candidate inputs cannot share the same explicit role")
    if left.role == "build" and right.role == "probe":
        return left, right
    if left.role == "probe" and right.role == "build":
        return right, left
    if left.role == "build":
        return left, right
    if right.role == "build":
        return right, left
    if left.role == "probe":
        return right, left
    if right.role == "probe":
        return left, right
    return right, left


def _dimension(geometry_input) -> int:
    layout = geometry_input.layout
    names = set(layout.field_names())
    return 3 if layout.name.endswith("3D") or "z" in names else 2


def _validate(compiled) -> None:
    # the reference lowering's checks and messages (lowering.py:41-62, 435-437, 500-502, 564-566)
    if compiled.backend not in {"rtdl", "rayjoin"}:
        raise ValueError(f"unsupported backend for RTDL lowering: {compiled.backend}")
    if compiled.candidates is None or compiled.refine_op is None or compiled.emit_op is None:
        raise ValueError("kernel is incomplete and cannot be lowered")
    if compiled.candidates.accel != "bvh":
        raise ValueError("the current RTDL lowering supports only accel='bvh' "
                         f"(got accel={compiled.candidates.accel!r})")
    if compiled.precision != "float_approx":
        raise ValueError("the current RTDL lowering supports only precision='float_approx'; "
                         "precision='exact' is not implemented yet")
    name = compiled.refine_op.predicate.name
    if name not in NEIGHBOR_PREDICATES:
        raise ValueError(f"unsupported predicate for b200 backend: {name!r}")
    left, right = compiled.candidates.left, compiled.candidates.right
    if left.geometry.name != "points" or right.geometry.name != "points":
        raise ValueError(f"{name} lowering requires point build input and point probe input")


def _options(predicate_name: str, options) -> dict:
    if predicate_name == "knn_rows":
        return {"k": int(options["k"])}
    return {"radius": float(options["radius"]), "k_max": int(options["k_max"])}


_HOST_STEP_OPTION = re.compile(r"\b(radius|k_max|k)=([^\s,]+?)[.,]?(?=\s|,|$)")


def _options_from_host_steps(predicate_name: str, host_steps) -> dict:
    """The reference lowering writes the predicate options into its host steps
    as ``radius=<repr>``, ``k_max=<repr>`` or ``k=<repr>`` (lowering.py:468, 532,
    597); repr of a float round-trips exactly."""
    found = {}
    for step in host_steps:
        for key, value in _HOST_STEP_OPTION.findall(step):
            found[key] = value
    try:
        if predicate_name == "knn_rows":
            return {"k": int(found["k"])}
        return {"radius": float(found["radius"]), "k_max": int(found["k_max"])}
    except KeyError as ex:
        raise ValueError(f"the plan does not state the predicate option {ex.args[0]!r}; "
                         "pass the compiled kernel as well") from None


def _plan(kernel_name, predicate, precision, build_input, probe_input, query_input, search_input, emit_fields,
          options, input_names, source_plan=None) -> B200ExecutionPlan:
    dim = _dimension(query_input)
    entry = _ENTRY_POINTS[(predicate, dim)]
    record = _RECORD_NAMES[predicate]
    point_type = "RtdlPoint3D" if dim == 3 else "RtdlPoint"
    launch = (
        ("query_points", f"const {point_type}*", "host_input_probe"),
        ("query_count", "size_t", "launch_size"),
        ("search_points", f"const {point_type}*", "host_input_build"),
        ("search_count", "size_t", "build_size"),
    )
    if predicate == "knn_rows":
        launch += (("k", "size_t", "predicate_option"),)
    else:
        launch += (("radius", "double", "predicate_option"), ("k_max", "size_t", "predicate_option"))
    launch += (
        ("rows_out", f"{record}**", "host_output"),
        ("row_count_out", "size_t*", "host_counter"),
        ("error_out", "char*", "error_message"),
        ("error_size", "size_t", "error_capacity"),
    )
    fields = tuple((f, _EMIT_FIELD_TYPES.get(f, "unknown")) for f in emit_fields)
    if predicate == "knn_rows":
        steps = (f"Build an LBVH over `{search_input.name}` on the device (Morton codes, radix sort, Karras "
                 "hierarchy, refit).",
                 f"For each point of `{query_input.name}`, seed a nearest list from the Morton window, walk the "
                 "tree in FP32, re-decide the k-th-distance band in FP64.",
                 f"Emit the k={options['k']!r} nearest rows per query with 1-based neighbor_rank, ordered by "
                 "(distance, neighbor_id), grouped by query_id.")
        programs = ("k_pass1<KNN>", "k_expand")
    else:
        steps = (f"Build an LBVH over `{search_input.name}` on the device (Morton codes, radix sort, Karras "
                 "hierarchy, refit).",
                 f"Collect the points of `{search_input.name}` within the inclusive radius={options['radius']!r} "
                 "of each query in FP32; re-decide the radius band in FP64.",
                 f"Sort each query's candidates by (distance, neighbor_id), keep the k_max={options['k_max']!r} "
                 "nearest, emit rows grouped by query_id with exact FP64 distances"
                 + (" and 1-based neighbor_rank." if predicate == "bounded_knn_rows" else "."))
        programs = ("k_collect_packet", "k_emit", "k_emit_list", "k_emit_fixup", "k_heavy_gather_bvh")
    return B200ExecutionPlan(
        kernel_name=kernel_name,
        workload_kind=predicate,
        backend="b200",
        precision=precision,
        build_input=build_input,
        probe_input=probe_input,
        accel_kind="lbvh",
        predicate=predicate,
        exact_refine_mode=_EXACT_MODE,
        emit_fields=tuple(emit_fields),
        launch_params=launch,
        host_steps=steps,
        device_programs=programs,
        output_record=(record, fields),
        bvh_policy="LBVH built on the device per call (or once per prepared scene); collapsed leaf buckets, "
                   "rope-linked pre-order records",
        predicate_options=options,
        query_input=query_input.name,
        search_input=search_input.name,
        dimension=dim,
        entry_point=entry,
        input_names=tuple(input_names),
        source_plan=source_plan,
    )


def lower_to_b200_plan(kernel_or_plan, *, compiled=None) -> B200ExecutionPlan:
    """Lower a kernel (``@rt.kernel`` function or compiled kernel) or the
    reference's ``RTExecutionPlan`` to this backend's plan.  With a reference
    plan, ``compiled`` (optional) supplies the predicate options and the
    runners' left/right binding; without it they come from the plan itself."""
    if isinstance(kernel_or_plan, B200ExecutionPlan):
        return kernel_or_plan
    if _is_plan(kernel_or_plan):
        plan = kernel_or_plan
        if plan.predicate not in NEIGHBOR_PREDICATES:
            raise ValueError(f"unsupported predicate for b200 backend: {plan.predicate!r}")
        if plan.precision != "float_approx":
            raise ValueError("RTDL CPU simulator currently supports only precision='float_approx'")
        if compiled is not None:
            compiled = _resolve_compiled(compiled)
            _validate(compiled)
            if compiled.refine_op.predicate.name != plan.predicate:
                raise ValueError("the plan and the compiled kernel name different predicates")
            options = _options(plan.predicate, compiled.refine_op.predicate.options)
            query, search = compiled.candidates.left, compiled.candidates.right
            names = tuple(item.name for item in compiled.inputs)
        else:
            options = _options_from_host_steps(plan.predicate, plan.host_steps)
            query, search = plan.probe_input, plan.build_input
            names = (plan.probe_input.name, plan.build_input.name)
        return _plan(plan.kernel_name, plan.predicate, plan.precision, plan.build_input, plan.probe_input, query,
                     search, plan.emit_fields, options, names, source_plan=plan)
    compiled = _resolve_compiled(kernel_or_plan)
    _validate(compiled)
    build, probe = choose_roles(compiled.candidates)
    pred = compiled.refine_op.predicate
    return _plan(compiled.name, pred.name, compiled.precision, build, probe, compiled.candidates.left,
                 compiled.candidates.right, compiled.emit_op.fields, _options(pred.name, pred.options),
                 tuple(item.name for item in compiled.inputs))
