"""Kernel-authoring mirror for the neighbor path (``input -> traverse -> refine -> emit``).

Same names, argument meaning and validation messages as the reference's DSL,
restricted to what the neighbor path uses, so an ``@rt.kernel`` written for
RTDL runs unchanged against this backend without the reference installed:

* ``kernel``/``input``/``traverse``/``refine``/``emit``/``compile_kernel``:
  rubaolee/rtdl ``src/rtdsl/api.py:16-75, 78-127, 254-279``;
* ``fixed_radius_neighbors``/``knn_rows``/``bounded_knn_rows``:
  ``src/rtdsl/api.py:172-200``;
* ``Points``/``Points3D`` and their layouts: ``src/rtdsl/layout_types.py:75-88, 188-198``;
* ``Point``/``Point3D`` records: ``src/rtdsl/reference.py:16-28``;
* IR nodes and ``CompiledKernel``: ``src/rtdsl/ir.py``.

Compiled kernels of the real ``rtdsl`` package are accepted by the runtime
too (duck-typed on the same attributes).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from functools import wraps


@dataclass(frozen=True)
class ScalarType:
    name: str
    c_type: str
    cuda_type: str
    size: int


f32 = ScalarType(name="f32", c_type="float", cuda_type="float", size=4)
u32 = ScalarType(name="u32", c_type="uint32_t", cuda_type="uint32_t", size=4)


@dataclass(frozen=True)
class Field:
    name: str
    dtype: ScalarType


@dataclass(frozen=True)
class Layout:
    name: str
    fields: tuple[Field, ...]

    def field_names(self) -> tuple[str, ...]:
        return tuple(f.name for f in self.fields)

    def require_fields(self, names: tuple[str, ...]) -> None:
        available = set(self.field_names())
        missing = [n for n in names if n not in available]
        if missing:
            raise ValueError(f"layout `{self.name}` is missing required fields: {', '.join(missing)}")


@dataclass(frozen=True)
class GeometryType:
    name: str
    dimension: int
    default_layout: Layout
    required_fields: tuple[str, ...] = ()


Point2DLayout = Layout("Point2D", (Field("x", f32), Field("y", f32), Field("id", u32)))
Point3DLayout = Layout("Point3D", (Field("x", f32), Field("y", f32), Field("z", f32), Field("id", u32)))
Points = GeometryType(name="points", dimension=0, default_layout=Point2DLayout, required_fields=("x", "y", "id"))
Points3D = GeometryType(name="points", dimension=0, default_layout=Point3DLayout, required_fields=("x", "y", "z", "id"))


@dataclass(frozen=True)
class Point:
    id: int
    x: float
    y: float


@dataclass(frozen=True)
class Point3D:
    id: int
    x: float
    y: float
    z: float


@dataclass(frozen=True)
class GeometryInput:
    name: str
    geometry: GeometryType
    layout: Layout
    role: str | None = None


@dataclass(frozen=True)
class CandidateSet:
    left: GeometryInput
    right: GeometryInput
    accel: str
    mode: str | None = None


@dataclass(frozen=True)
class Predicate:
    name: str
    options: dict


@dataclass(frozen=True)
class RefineOp:
    candidates: CandidateSet
    predicate: Predicate


@dataclass(frozen=True)
class EmitOp:
    source: RefineOp
    fields: tuple[str, ...]


@dataclass(frozen=True)
class CompiledKernel:
    name: str
    backend: str
    precision: str
    inputs: tuple[GeometryInput, ...]
    candidates: CandidateSet | None
    refine_op: RefineOp | None
    emit_op: EmitOp | None
    lowering_plan: tuple[str, ...] = ()


@dataclass
class _KernelContext:
    name: str
    backend: str
    precision: str
    inputs: list = field(default_factory=list)
    candidates: CandidateSet | None = None
    refine_op: RefineOp | None = None
    emit_op: EmitOp | None = None

    def compile(self) -> CompiledKernel:
        return CompiledKernel(
            name=self.name,
            backend=self.backend,
            precision=self.precision,
            inputs=tuple(self.inputs),
            candidates=self.candidates,
            refine_op=self.refine_op,
            emit_op=self.emit_op,
            lowering_plan=(
                "Build an LBVH over the build-role points on the device.",
                "Traverse in FP32 and re-decide the error band in FP64.",
                "Emit rows grouped by query_id with exact FP64 distances.",
            ),
        )


_context_stack: list[_KernelContext] = []


def _current_context() -> _KernelContext:
    if not _context_stack:
        raise RuntimeError("RTDL operations must run inside @rt.kernel compilation")
    return _context_stack[-1]


def kernel(*, backend: str, precision: str):
    def decorator(fn):
        @wraps(fn)
        def wrapper():
            context = _KernelContext(name=fn.__name__, backend=backend, precision=precision)
            _context_stack.append(context)
            try:
                result = fn()
                if not isinstance(result, EmitOp):
                    raise TypeError("kernel function must return rt.emit(...)")
                return context.compile()
            finally:
                _context_stack.pop()

        wrapper._rtdsl_kernel = True
        return wrapper

    return decorator


def input(name: str, geometry: GeometryType, *, layout: Layout | None = None, role: str | None = None) -> GeometryInput:  # noqa: A001
    context = _current_context()
    if role is not None and role not in {"build", "probe"}:
        raise ValueError("input role must be one of: build, probe")
    if any(existing.name == name for existing in context.inputs):
        raise ValueError(f"duplicate input name in kernel: {name}")
    resolved = layout or geometry.default_layout
    if geometry.required_fields:
        resolved.require_fields(geometry.required_fields)
    node = GeometryInput(name=name, geometry=geometry, layout=resolved, role=role)
    context.inputs.append(node)
    return node


def traverse(left: GeometryInput, right: GeometryInput, *, accel: str = "bvh", mode: str | None = None) -> CandidateSet:
    context = _current_context()
    if mode is not None and mode not in {"graph_expand", "graph_intersect", "db_scan", "db_group"}:
        raise ValueError("traverse mode must be one of: graph_expand, graph_intersect, db_scan, db_group")
    node = CandidateSet(left=left, right=right, accel=accel, mode=mode)
    context.candidates = node
    return node


def fixed_radius_neighbors(*, radius: float, k_max: int) -> Predicate:
    if radius < 0.0:
        raise ValueError("fixed_radius_neighbors radius must be non-negative")
    if k_max <= 0:
        raise ValueError("fixed_radius_neighbors k_max must be positive")
    return Predicate(name="fixed_radius_neighbors", options={"radius": float(radius), "k_max": int(k_max)})


def knn_rows(*, k: int) -> Predicate:
    if k <= 0:
        raise ValueError("knn_rows k must be positive")
    return Predicate(name="knn_rows", options={"k": int(k)})


def bounded_knn_rows(*, radius: float, k_max: int) -> Predicate:
    if radius < 0.0:
        raise ValueError("bounded_knn_rows radius must be non-negative")
    if k_max <= 0:
        raise ValueError("bounded_knn_rows k_max must be positive")
    return Predicate(name="bounded_knn_rows", options={"radius": float(radius), "k_max": int(k_max)})


def refine(candidates: CandidateSet, *, predicate: Predicate) -> RefineOp:
    context = _current_context()
    node = RefineOp(candidates=candidates, predicate=predicate)
    context.refine_op = node
    return node


def emit(source: RefineOp, *, fields: list[str]) -> EmitOp:
    context = _current_context()
    node = EmitOp(source=source, fields=tuple(fields))
    context.emit_op = node
    return node


def compile_kernel(fn) -> CompiledKernel:
    if not callable(fn):
        raise TypeError("compile_kernel expects a kernel function")
    return fn()
