"""``rt.run`` facade and registration into RTDL's backend dispatch.

* ``run(kernel, inputs, execution=ExecutionPolicy(backend="b200"))`` mirrors
  rubaolee/rtdl ``src/rtdsl/execution.py:96-149`` for this backend, so code
  written against ``rt.run`` works without the reference installed.  There is
  no CPU fallback: ``allow_fallback=True`` is rejected, because a silent
  fallback would hide a failed GPU call.
* ``register_with_rtdsl()`` adds ``"b200"`` to the reference's
  ``_SUPPORTED_BACKENDS`` (``execution.py:16-25``) and routes it from
  ``_run_selected_backend`` (``execution.py:169-204``) to ``run_b200``, without
  editing the reference's files.
"""
from __future__ import annotations

import platform
from dataclasses import asdict, dataclass, field
from typing import Any, Mapping

from .runtime import _lower, run_b200

SUPPORTED_BACKENDS = ("b200",)


@dataclass(frozen=True)
class ExecutionPolicy:
    backend: str = "b200"
    partner: str | None = None
    allow_fallback: bool = False
    require_rt_core: bool = False
    explain: bool = True
    result_mode: str = "dict"

    def __post_init__(self) -> None:
        if self.backend not in SUPPORTED_BACKENDS:
            raise ValueError("backend must be one of: " + ", ".join(SUPPORTED_BACKENDS))
        if self.allow_fallback:
            raise ValueError("the b200 backend has no fallback; allow_fallback must be False")
        if self.require_rt_core:
            raise ValueError("require_rt_core is only supported with backend='auto' or backend='optix'")
        if self.result_mode not in {"dict", "raw"}:
            raise ValueError("result_mode must be 'dict' or 'raw'")


@dataclass(frozen=True)
class ExecutionReport:
    requested_backend: str
    selected_backend: str
    primitive_family: str
    predicate: str | None
    output_schema: tuple[str, ...]
    accel_kind: str
    exact_mode: str
    reproducibility: Mapping[str, str]
    notes: tuple[str, ...] = field(default_factory=tuple)

    def to_dict(self) -> dict[str, Any]:
        d = asdict(self)
        d["output_schema"] = list(self.output_schema)
        d["notes"] = list(self.notes)
        d["reproducibility"] = dict(self.reproducibility)
        return d


@dataclass(frozen=True)
class ExecutionResult:
    rows: Any
    execution_report: ExecutionReport

    def to_dict(self) -> dict[str, object]:
        rows = self.rows if isinstance(self.rows, tuple) else ()
        return {"rows": list(rows), "execution_report": self.execution_report.to_dict()}


def run(kernel_fn_or_compiled, inputs: Mapping[str, object] | None = None, *, execution: ExecutionPolicy | None = None,
        **input_kwargs) -> ExecutionResult:
    policy = execution or ExecutionPolicy()
    merged = dict(inputs or {})
    merged.update(input_kwargs)
    plan = _lower(kernel_fn_or_compiled)
    rows = run_b200(plan, result_mode=policy.result_mode, **merged)
    report = ExecutionReport(
        requested_backend=policy.backend,
        selected_backend="b200",
        primitive_family="nearest_neighbor",
        predicate=plan.predicate,
        output_schema=tuple(plan.emit_fields),
        accel_kind=plan.accel_kind,
        exact_mode=plan.exact_refine_mode,
        reproducibility={"python": platform.python_version(), "platform": platform.platform()},
        notes=("Rows from librtdl_b200 (sm_100a); FP32 traversal with FP64 re-decision inside the error band.",),
    )
    return ExecutionResult(rows=tuple(rows) if policy.result_mode == "dict" else rows, execution_report=report)


def register_with_rtdsl(rtdsl_module=None) -> None:
    """Register ``"b200"`` as one more backend name in the reference's dispatch."""
    if rtdsl_module is None:
        import rtdsl as rtdsl_module  # noqa: F401  (the reference package, when installed)
    import importlib

    ex = importlib.import_module(rtdsl_module.__name__ + ".execution")
    if "b200" not in ex._SUPPORTED_BACKENDS:
        ex._SUPPORTED_BACKENDS = tuple(ex._SUPPORTED_BACKENDS) + ("b200",)
    original = ex._run_selected_backend
    if getattr(original, "_rtdl_b200_patched", False):
        return

    def _run_selected_backend(backend, kernel_fn_or_compiled, *, policy, inputs):
        if backend == "b200":
            return run_b200(kernel_fn_or_compiled, result_mode=policy.result_mode, **dict(inputs))
        return original(backend, kernel_fn_or_compiled, policy=policy, inputs=inputs)

    _run_selected_backend._rtdl_b200_patched = True
    ex._run_selected_backend = _run_selected_backend
    rtdsl_module.run_b200 = run_b200
    from .lowering import lower_to_b200_plan

    rtdsl_module.lower_to_b200_plan = lower_to_b200_plan
