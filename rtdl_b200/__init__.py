"""rtdl_b200 -- B200-native backend for RTDL's neighbor path.

Fixed-radius neighbor rows, bounded-KNN rows, KNN rows and the directed
Hausdorff nearest-distance reduction, computed by hand-written sm_100a CUDA
kernels in ``librtdl_b200.so`` (C ABI: ``include/rtdl_b200.h``) and called
through ctypes.  The authoring API mirrors RTDL's (``rt.kernel``, ``rt.input``,
``rt.traverse``, ``rt.refine``, ``rt.emit``), so::

    import rtdl_b200 as rt

    @rt.kernel(backend="rtdl", precision="float_approx")
    def frn():
        q = rt.input("query_points", rt.Points3D, role="probe")
        s = rt.input("search_points", rt.Points3D, role="build")
        hits = rt.refine(rt.traverse(q, s, accel="bvh"),
                         predicate=rt.fixed_radius_neighbors(radius=0.1, k_max=64))
        return rt.emit(hits, fields=["query_id", "neighbor_id", "distance"])

    rows = rt.run_b200(frn, query_points=..., search_points=...)
"""
from .dsl import (  # noqa: F401
    CompiledKernel,
    Point,
    Point3D,
    Points,
    Points3D,
    bounded_knn_rows,
    compile_kernel,
    emit,
    fixed_radius_neighbors,
    input,
    kernel,
    knn_rows,
    refine,
    traverse,
)
from .execution import ExecutionPolicy, ExecutionResult, register_with_rtdsl, run  # noqa: F401
from .lowering import B200ExecutionPlan, lower_to_b200_plan  # noqa: F401
from .runtime import (  # noqa: F401
    B200Queries,
    B200RowView,
    B200Scene,
    PackedPoints,
    PreparedB200FixedRadiusNeighbors3D,
    PreparedB200FixedRadiusQueryPoints3D,
    PreparedB200FixedRadiusRankedSummaryAggregateBatchGraph3D,
    PreparedB200FixedRadiusCountThreshold2D,
    PreparedB200FixedRadiusCountThreshold3D,
    PreparedB200PointGroupNearestWitness2D,
    directed_hausdorff,
    fixed_radius_count_threshold_2d,
    prepare_b200_fixed_radius_count_threshold_2d,
    prepare_b200_fixed_radius_count_threshold_2d_device_search_columns,
    prepare_b200_fixed_radius_count_threshold_3d,
    prepare_b200_point_group_nearest_witness_2d,
    hausdorff_distance,
    pack_points,
    prepare_b200,
    prepare_b200_fixed_radius_neighbors_3d,
    run_b200,
    set_device,
    set_tuning,
)
from ._native import last_phase_timings, load_library  # noqa: F401

__version__ = "0.1.0"
