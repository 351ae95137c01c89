/*
 * rtdl_b200.h -- C ABI of librtdl_b200.so, the B200-native RTDL neighbor backend.
 *
 * The entry points are the ones RTDL's ctypes layer binds for its OptiX
 * neighbor path, renamed from rtdl_optix_* to rtdl_b200_* with the same
 * argument order, meaning, ownership and error convention, so a Python or C
 * caller switches backends by changing the symbol prefix.  Citations are to
 * rubaolee/rtdl (paths within that project).
 *
 * Conventions shared by every int-returning entry point
 * (src/native/optix/rtdl_optix_core.cpp:58-66, rtdl_optix_api.cpp:4084-4100):
 *   - returns 0 on success, 1 on failure with a NUL-terminated message copied
 *     into error_out (truncated to error_size); nothing is thrown across the ABI;
 *   - *rows_out / *row_count_out are zeroed before any work; empty query or
 *     search sets return 0 rows;
 *   - rows are owned by the caller and released with rtdl_b200_free_rows
 *     (rtdl_optix_api.cpp:5698); inputs are borrowed for the call only;
 *   - validation messages match the reference: "radius must be non-negative",
 *     "k_max must be positive", "... exceeds uint32 limit".
 * Row order equals the reference's cpu_python_reference
 * (src/rtdsl/reference.py:349-434): rows grouped by query_id (stable in query
 * input order), within a query by (distance, neighbor_id, search input order).
 * Row sets and distances are bit-identical to that reference: the device
 * decides in FP32 and re-decides every case within the error band in FP64,
 * and each emitted distance is sqrt((dx*dx + dy*dy) + dz*dz) in FP64 with no
 * fused multiply-add.
 */
#ifndef RTDL_B200_H
#define RTDL_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(RTDL_B200_BUILD) && defined(__GNUC__)
#define RTDL_B200_API __attribute__((visibility("default")))
#else
#define RTDL_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Point and row records: same layouts as src/native/optix/rtdl_optix_prelude.h
 * :103-106 (RtdlPoint), :138-141 (RtdlPoint3D), :254-260
 * (RtdlFixedRadiusNeighborRow, 16 B) and :289-295 (RtdlKnnNeighborRow, 24 B). */
typedef struct RtdlPoint {
  uint32_t id;
  double x, y;
} RtdlPoint;

typedef struct RtdlPoint3D {
  uint32_t id;
  double x, y, z;
} RtdlPoint3D;

typedef struct RtdlFixedRadiusNeighborRow {
  uint32_t query_id, neighbor_id;
  double distance;
} RtdlFixedRadiusNeighborRow;

typedef struct RtdlKnnNeighborRow {
  uint32_t query_id, neighbor_id;
  double distance;
  uint32_t neighbor_rank;
} RtdlKnnNeighborRow;

/* Per-query ranked summary and its aggregate over a query set: same layouts
 * as src/native/optix/rtdl_optix_prelude.h:300-316
 * (RtdlFixedRadiusRankedNeighborSummary, 40 B) and :318-329
 * (RtdlFixedRadiusRankedNeighborAggregate, 40 B).  A query without
 * neighbours in radius has count 0, ids 0xFFFFFFFF and distances 0. */
typedef struct RtdlFixedRadiusRankedNeighborSummary {
  uint32_t query_id;
  uint32_t neighbor_count;       /* min(in-radius count, k_max) */
  uint32_t nearest_neighbor_id;  /* first row of the query's fixed_radius_neighbors rows */
  uint32_t kth_neighbor_id;      /* last row */
  double nearest_distance;
  double kth_distance;
  double sum_distance;           /* the rows' distances added in row order */
} RtdlFixedRadiusRankedNeighborSummary;

typedef struct RtdlFixedRadiusRankedNeighborAggregate {
  size_t query_count;
  size_t bounded_neighbor_count;  /* sum of neighbor_count */
  uint64_t nearest_id_checksum;   /* sum of nearest_neighbor_id (mod 2^64) */
  uint64_t kth_id_checksum;       /* sum of kth_neighbor_id (mod 2^64) */
  double sum_distance;            /* sum of sum_distance (fixed reduction order, run to run identical) */
} RtdlFixedRadiusRankedNeighborAggregate;

/* One row of fixed_radius_count_threshold: same layout as
 * src/native/optix/rtdl_optix_prelude.h:276-280 (RtdlFixedRadiusCountRow, 12 B). */
typedef struct RtdlFixedRadiusCountRow {
  uint32_t query_id;
  uint32_t neighbor_count;     /* in-radius count, capped at the threshold when it is positive */
  uint32_t threshold_reached;  /* 1 when the threshold is positive and was reached */
} RtdlFixedRadiusCountRow;

/* A group of search points for the point-group witness: a span of the search
 * array and its bounding box; same layout as
 * src/native/optix/rtdl_optix_prelude.h:282-287 (RtdlPointGroupBounds2D, 48 B). */
typedef struct RtdlPointGroupBounds2D {
  uint32_t id;
  uint32_t point_offset;
  uint32_t point_count;
  double min_x, min_y, max_x, max_y;
} RtdlPointGroupBounds2D;

/* Version triple (the reference exports rtdl_optix_get_version,
 * rtdl_optix_api.cpp:1-7). */
RTDL_B200_API int rtdl_b200_get_version(int* major, int* minor, int* patch);

/* Makes `device` current for the calling thread's later calls (the library
 * links the CUDA runtime statically, so it keeps its own current device).
 * No counterpart in the reference, which drives one GPU. */
RTDL_B200_API int rtdl_b200_set_device(int device);

/* ---- plain per-call launches ------------------------------------------- */

/* Replaces rtdl_optix_run_fixed_radius_neighbors (rtdl_optix_api.cpp:4076-4105). */
RTDL_B200_API int rtdl_b200_run_fixed_radius_neighbors(
    const RtdlPoint* query_points, size_t query_count,
    const RtdlPoint* search_points, size_t search_count,
    double radius, size_t k_max,
    RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_run_fixed_radius_neighbors_3d (rtdl_optix_api.cpp:4107-4150). */
RTDL_B200_API int rtdl_b200_run_fixed_radius_neighbors_3d(
    const RtdlPoint3D* query_points, size_t query_count,
    const RtdlPoint3D* search_points, size_t search_count,
    double radius, size_t k_max,
    RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* No counterpart in the reference: the plain per-call form with device
 * buffers (records already in HBM).  Builds the scene of search_points_dev and
 * writes the fixed_radius_neighbors rows of query_points_dev (the
 * RtdlPoint / RtdlPoint3D layout of `dimension`) into rows_dev, like
 * rtdl_b200_run_fixed_radius_neighbors[_3d] (rows in the reference's order);
 * rows_dev NULL only counts.  overflow_dev (optional, one byte per query) is
 * 1 where the in-radius count exceeds k_max.  With k_max <= 64 the query set
 * is prepared on a second stream while the scene builds.  Work runs on
 * `stream` (NULL = the library's stream), which is synchronised before return. */
RTDL_B200_API int rtdl_b200_run_fixed_radius_neighbors_device(
    const void* query_points_dev, size_t query_count, const void* search_points_dev, size_t search_count,
    int dimension, double radius, size_t k_max, void* rows_dev, size_t rows_capacity, size_t* row_count_out,
    uint8_t* overflow_dev, void* stream, char* error_out, size_t error_size);

/* bounded_knn_rows with ranks assigned on the device.  The reference builds
 * these rows in Python from the FRN rows (src/rtdsl/optix_runtime.py:15834-15862);
 * the rows equal src/rtdsl/reference.py:406-434. */
RTDL_B200_API int rtdl_b200_run_bounded_knn_rows(
    const RtdlPoint* query_points, size_t query_count,
    const RtdlPoint* search_points, size_t search_count,
    double radius, size_t k_max,
    RtdlKnnNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

RTDL_B200_API int rtdl_b200_run_bounded_knn_rows_3d(
    const RtdlPoint3D* query_points, size_t query_count,
    const RtdlPoint3D* search_points, size_t search_count,
    double radius, size_t k_max,
    RtdlKnnNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_run_k_closest_hits (rtdl_optix_api.cpp:4971-4997). */
RTDL_B200_API int rtdl_b200_run_k_closest_hits(
    const RtdlPoint* query_points, size_t query_count,
    const RtdlPoint* search_points, size_t search_count,
    size_t k,
    RtdlKnnNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_run_k_closest_hits_3d (rtdl_optix_api.cpp:4999-5025). */
RTDL_B200_API int rtdl_b200_run_k_closest_hits_3d(
    const RtdlPoint3D* query_points, size_t query_count,
    const RtdlPoint3D* search_points, size_t search_count,
    size_t k,
    RtdlKnnNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_free_rows (rtdl_optix_api.cpp:5698). */
RTDL_B200_API void rtdl_b200_free_rows(void* rows);

/* ---- prepared scenes (resident BVH on the device) ---------------------- */

/* Replaces rtdl_optix_prepare_fixed_radius_neighbors_3d (rtdl_optix_api.cpp:4152-4171).
 * The scene is an LBVH over the search points kept resident on the device;
 * max_radius is validated like the reference (must be positive) and recorded,
 * and later calls must use radius <= max_radius. */
RTDL_B200_API int rtdl_b200_prepare_fixed_radius_neighbors_3d(
    const RtdlPoint3D* search_points, size_t search_count,
    double max_radius,
    void** prepared_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_run_prepared_fixed_radius_neighbors_3d (rtdl_optix_api.cpp:4173-4186). */
RTDL_B200_API int rtdl_b200_run_prepared_fixed_radius_neighbors_3d(
    void* prepared,
    const RtdlPoint3D* query_points, size_t query_count,
    double radius, size_t k_max,
    RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_destroy_prepared_fixed_radius_neighbors_3d (rtdl_optix_api.cpp:4432). */
RTDL_B200_API void rtdl_b200_destroy_prepared_fixed_radius_neighbors_3d(void* prepared);

/* ---- scenes of either dimension (new: the reference only prepares 3D FRN) --
 * A scene is an LBVH built on the device over 2D or 3D search points.  One
 * scene serves FRN, bounded KNN, KNN and nearest-distance calls. */

/* dimension is 2 (points are RtdlPoint) or 3 (RtdlPoint3D).  points_on_device
 * != 0 means `points` is a device pointer.  stream may be NULL (the library's
 * own stream). */
RTDL_B200_API int rtdl_b200_scene_create(
    const void* points, size_t count, int dimension, int points_on_device,
    void* stream, void** scene_out,
    char* error_out, size_t error_size);

RTDL_B200_API void rtdl_b200_scene_destroy(void* scene);

/* Host-buffer call on a scene.  predicate: 0 = fixed_radius_neighbors
 * (RtdlFixedRadiusNeighborRow rows), 1 = bounded_knn_rows and 2 = knn_rows
 * (RtdlKnnNeighborRow rows).  `limit` is k_max (0, 1) or k (2); radius is
 * ignored for knn_rows.  overflow_out (optional, query_count bytes, query
 * input order) receives 1 where a query had more than k_max neighbors inside
 * the radius (the rows still hold the k_max nearest). */
RTDL_B200_API int rtdl_b200_scene_query(
    void* scene, const void* query_points, size_t query_count,
    int predicate, double radius, size_t limit,
    void** rows_out, size_t* row_count_out, uint8_t* overflow_out,
    char* error_out, size_t error_size);

/* Device-resident call: query points, rows and flags live in device memory
 * and the work is enqueued on `stream`; no host buffer is touched.  Rows
 * beyond rows_capacity are not written; *row_count_out receives the full row
 * count, so a caller whose capacity was too small retries with more.
 * overflow_dev (optional) receives one byte per query (query input order). */
RTDL_B200_API int rtdl_b200_scene_query_device(
    void* scene, const void* query_points_dev, size_t query_count,
    int predicate, double radius, size_t limit,
    void* rows_dev, size_t rows_capacity, size_t* row_count_out,
    uint8_t* overflow_dev, void* stream,
    char* error_out, size_t error_size);

/* Directed nearest-distance reduction (Hausdorff).  For every query the exact
 * nearest (distance, neighbor_id) of knn_rows(k=1); then the witness is the
 * maximum of (distance, -query_id, -neighbor_id) over all queries, the rule of
 * examples/v2_0/research_benchmarks/hausdorff_xhd/rtdl_hausdorff_distance_app.py:108-130,
 * reduced on the device in FP64.  nearest_distance_out / nearest_id_out are
 * optional host arrays of query_count entries in query input order. */
RTDL_B200_API int rtdl_b200_scene_directed_hausdorff(
    void* scene, const void* query_points, size_t query_count,
    double* distance_out, uint32_t* source_id_out, uint32_t* target_id_out,
    double* nearest_distance_out, uint32_t* nearest_id_out,
    char* error_out, size_t error_size);

/* Device-resident form of rtdl_b200_scene_directed_hausdorff: the queries and
 * the optional per-query outputs are device pointers, the work runs on
 * `stream` (NULL = the scene's stream) and the witness is returned to the
 * host after the stream finishes. */
RTDL_B200_API int rtdl_b200_scene_directed_hausdorff_device(
    void* scene, const void* query_points_dev, size_t query_count,
    double* nearest_distance_dev, uint32_t* nearest_id_dev,
    double* distance_out, uint32_t* source_id_out, uint32_t* target_id_out,
    void* stream, char* error_out, size_t error_size);

/* ---- problem batches -------------------------------------------------------
 * Many independent fixed-radius problems of uneven sizes answered together:
 * one LBVH build over all problems' points (the sort key carries the problem
 * id, so every problem is a subtree of its own) and one collect / emit launch
 * sequence over all queries, each warp walking its problem's subtree.  No
 * reference counterpart: the reference runs one call per problem
 * (rtdl_optix_api.cpp:4076-4150); its batched form only splits one query set
 * into chunks (rtdl_optix_workloads.cpp:14380-14409). */

/* Builds the batch.  points: the problems' RtdlPoint / RtdlPoint3D records back
 * to back, problem p at [point_offsets[p], point_offsets[p + 1]) (host array
 * of problems + 1 entries, starting at 0); points_on_device says whether
 * `points` is a device pointer.  At most 67,108,864 points in all.  The
 * handle is released with rtdl_b200_batch_destroy. */
RTDL_B200_API int rtdl_b200_batch_create(
    const void* points, const unsigned long long* point_offsets, uint32_t problems,
    int dimension, int points_on_device, void* stream, void** batch_out,
    char* error_out, size_t error_size);

RTDL_B200_API void rtdl_b200_batch_destroy(void* batch);

/* fixed_radius_neighbors for every problem: problem p's queries are
 * [query_offsets[p], query_offsets[p + 1]) of query_points (host records),
 * with radius[p] and k_max[p] (1..64).  Rows come back problem by problem,
 * each problem's exactly as rtdl_b200_run_fixed_radius_neighbors[_3d] returns
 * them for that problem alone; row_offsets_out (problems + 1 entries) receives
 * each problem's first row and the total.  *rows_out is released with
 * rtdl_b200_free_rows.  overflow_out (optional, one byte per query) is 1 where
 * a query had more than k_max points in radius. */
RTDL_B200_API int rtdl_b200_batch_fixed_radius_neighbors(
    void* batch, const void* query_points, const unsigned long long* query_offsets,
    const double* radius, const uint32_t* k_max,
    RtdlFixedRadiusNeighborRow** rows_out, unsigned long long* row_offsets_out,
    uint8_t* overflow_out, char* error_out, size_t error_size);

/* Device-resident form: query records and rows are device pointers, rows are
 * written up to rows_capacity (row_offsets_out still reports every problem's
 * full count, so a first call with capacity 0 sizes the buffer); the work runs
 * on `stream` (NULL = the batch's stream). */
RTDL_B200_API int rtdl_b200_batch_fixed_radius_neighbors_device(
    void* batch, const void* query_points_dev, const unsigned long long* query_offsets,
    const double* radius, const uint32_t* k_max, void* rows_dev, size_t rows_capacity,
    unsigned long long* row_offsets_out, uint8_t* overflow_dev, void* stream,
    char* error_out, size_t error_size);

/* ---- captured graph over prepared problem batches ---------------------------
 * The reference's batch graph (rtdl_optix_api.cpp:4323-4396,
 * rtdl_optix_workloads.cpp:14378-14393: capture once, replay a launch over
 * prepared inputs) for problem batches.  `batches` are batch_count handles of
 * rtdl_b200_batch_create; their problems are numbered in order (batch 0's
 * first).  query_points_dev holds every problem's device query records back
 * to back, problem p at [query_offsets[p], query_offsets[p + 1]) (host array,
 * total problems + 1 entries), with radius[p] and k_max[p] (1..64).  One
 * replay answers every problem: per batch one persistent collect launch takes
 * 32-query packets from a device work queue, then the scan, the radius
 * refinement and the emit run device-driven (nothing is read back inside the
 * graph).  Rows go to rows_dev (device, capacity rows_capacity rows) problem
 * by problem, each problem's exactly as rtdl_b200_batch_fixed_radius_neighbors
 * returns them.  The query records, the batches and rows_dev must stay valid
 * until the graph is destroyed. */
RTDL_B200_API int rtdl_b200_batch_graph_create(
    void* const* batches, uint32_t batch_count, const void* query_points_dev,
    const unsigned long long* query_offsets, const double* radius, const uint32_t* k_max,
    void* rows_dev, size_t rows_capacity, void** graph_out, char* error_out, size_t error_size);

/* Replays the graph and waits: row_offsets_out (optional, problems + 1
 * entries) receives each problem's first row and the total; status_out
 * (optional) the OR of the batches' status bits (4: the rows exceeded
 * rows_capacity, rows past it were not written).  A batch with heavy queries
 * the refinement did not resolve is recomputed by the plain batch call. */
RTDL_B200_API int rtdl_b200_batch_graph_replay(
    void* graph, unsigned long long* row_offsets_out, uint32_t* status_out, char* error_out, size_t error_size);

/* Enqueues one replay ordered after `stream`'s earlier work and before its
 * later work, without waiting or reading anything back (no recompute of
 * flagged batches: check with a replay when unsure). */
RTDL_B200_API int rtdl_b200_batch_graph_launch(void* graph, void* stream, char* error_out, size_t error_size);

/* Problems, kernel nodes of one replay, batches recomputed so far. */
RTDL_B200_API int rtdl_b200_batch_graph_info(void* graph, uint32_t* problems_out, int* kernel_nodes_out,
                                             unsigned long long* fallbacks_out);

RTDL_B200_API void rtdl_b200_batch_graph_destroy(void* graph);

/* Several fixed_radius_neighbors requests against one resident scene (from
 * rtdl_b200_scene_create) answered by one launch sequence: request r's
 * queries are [query_offsets[r], query_offsets[r + 1]) of query_points_dev,
 * with radius[r] and k_max[r] (1..64).  Rows come out request by request,
 * each request's exactly as rtdl_b200_scene_query_device returns them for
 * that request alone; row_offsets_out (requests + 1 entries) receives each
 * request's first row and the total.  The served request loop batches with
 * it.  No reference counterpart (the reference serves one query set per
 * call, rtdl_optix_api.cpp:4152-4435). */
RTDL_B200_API int rtdl_b200_scene_fixed_radius_neighbors_multi_device(
    void* scene, const void* query_points_dev, const unsigned long long* query_offsets, uint32_t requests,
    const double* radius, const uint32_t* k_max, void* rows_dev, size_t rows_capacity,
    unsigned long long* row_offsets_out, uint8_t* overflow_dev, void* stream,
    char* error_out, size_t error_size);

/* ---- ranked summaries --------------------------------------------------------
 * fixed_radius_neighbors reduced per query to the reference's ranked summary
 * (neighbour count, first and last row, sum of the row distances) and to the
 * aggregate over the query set, without returning rows.  k_max <= 64. */

/* Replaces rtdl_optix_run_prepared_ranked_fixed_radius_neighbor_summaries_3d
 * (rtdl_optix_api.cpp:4218-4231): one summary per query, in query order;
 * *rows_out is released with rtdl_b200_free_rows. */
RTDL_B200_API int rtdl_b200_run_prepared_ranked_fixed_radius_neighbor_summaries_3d(
    void* prepared, const RtdlPoint3D* query_points, size_t query_count, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborSummary** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replaces rtdl_optix_aggregate_prepared_ranked_fixed_radius_neighbor_summaries_3d
 * (rtdl_optix_api.cpp:4251-4266). */
RTDL_B200_API int rtdl_b200_aggregate_prepared_ranked_fixed_radius_neighbor_summaries_3d(
    void* prepared, const RtdlPoint3D* query_points, size_t query_count, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, char* error_out, size_t error_size);

/* Device-resident form on any scene (2D or 3D): query records on the device,
 * optional per-query summaries written to summaries_dev (query order), the
 * aggregate returned to the host after `stream` (NULL = the scene's stream)
 * finishes.  Against an empty scene nothing is written to summaries_dev and
 * the aggregate is zero apart from query_count. */
RTDL_B200_API int rtdl_b200_scene_ranked_summaries_device(
    void* scene, const void* query_points_dev, size_t query_count, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborSummary* summaries_dev,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, void* stream,
    char* error_out, size_t error_size);

/* ---- prepared query sets -------------------------------------------------------
 * A query set prepared once (uploaded, converted, ordered) for repeated
 * fixed-radius calls against resident scenes.  Handles are released with
 * rtdl_b200_queries_destroy. */
RTDL_B200_API int rtdl_b200_queries_create(
    const void* points, size_t count, int dimension, int points_on_device, void* stream,
    void** queries_out, char* error_out, size_t error_size);

RTDL_B200_API void rtdl_b200_queries_destroy(void* queries);

/* Replaces rtdl_optix_prepare_fixed_radius_query_points_3d
 * (rtdl_optix_api.cpp:4233-4249) and its destroy (:4437). */
RTDL_B200_API int rtdl_b200_prepare_fixed_radius_query_points_3d(
    const RtdlPoint3D* query_points, size_t query_count, void** prepared_queries_out,
    char* error_out, size_t error_size);

RTDL_B200_API void rtdl_b200_destroy_prepared_fixed_radius_query_points_3d(void* prepared_queries);

/* Replaces rtdl_optix_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d_f32
 * (rtdl_optix_api.cpp:4284-4299); the _f32 name computes the same exact
 * aggregate. */
RTDL_B200_API int rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d(
    void* prepared, void* prepared_queries, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, char* error_out, size_t error_size);

RTDL_B200_API int rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d_f32(
    void* prepared, void* prepared_queries, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, char* error_out, size_t error_size);

/* Ranked summaries and fixed_radius_neighbors rows (k_max <= 64) of a
 * prepared query set against a resident scene, device-resident outputs, on
 * `stream` (NULL = the scene's stream). */
RTDL_B200_API int rtdl_b200_scene_ranked_summaries_prepared_device(
    void* scene, void* queries, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborSummary* summaries_dev,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, void* stream,
    char* error_out, size_t error_size);

RTDL_B200_API int rtdl_b200_scene_query_prepared_device(
    void* scene, void* queries, double radius, size_t k_max, void* rows_dev, size_t rows_capacity,
    size_t* row_count_out, uint8_t* overflow_dev, void* stream, char* error_out, size_t error_size);

/* ---- fixed_radius_count_threshold and the nearest in-radius witness ------------
 * Counts follow the reference's generic count (src/rtdsl/generic_primitives.py
 * :198-227): a query's points within radius (inclusive, FP64 distances) are
 * counted until a positive threshold is reached; threshold 0 counts them all.
 * One RtdlFixedRadiusCountRow / output element per query, in input order.
 * Prepared handles are scenes with a max_radius; radius may exceed it by at
 * most 1e-7, as in the reference. */

/* Replaces rtdl_optix_run_fixed_radius_count_threshold (rtdl_optix_api.cpp:4738-4765). */
RTDL_B200_API int rtdl_b200_run_fixed_radius_count_threshold(
    const RtdlPoint* query_points, size_t query_count, const RtdlPoint* search_points, size_t search_count,
    double radius, size_t threshold, RtdlFixedRadiusCountRow** rows_out, size_t* row_count_out,
    char* error_out, size_t error_size);

/* Replace rtdl_optix_prepare_fixed_radius_count_threshold_2d[_device_search_columns]
 * (rtdl_optix_api.cpp:4767-4810); the columns are device buffers. */
RTDL_B200_API int rtdl_b200_prepare_fixed_radius_count_threshold_2d(
    const RtdlPoint* search_points, size_t search_count, double max_radius, void** prepared_out,
    char* error_out, size_t error_size);
RTDL_B200_API int rtdl_b200_prepare_fixed_radius_count_threshold_2d_device_search_columns(
    const uint32_t* search_ids, const double* search_x, const double* search_y, size_t search_count,
    double max_radius, void** prepared_out, char* error_out, size_t error_size);

/* Replaces rtdl_optix_run_prepared_fixed_radius_count_threshold_2d
 * (rtdl_optix_workloads.cpp:13242-13320); rows are released with rtdl_b200_free_rows. */
RTDL_B200_API int rtdl_b200_run_prepared_fixed_radius_count_threshold_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius, size_t threshold,
    RtdlFixedRadiusCountRow** rows_out, size_t* row_count_out, char* error_out, size_t error_size);

/* Replaces rtdl_optix_write_prepared_fixed_radius_count_threshold_2d_device_query_columns
 * (rtdl_optix_workloads.cpp:13322-13400): device query columns in, device output
 * columns out; needs a handle prepared from device search columns. */
RTDL_B200_API int rtdl_b200_write_prepared_fixed_radius_count_threshold_2d_device_query_columns(
    void* prepared, const uint32_t* query_ids, const double* query_x, const double* query_y, size_t query_count,
    double radius, size_t threshold, uint32_t* query_ids_out, uint32_t* neighbor_counts_out,
    uint32_t* threshold_flags_out, char* error_out, size_t error_size);

/* Replaces rtdl_optix_count_prepared_fixed_radius_threshold_reached_2d
 * (rtdl_optix_workloads.cpp:13400-13466): how many queries reached the threshold. */
RTDL_B200_API int rtdl_b200_count_prepared_fixed_radius_threshold_reached_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius, size_t threshold,
    size_t* threshold_reached_count_out, char* error_out, size_t error_size);

/* Replaces rtdl_optix_run_prepared_fixed_radius_nearest_witness_2d
 * (rtdl_optix_workloads.cpp:13468-13552): one row per query in input order,
 * the nearest point within radius (ties to the smaller id; exact FP64
 * distance), or neighbor_id 0xFFFFFFFF and distance FLT_MAX when none. */
RTDL_B200_API int rtdl_b200_run_prepared_fixed_radius_nearest_witness_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius,
    RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out, char* error_out, size_t error_size);

RTDL_B200_API void rtdl_b200_destroy_prepared_fixed_radius_count_threshold_2d(void* prepared);

/* Replace rtdl_optix_prepare_fixed_radius_count_threshold_3d and
 * rtdl_optix_write_prepared_fixed_radius_count_threshold_3d_device_outputs
 * (rtdl_optix_api.cpp:4442-4470, rtdl_optix_workloads.cpp:16491-16560): host
 * query records in, device output columns out.  As in the reference's 3-D
 * contract, threshold 0 gives every query count 0 and flag 1. */
RTDL_B200_API int rtdl_b200_prepare_fixed_radius_count_threshold_3d(
    const RtdlPoint3D* search_points, size_t search_count, double max_radius, void** prepared_out,
    char* error_out, size_t error_size);
RTDL_B200_API int rtdl_b200_write_prepared_fixed_radius_count_threshold_3d_device_outputs(
    void* prepared, const RtdlPoint3D* query_points, size_t query_count, double radius, size_t threshold,
    uint32_t* query_ids_out, uint32_t* neighbor_counts_out, uint32_t* threshold_flags_out,
    char* error_out, size_t error_size);
RTDL_B200_API void rtdl_b200_destroy_prepared_fixed_radius_count_threshold_3d(void* prepared);

/* ---- point-group witness (2-D) ----------------------------------------------------
 * Replace the entry points of the reference's prepared point-group nearest
 * witness (rtdl_optix_prelude.h:1480-1512; rtdl_optix_api.cpp:4885-4990 and
 * rtdl_optix_workloads.cpp:13554-13880).  Groups are spans of the search array
 * with a bounding box; a search point takes part for a query when it and its
 * group's box are within radius (FP64, inclusive), once per group that holds
 * it.  Threshold: counting stops at a positive threshold; the flag is 1 when it
 * was reached (0 for threshold 0, except without groups, where threshold 0
 * counts as reached, as in the reference).  Witness: per query (input order)
 * the nearest such point by exact distance then smaller id, or neighbor_id
 * 0xFFFFFFFF and distance FLT_MAX.  Max distance: the witness row of largest
 * distance (then smaller query id, then smaller neighbour id), a query without
 * a witness counting as infinitely far; {0xFFFFFFFF, 0xFFFFFFFF, inf} when
 * there are no queries or groups. */
RTDL_B200_API int rtdl_b200_prepare_point_group_nearest_witness_2d(
    const RtdlPoint* search_points, size_t search_count, const RtdlPointGroupBounds2D* groups, size_t group_count,
    double max_radius, void** prepared_out, char* error_out, size_t error_size);
RTDL_B200_API int rtdl_b200_count_prepared_point_group_threshold_reached_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius, size_t threshold,
    size_t* threshold_reached_count_out, char* error_out, size_t error_size);
/* threshold_flags_out: host array of query_count words. */
RTDL_B200_API int rtdl_b200_write_prepared_point_group_threshold_flags_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius, size_t threshold,
    uint32_t* threshold_flags_out, char* error_out, size_t error_size);
RTDL_B200_API int rtdl_b200_run_prepared_point_group_nearest_witness_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius,
    RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out, char* error_out, size_t error_size);
RTDL_B200_API int rtdl_b200_reduce_prepared_point_group_nearest_max_distance_2d(
    void* prepared, const RtdlPoint* query_points, size_t query_count, double radius,
    RtdlFixedRadiusNeighborRow* row_out, char* error_out, size_t error_size);
RTDL_B200_API void rtdl_b200_destroy_prepared_point_group_nearest_witness_2d(void* prepared);

/* ---- captured batch graph of prepared-query aggregates -----------------------
 * Replace the batch-graph entry points of rtdl_optix_api.cpp:4323-4396
 * (prepare / replay / launch-with-device-partials / update / destroy).
 * One CUDA graph holds, for each (radius, k_max) request in order, the whole
 * fixed-radius path over the prepared query set (collect, device-driven
 * heavy-query refinement, emit into an internal row buffer, ranked summary,
 * aggregate); all buffers are allocated at prepare.  The graph runs on its own
 * stream.  update re-captures it with new requests (same request_count).
 * The aggregates are the exact ones of
 * rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d.
 * Requests: radius in [0, max_radius], 1 <= k_max <= 64; both handles
 * non-empty.  No query-count cap beyond device memory (nq x 2 KiB of slab plus
 * nq x k_max rows). */
RTDL_B200_API int rtdl_b200_prepare_fixed_radius_ranked_summary_aggregate_batch_graph_3d(
    void* prepared, void* prepared_queries, const double* radii, const size_t* k_values, size_t request_count,
    void** graph_out, char* error_out, size_t error_size);

/* Replays the graph and writes request_count aggregates.  A request whose
 * heavy queries the refinement passes left unresolved is recomputed by the
 * plain call (its generic path) before this returns. */
RTDL_B200_API int rtdl_b200_replay_fixed_radius_ranked_summary_aggregate_batch_graph_3d(
    void* graph, RtdlFixedRadiusRankedNeighborAggregate* aggregates_out, char* error_out, size_t error_size);

/* Enqueues a replay and returns without waiting: the partials are one
 * RtdlFixedRadiusRankedNeighborAggregate per request in device memory
 * (query_block_count = 1), valid once the returned stream reaches this point.
 * A request whose device status word (below) is nonzero has no valid partial:
 * replay computes it. */
RTDL_B200_API int rtdl_b200_launch_fixed_radius_ranked_summary_aggregate_batch_graph_device_partials_3d(
    void* graph, uint64_t* partials_device_ptr_out, size_t* partial_count_out, size_t* request_count_out,
    size_t* query_block_count_out, uint64_t* cuda_stream_ptr_out, char* error_out, size_t error_size);

/* No counterpart in the reference: the device address of the per-request
 * status words of the last replay (0 = the partial is valid; bit 0 traversal
 * stack overflow; bit 1 heavy queries left for the generic path) and how many
 * requests replay has recomputed by the plain call so far. */
RTDL_B200_API int rtdl_b200_fixed_radius_ranked_summary_aggregate_batch_graph_status_device_3d(
    void* graph, uint64_t* status_device_ptr_out, uint64_t* fallback_count_out, char* error_out, size_t error_size);

RTDL_B200_API int rtdl_b200_update_fixed_radius_ranked_summary_aggregate_batch_graph_3d(
    void* graph, const double* radii, const size_t* k_values, size_t request_count, char* error_out,
    size_t error_size);

RTDL_B200_API void rtdl_b200_destroy_fixed_radius_ranked_summary_aggregate_batch_graph_3d(void* graph);

/* Result record of rtdl_b200_scene_directed_hausdorff_noalloc (device memory).
 * status: 0 = ok, 1 = a coordinate is non-finite or beyond 1e18, 3 = a
 * radix-sort wait of the scene build ran out (the scene is not valid).  The
 * value 2 is not used (the nearest walk is stackless and cannot overflow). */
typedef struct RtdlB200Witness {
  double distance;
  uint32_t source_id, target_id;
  uint32_t status, reserved;
} RtdlB200Witness;

/* Directed Hausdorff on a scene without allocating device memory.  No
 * counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc while they run the query -- an application whose allocator owns
 * the whole device heap, code running inside a larger CUDA graph it does not
 * own, or a real-time loop where an allocation could stall.  Inputs and
 * outputs are device pointers the caller owns: query_points_dev (RtdlPoint or
 * RtdlPoint3D records matching the scene's dimension), the optional per-query
 * nearest_distance_dev / nearest_id_dev arrays (query input order) and
 * witness_dev.  The work is enqueued on `stream` (NULL = the legacy default
 * stream) and the call returns without waiting; read witness_dev->status after
 * the stream has finished.  All scratch comes from one fixed device array of
 * 9.75 MiB that every GPU loading the library holds until the process exits,
 * which caps query_count at 262,144; larger counts are rejected with an
 * error.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call reuses the same array, so calls that overlap on the GPU (on
 * different streams, or from different threads) race and must be serialized
 * by the caller.  Results equal rtdl_b200_scene_directed_hausdorff. */
RTDL_B200_API int rtdl_b200_scene_directed_hausdorff_noalloc(
    void* scene, const void* query_points_dev, size_t query_count,
    double* nearest_distance_dev, uint32_t* nearest_id_dev, RtdlB200Witness* witness_dev,
    void* stream, char* error_out, size_t error_size);

/* Phase timings of the last call on this thread, in milliseconds (device
 * events).  Mirrors rtdl_optix_fixed_radius_neighbors_3d_get_last_phase_timings
 * (src/rtdsl/optix_runtime.py:4916, 5029-5106).  Fills up to `capacity`
 * (name, value) pairs; returns the number of phases. */
RTDL_B200_API int rtdl_b200_get_last_phase_timings(const char** names_out, double* values_ms_out, int capacity);

/* Traversal counters of this thread's last query, recorded only when the
 * environment variable RTDL_B200_STATS is set at load time: nodes visited,
 * leaf points tested, in-radius candidates, list inserts, list shifts, FP64
 * band re-decisions, largest leaf-point count of one query.  Returns the
 * number of counters. */
RTDL_B200_API int rtdl_b200_get_last_query_stats(unsigned long long* values_out, int capacity);

/* Number of kernels this library has launched in the process so far (all
 * devices).  Benchmarks read it before and after a timed region. */
RTDL_B200_API int rtdl_b200_get_launch_count(unsigned long long* count_out);

/* Tuning knobs; the autotuner sets these.  leaf_size: points per LBVH leaf
 * bucket (1..32, applies to scenes built afterwards; 0, the default: 32);
 * block_threads: 64, 128
 * or 256; traversal: 0 = one warp walks the tree for 32 neighbouring queries
 * (packet), 1 = one thread per query, 2 = packet with the query's bounding
 * cube tested at internal nodes, 3 = packet whose leaf buckets are tested
 * point-major (a lane per point, the reaching queries in turn), 4 (the
 * default) = packet choosing lane- or point-major per bucket (point-major when
 * at most half as many of the packet's queries reach it as it holds points).
 * Every setting returns the same rows.  Returns 0 on success. */
RTDL_B200_API int rtdl_b200_set_tuning(int leaf_size, int block_threads, int traversal);

#ifdef __cplusplus
}
#endif

#endif /* RTDL_B200_H */
