// internal.cuh -- shared declarations of librtdl_b200 (device structures,
// launch helpers and the host-side plumbing every translation unit uses).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rtdl_b200.h"

namespace rtdl_b200 {

#define RTDL_CUDA_CHECK(call)                                                          \
  do {                                                                                 \
    cudaError_t _e = (call);                                                           \
    if (_e != cudaSuccess)                                                             \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(_e) + \
                               " at " #call);                                          \
  } while (0)

// Counts kernel launches made by this library (reported by
// rtdl_b200_get_launch_count) and checks the launch status right after the
// launch.  Every entry point clears the thread's last runtime error before it
// starts and every cleanup call consumes its own, so an error reported here
// belongs to the launch at `file:line` (the message names it).
void count_launches(int n);
unsigned long long launches_counted();
void check_launch(int n, const char* file, int line);
#define RTDL_LAUNCHED(n) ::rtdl_b200::check_launch((n), __FILE__, __LINE__)

// A runtime error met while releasing resources (cudaFreeAsync, event
// destruction) is consumed at once, so it cannot surface at an unrelated later
// check, and kept for the entry point, which reports it as the call's error
// when nothing failed before it.
void note_cleanup_error(cudaError_t e, const char* what);
// Synchronizes a stream on an error path or in a destructor: the original
// exception is the one reported, so a failure here is only consumed.
inline void sync_quietly(cudaStream_t s) {
  if (cudaStreamSynchronize(s) != cudaSuccess) cudaGetLastError();
}

constexpr int kSmCount = 148;          // B200: 2 dies x 74 SMs
constexpr int kMaxList = 64;           // per-query list capacity held in shared memory
constexpr int kStackDepth = 64;        // traversal stack; Karras depth <= 30 code bits + 32 index bits
constexpr uint32_t kNone = 0xFFFFFFFFu;

// ---- reductions over an input point set ------------------------------------
// Min/max use an order-preserving uint encoding of the float bits.
struct PointStats {
  unsigned int lo[3];
  unsigned int hi[3];
  unsigned long long max_abs_bits;  // bits of the largest |coordinate| (double)
  unsigned int inexact;             // a coordinate is not exactly representable in FP32
  unsigned int bad;                 // kBadCoordinates | kBadSortWait bits
  unsigned int ids_unsorted;        // ids decrease somewhere in input order
  unsigned int pad;
};
constexpr double kMaxCoordinate = 1.0e18;
constexpr unsigned int kBadCoordinates = 1u;  // non-finite or |coordinate| > kMaxCoordinate
constexpr unsigned int kBadSortWait = 2u;     // a radix-sort look-back wait ran out (the order is not valid)

// Turns a set's bad bits into the call's error.
inline void throw_if_bad(unsigned int bad) {
  if (bad & kBadSortWait) throw std::runtime_error("radix sort look-back wait exceeded its limit");
  if (bad) throw std::runtime_error("point coordinates must be finite with magnitude <= 1e18");
}

__host__ __device__ inline unsigned int float_to_ordered(float f) {
#ifdef __CUDA_ARCH__
  unsigned int b = __float_as_uint(f);
#else
  unsigned int b;
  memcpy(&b, &f, 4);
#endif
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float ordered_to_float(unsigned int o) {
  unsigned int b = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

// ---- a built scene (LBVH over the search points) ---------------------------
// Node layout: the collapsed tree in depth-first pre-order, 2 x float4 = 32 B
// per node, traversed without a stack:
//   n[0] = {lo.xyz, ref}   ref == kInternalNode: an internal node, its left
//                          child is the next record (descend on overlap);
//                          ref < 0: leaf bucket, see leaf_first / leaf_count
//   n[1] = {hi.xyz, rope}  next record when the subtree is done or missed;
//                          kRopeEnd ends the traversal
// The root is record 0.
constexpr int kRopeEnd = -1;
constexpr int kInternalNode = 0;
constexpr uint32_t kMaxScenePoints = 1u << 26;  // leaf references keep 26 bits for the first point
__host__ __device__ inline int leaf_ref(int first, int count) { return ~((first << 5) | (count - 1)); }
__host__ __device__ inline int leaf_first(int hit) { return (~hit) >> 5; }
__host__ __device__ inline int leaf_count(int hit) { return ((~hit) & 31) + 1; }

struct SceneView {
  const float4* pts;      // n sorted points: x, y, z (0 for 2D), w = record id bits
  const uint32_t* perm;   // sorted index -> search input index
  const double* pts64;    // 3 doubles per sorted point (exact coordinates), used when inexact
  const float4* nodes;    // 2 float4 per node, collapsed tree in pre-order
  uint32_t n;
  const unsigned int* inexact;  // device flag: scene coordinates are not all FP32-exact
  const int* prob_root;   // problem batch: pre-order index of each problem's subtree (nullptr: one problem)
};

struct Scene {
  int dim = 3;
  int device = 0;
  uint32_t n = 0;
  double max_radius = 0.0;  // prepared-FRN contract only
  bool device_columns = false;  // built from partner-owned device columns (count-threshold contract)
  int leaf_size = 8;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  float4* pts = nullptr;
  uint32_t* perm = nullptr;
  double* pts64 = nullptr;
  float4* nodes = nullptr;
  uint32_t* codes = nullptr;    // Morton codes of the sorted points (seed nearest searches)
  PointStats* stats = nullptr;  // device copy of the build statistics
  // A batch of independent problems (problems > 0) is built as one tree: the
  // sort key is (problem << code_bits) | Morton code in the problem's own box,
  // so every problem is one subtree; prob_root holds its pre-order index
  // (kRopeEnd for a problem without points) and the subtree ends at that
  // node's rope.
  uint32_t problems = 0;
  int code_bits = 0;
  PointStats* prob_stats = nullptr;  // device, per problem: the box of its Morton codes
  int* prob_root = nullptr;          // device, per problem
  std::vector<unsigned long long> prob_offsets;  // host, problems + 1: input offsets of each problem's points
  SceneView view() const {
    SceneView v;
    v.pts = pts;
    v.perm = perm;
    v.pts64 = pts64;
    v.nodes = nodes;
    v.n = n;
    v.inexact = stats ? &stats->inexact : nullptr;
    v.prob_root = prob_root;
    return v;
  }
};

// ---- tuning ---------------------------------------------------------------
struct Tuning {
  int leaf_size = 0;  // 0: automatic (scene_leaf_size)
  int block_threads = 128;
  int traversal = 4;  // fixed-radius collect: 0 = one warp per 32 queries (packet), 1 = one thread per
                      // query, 2 = packet with cube tests at internal nodes, 3 = packet with
                      // point-major leaf tests, 4 (default) = packet choosing lane- or point-major
                      // per leaf
};
// The tuning a call runs with: a copy of the process-wide setting taken when
// the entry point starts (rtdl_b200_set_tuning from another thread changes the
// next call, never one in progress).
const Tuning& tuning();
void set_tuning(const Tuning& t);
struct TuningScope {  // takes the calling thread's snapshot for one entry point
  TuningScope();
  ~TuningScope();
  bool outer;
};

// ---- phase timing (CUDA events, read after the call's final sync) ----------
struct PhaseTimer {
  cudaStream_t stream;
  std::vector<std::pair<const char*, cudaEvent_t>> marks;
  explicit PhaseTimer(cudaStream_t s);
  ~PhaseTimer();
  void mark(const char* name);
  void publish();  // after a sync: converts to milliseconds for get_last_phase_timings
};

// ---- stream-ordered allocation (pooled: no OS calls after warm-up) --------
void* dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);
void ensure_pool_configured(int device);

// ---- sort / scan (sort_scan.cu) -------------------------------------------
// Exclusive scan of `counts` (optionally gathered through `order`, or identity
// when *identity_flag != 0) into out[0..n] (u64); out[n] is the total.
void scan_counts_u64(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag,
                     uint32_t n, unsigned long long* out, cudaStream_t s);
// The same with a caller-owned workspace of scan_workspace_bytes(n) bytes (no
// allocation: usable inside stream capture).
size_t scan_workspace_bytes(uint32_t n);
void scan_counts_u64_ws(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag, uint32_t n,
                        unsigned long long* out, void* workspace, cudaStream_t s);
// Stable LSD radix sort of (key, value) pairs over bits [begin_bit, end_bit),
// 8 bits per pass.  The result is left in keys/vals.  When *skip_flag != 0
// (device memory) every pass returns immediately and the input stays in place.
// A look-back wait that runs out sets kBadSortWait in *wait_error (the sorted
// set's PointStats::bad), which the caller's input check turns into an error.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, int begin_bit, int end_bit,
                      const unsigned int* skip_flag, unsigned int* wait_error, cudaStream_t s);
void iota_u32(uint32_t* out, uint32_t n, cudaStream_t s);

// ---- scene build (lbvh.cu) -------------------------------------------------
// `points` is a device AoS of RtdlPoint (dim 2) or RtdlPoint3D (dim 3).
Scene* build_scene(const void* points_dev, uint32_t n, int dim, cudaStream_t s, int leaf_size);
// Problem batch: points_dev holds the problems' points back to back, problem
// p at [offsets[p], offsets[p + 1]) (host array of problems + 1 entries).
Scene* build_scene_batch(const void* points_dev, const unsigned long long* offsets, uint32_t problems, int dim,
                         cudaStream_t s, int leaf_size);
// Bits of the problem id in a batch's sort keys, and the Morton bits below it.
int batch_problem_bits(uint32_t problems);
int batch_code_bits(uint32_t problems, int dim);
// Per-point problem ids and per-problem boxes for points laid out by offsets_dev
// (problems + 1 entries), then composite codes (p << code_bits) | Morton.
void batch_problem_ids(const unsigned long long* offsets_dev, uint32_t problems, uint32_t n, uint32_t* pid,
                       cudaStream_t s);
void batch_boxes(const float4* pts, const uint32_t* pid, uint32_t n, PointStats* prob_stats, uint32_t problems,
                 cudaStream_t s);
void batch_codes(const float4* pts, const uint32_t* pid, uint32_t n, int dim, const PointStats* prob_stats,
                 int stats_stride, int code_bits, uint32_t* codes, cudaStream_t s);
void destroy_scene(Scene* sc);
// Converts AoS points to float4 (w = id bits) and accumulates statistics.
void prep_points(const void* points_dev, uint32_t n, int dim, float4* out, PointStats* stats, cudaStream_t s);
void reset_stats(PointStats* stats, cudaStream_t s);
// 32-bit Morton codes relative to the box held in `box_stats` (clamped).
void morton_codes(const float4* pts, uint32_t n, int dim, const PointStats* box_stats, uint32_t* codes,
                  cudaStream_t s);

// ---- queries (query.cu) -----------------------------------------------------
enum Predicate { kFrn = 0, kBounded = 1, kKnn = 2 };

struct QueryResult {
  unsigned long long rows = 0;   // total rows
  unsigned int heavy = 0;        // queries resolved by the generic path
};

// fixed_radius_neighbors over a batch of problems (see build_scene_batch):
// problem p's queries are [qoff[p], qoff[p + 1]) of the query records, with
// its own radius and kmax; rows come out problem by problem, each problem's
// in the order a single query would give.  On a plain scene every problem
// searches the whole scene: several requests against one resident scene
// answered by one launch sequence.
struct BatchSpec {
  uint32_t problems = 0;
  const unsigned long long* qoff = nullptr;  // host, problems + 1
  const double* radius = nullptr;            // host, problems
  const uint32_t* kmax = nullptr;            // host, problems (1..64)
  unsigned long long* row_offsets = nullptr; // host out, problems + 1: first row of each problem, then the total
};
// A query set prepared once for repeated fixed-radius calls: device records,
// FP32 points, Morton processing order (in the set's own box) and output
// order, so a call only computes its bands.
struct PreparedQueries {
  int dim = 3;
  int device = 0;
  uint32_t n = 0;
  cudaStream_t stream = nullptr;
  void* raw = nullptr;            // device copy of the records (owned)
  PointStats* qst = nullptr;
  float4* qpts = nullptr;
  uint32_t* qorder = nullptr;     // processing rank -> input index
  uint32_t* oorder = nullptr;     // output rank -> input index
  uint32_t* qrank = nullptr;      // input index -> output rank
  unsigned int* identity = nullptr;  // device flag: ids ascend (output order == input order)
};
PreparedQueries* prepare_query_set(const void* records_dev, uint32_t n, int dim, cudaStream_t s);
void destroy_query_set(PreparedQueries* pq);
QueryResult run_query_prepared(Scene* sc, const PreparedQueries* pq, double radius, uint32_t kmax, void* rows_dev,
                               size_t rows_capacity, uint8_t* overflow_dev, cudaStream_t s, PhaseTimer* timer);

// fixed_radius_neighbors reduced to per-query ranked summaries (query input
// order, device, optional) and their aggregate (host), without row output to
// the caller.
QueryResult run_ranked_summaries(Scene* sc, const void* queries_dev, uint32_t nq, double radius, uint32_t kmax,
                                 RtdlFixedRadiusRankedNeighborSummary* summaries_dev,
                                 RtdlFixedRadiusRankedNeighborAggregate* aggregate_host, cudaStream_t s,
                                 PhaseTimer* timer, const PreparedQueries* pq = nullptr);
// fixed_radius_count_threshold over a scene: per query (input order) its id,
// its in-radius count (capped at a positive threshold) and whether a positive
// threshold was reached; every output is optional (device buffers, except
// reached_host: the number of queries that reached the threshold).
struct CountOutputs {
  uint32_t* ids = nullptr;
  uint32_t* counts = nullptr;
  uint32_t* flags = nullptr;
  RtdlFixedRadiusCountRow* rows = nullptr;
  unsigned long long* reached_host = nullptr;
};
void run_count_threshold(Scene* sc, const void* queries_dev, uint32_t nq, double radius, uint32_t threshold,
                         const CountOutputs& out, cudaStream_t s);
// Point groups (spans of a search array with their boxes): a scene over every
// group's points, each tagged with its group; a candidate counts when it and its
// group's box are within radius (a point in two groups counts twice).
struct PointGroupScene {
  Scene* sc = nullptr;
  uint32_t* group_of = nullptr;  // device, group of each scene point (scene input order)
  double* boxes = nullptr;       // device, min_x, min_y, max_x, max_y per group
  uint32_t groups = 0, points = 0;
  double max_radius = 0.0;
};
PointGroupScene* point_group_create(const RtdlPoint* points, size_t count, const RtdlPointGroupBounds2D* groups,
                                    size_t group_count, double max_radius, int leaf_size, cudaStream_t s);
void point_group_destroy(PointGroupScene* pg);
void point_group_count(PointGroupScene* pg, const void* queries_dev, uint32_t nq, double radius, uint32_t threshold,
                       const CountOutputs& out, cudaStream_t s);
// One witness row per query (input order) into rows_dev; with max_row_host, also
// the row of largest distance (a query without a witness counts as infinitely far).
void point_group_nearest(PointGroupScene* pg, const void* queries_dev, uint32_t nq, double radius,
                         RtdlFixedRadiusNeighborRow* rows_dev, RtdlFixedRadiusNeighborRow* max_row_host,
                         cudaStream_t s);
// Device id / x / y columns to RtdlPoint records (device).
void columns_to_records_2d(const uint32_t* ids, const double* x, const double* y, uint32_t n, void* out,
                           cudaStream_t s);
// Every query reaches threshold 0 with a count of 0 (the 3-D device-output contract).
void run_count_trivial(const void* queries_dev, uint32_t nq, int dim, const CountOutputs& out, cudaStream_t s);
// Nearest in-radius neighbour of each query, one RtdlFixedRadiusNeighborRow per
// query in input order (neighbor id 0xFFFFFFFF, distance FLT_MAX when none);
// *rows_alloc receives a device buffer of nq rows.
QueryResult run_nearest_witness(Scene* sc, const void* queries_dev, uint32_t nq, double radius, void** rows_alloc,
                                cudaStream_t s, PhaseTimer* timer);

// The plain per-call form: builds the scene of the search records and answers
// the query records (device, or host when query_host is set: uploaded inside).
// fixed_radius_neighbors / bounded_knn_rows with k_max <= 64 prepare the query
// set (statistics, own-box Morton order, output order) on `aux` while the scene
// builds on `s`; the coordinates of both sets are checked at the query's first
// read-back.  *scene_out and *query_owned (an uploaded copy) are the caller's to
// release on `s` once the rows are used.
struct BuildQueryInputs {
  const void* search_dev;
  uint32_t ns;
  const void* query_dev;   // device records, or
  const void* query_host;  // host records (uploaded on the query side's stream)
  uint32_t nq;
  int dim;
};
// Rows copied to the host while they are written: once the row count is known
// the query takes a host buffer from `alloc` and, for each range of queries in
// output order whose rows are complete, queues the copy of those rows on
// `copy` behind an event on the query's stream, so the copies overlap the
// emission of later ranges.  `copies` counts the copies queued; the caller
// makes its stream wait for `copy` before it uses or releases the rows.
struct RowDownload {
  void* (*alloc)(size_t bytes, bool* pinned) = nullptr;
  void* host_fixed = nullptr;  // instead of `alloc`: the rows go here (pinned memory the caller holds)
  cudaStream_t copy = nullptr;
  void* host = nullptr;
  bool pinned = false;
  int copies = 0;
};
QueryResult run_build_and_query(const BuildQueryInputs& in, int predicate, double radius, uint32_t limit,
                                void* rows_dev, size_t rows_capacity, void** rows_alloc, uint8_t* overflow_dev,
                                cudaStream_t s, cudaStream_t aux, PhaseTimer* timer, Scene** scene_out,
                                void** query_owned, RowDownload* download = nullptr);
// The plain per-call form with rows to host memory, the queries taken in
// `chunks` ranges of their input order so that the copy of each range's rows
// overlaps the query of the next (rows land in host_rows, pinned memory of
// host_capacity_rows rows held by the caller; `copy` carries the copies, and
// work queued on `s` after the call follows them).  Query records are read
// from in.query_host.
QueryResult run_build_and_query_chunked(const BuildQueryInputs& in, int predicate, double radius, uint32_t limit,
                                        cudaStream_t s, cudaStream_t copy, PhaseTimer* timer, Scene** scene_out,
                                        void* host_rows, unsigned long long host_capacity_rows, int chunks);
// Further streams of this thread on the current device: 0 is the query side of
// run_build_and_query and the row copies, 1 the heavy queries' refinement
// beside the emit kernels and the query ranges' preparation one range ahead.
cudaStream_t aux_stream(int which = 0);
// Leaf-bucket size of a scene build: the tuning's when set, else 32, the
// largest a leaf reference holds.  Larger buckets shorten the walks: the
// fixed-radius collect tests a bucket's points with four loads in flight
// (0.69 ms at 32 points, 0.73 at 24, 0.76 at 20 on the clustered 1M x 1M
// sets), and the nearest walks visit a bucket few lanes need a lane per point
// (k = 16 walk 3.44 ms at 32 or 24 points against 3.65 ms at 8, the 4M x 4M
// Hausdorff nearest 1.21 against 1.39 ms).
int scene_leaf_size();

// Ranked-summary aggregates of several (radius, k_max) requests over one
// prepared query set and one plain scene, captured once as a CUDA graph over
// buffers allocated at creation (worst-case sizes) and replayed on the graph's
// own stream.  The captured path is the fixed-radius path without host reads:
// list lengths and refinement counts stay on the device and every pass is
// launched.  A request whose heavy queries do not resolve in the refinement
// passes (the plain call takes its generic path for them) is marked in the
// status words and recomputed by the plain call at replay.
struct SummaryGraph;
SummaryGraph* summary_graph_create(Scene* sc, const PreparedQueries* pq, const double* radii, const uint32_t* kmax,
                                   uint32_t requests);
void summary_graph_update(SummaryGraph* g, const double* radii, const uint32_t* kmax, uint32_t requests);
// Enqueues one replay on the graph's stream (nothing is read back).
void summary_graph_launch(SummaryGraph* g);
// Replays, reads the aggregates back, recomputes marked requests by the plain call.
void summary_graph_replay(SummaryGraph* g, RtdlFixedRadiusRankedNeighborAggregate* out);
const RtdlFixedRadiusRankedNeighborAggregate* summary_graph_device_aggregates(const SummaryGraph* g);
const unsigned int* summary_graph_device_status(const SummaryGraph* g);
cudaStream_t summary_graph_stream(const SummaryGraph* g);
uint32_t summary_graph_requests(const SummaryGraph* g);
uint64_t summary_graph_fallbacks(const SummaryGraph* g);
void summary_graph_destroy(SummaryGraph* g);

// Prepared problem batches answered by one captured CUDA graph (one
// persistent collect launch per batch, rows of all problems problem-major into
// the caller's buffer); see query.cu.
struct BatchGraph;
BatchGraph* batch_graph_create(Scene* const* batches, uint32_t batch_count, const void* queries_dev,
                               const unsigned long long* query_offsets, const double* radius, const uint32_t* kmax,
                               void* rows_dev, unsigned long long rows_capacity);
// Enqueues one replay (the graph runs on its own stream, ordered after `s`'s
// work and before `s`'s later work); nothing is read back.
void batch_graph_launch(BatchGraph* g, cudaStream_t s);
// Replays, reads the per-problem row offsets and status back, and recomputes
// flagged batches by the plain batch call.
void batch_graph_replay(BatchGraph* g, unsigned long long* row_offsets_out, unsigned int* status_out);
uint32_t batch_graph_problems(const BatchGraph* g);
int batch_graph_kernels(const BatchGraph* g);
uint64_t batch_graph_fallbacks(const BatchGraph* g);
void batch_graph_destroy(BatchGraph* g);

QueryResult run_query_batch(Scene* sc, const void* queries_dev, const BatchSpec& bs, void* rows_dev,
                            size_t rows_capacity, void** rows_alloc, uint8_t* overflow_dev, cudaStream_t s,
                            PhaseTimer* timer);

// Runs a neighbor query on a scene.  All buffers are device buffers; rows are
// written as RtdlFixedRadiusNeighborRow (kFrn) or RtdlKnnNeighborRow.  When
// rows_dev is null the rows are only counted.  When rows_alloc is set, a
// device buffer of exactly the row count is allocated into *rows_alloc.
QueryResult run_query(Scene* sc, const void* queries_dev, uint32_t nq, int predicate, double radius,
                      uint32_t limit, void* rows_dev, size_t rows_capacity, void** rows_alloc,
                      uint8_t* overflow_dev, cudaStream_t s, PhaseTimer* timer);

struct HausdorffResult {
  double distance;
  uint32_t source_id, target_id;
};
HausdorffResult run_directed_hausdorff(Scene* sc, const void* queries_dev, uint32_t nq, double* nearest_dist_dev,
                                       uint32_t* nearest_id_dev, cudaStream_t s, PhaseTimer* timer);

// Traversal counters of the last query on this thread (filled only when the
// environment variable RTDL_B200_STATS is set): nodes visited, leaf points
// tested, in-radius candidates, list inserts, list shifts, FP64 band checks,
// max count of one query, queries on the generic path, queries with 65..128
// candidates.
std::vector<unsigned long long>& last_stats();

// Allocation-free directed Hausdorff (scratch in a fixed device array);
// results and status land in witness_dev on stream s.
void run_directed_hausdorff_noalloc(Scene* sc, const void* queries_dev, uint32_t nq, double* nearest_dist_dev,
                                    uint32_t* nearest_id_dev, RtdlB200Witness* witness_dev, cudaStream_t s);

inline unsigned int div_up(unsigned long long a, unsigned long long b) { return (unsigned int)((a + b - 1) / b); }

}  // namespace rtdl_b200
