// query.cu -- fixed-radius / bounded-KNN / KNN rows and the directed
// nearest-distance (Hausdorff) reduction over a built scene.
//
// Semantics (rubaolee/rtdl src/rtdsl/reference.py:349-434, 882-890): a search
// point is a fixed-radius neighbor when the FP64 value ((dx*dx + dy*dy) +
// dz*dz), dx = search - query, is <= radius*radius; neighbors of one query are
// ordered by (sqrt(d2), neighbor_id, search input index) and the first k_max
// (or k) are kept; rows are grouped by query_id in query input order.
//
// How the device reaches that exactly:
//   * Traversal and candidate tests run in FP32 on float4 points.  A candidate
//     is accepted without further work when its FP32 d2 is below lo2, dropped
//     above hi2, and re-decided in FP64 in between.  lo2/hi2 bracket r^2 by a
//     relative band (1e-5) plus, for inputs that are not FP32-exact, an
//     absolute band of 8 * 2^-24 * max|coordinate| (the FP32 rounding of the
//     inputs); see k_bands.
//   * The per-query list keeps the best L candidates in shared memory, one
//     column per lane ([slot][lane], bank-conflict free), sorted by insertion.
//     Two keys whose FP32 values are closer than the same band are compared
//     exactly: FP64 sqrt(d2), then neighbor id, then search input index.
//   * Once a query provably has more than k_max in-radius neighbors (or its
//     KNN list is full), subtrees whose box is definitely beyond the current
//     k-th key are skipped.
//   * Rows are written by a warp per query in output order, computing the FP64
//     distance without fused multiply-adds, so distances are bit-identical to
//     the reference.
//   * Queries needing more than 64 rows with more than 64 candidates (large
//     k_max, or k > 64) go to a generic block-per-query path (gather, bitonic
//     sort in global memory, emit).
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>

#include "internal.cuh"

namespace rtdl_b200 {

namespace {

constexpr float kU = 5.9604644775390625e-08f;  // 2^-24, FP32 unit roundoff
constexpr int kExpandThreads = 256;
constexpr int kHeavyThreads = 256;

struct DevBands {
  float hi2, lo2, box_hi2;
  float rho, e_abs, floor2;
  double r2;
  unsigned int ids_sorted;
  unsigned int any_inexact;
};

// Band constants from the statistics of both point sets.  Error model (FP32
// d2 from FP32-rounded coordinates vs the exact distance d):
//   |d_fp32 - d| <= 3u*d + 3.5u*M (u = 2^-24, M = max |coordinate|; the M
//   term is absent when every coordinate is FP32-exact).
// The bands below are wider: relative 1e-5 and absolute 8u*M.
__device__ DevBands make_bands(const PointStats* scene, const PointStats* queries, double radius, int has_radius) {
  const double M = fmax(__longlong_as_double((long long)scene->max_abs_bits),
                        __longlong_as_double((long long)queries->max_abs_bits));
  const bool inexact = scene->inexact || queries->inexact;
  const double u = 5.9604644775390625e-08;
  const double e_abs = inexact ? 8.0 * u * M : 0.0;
  const double rho = 1.0e-5;
  DevBands b;
  b.rho = (float)rho;
  b.e_abs = __double2float_ru(e_abs);
  b.floor2 = 1.0e-30f;
  b.any_inexact = inexact ? 1u : 0u;
  b.ids_sorted = queries->ids_unsorted ? 0u : 1u;
  if (has_radius) {
    const double r_hi = radius * (1.0 + rho) + e_abs + 1.0e-18;
    const double r_lo = radius * (1.0 - rho) - e_abs;
    float hi2 = __double2float_ru(r_hi * r_hi);
    if (hi2 < b.floor2) hi2 = b.floor2;
    b.hi2 = hi2;
    b.lo2 = r_lo > 0.0 ? __double2float_rd(r_lo * r_lo) : 0.0f;
    b.box_hi2 = __double2float_ru((double)hi2 * (1.0 + 1.0e-6));
    b.r2 = radius * radius;
  } else {
    b.hi2 = INFINITY;
    b.lo2 = INFINITY;
    b.box_hi2 = INFINITY;
    b.r2 = INFINITY;
  }
  return b;
}

__global__ void k_bands(const PointStats* scene, const PointStats* queries, double radius, int has_radius,
                        DevBands* out) {
  if (threadIdx.x == 0) *out = make_bands(scene, queries, radius, has_radius);
}

// Problem batch: bands per problem (the statistics are the whole batch's, which
// only widens the bands); ids_sorted from the batch's per-problem check.
__global__ void k_bands_batch(const PointStats* scene, const PointStats* queries, const double* radius, uint32_t m,
                              const unsigned int* ids_sorted, DevBands* out) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
    DevBands b = make_bands(scene, queries, radius[p], 1);
    b.ids_sorted = *ids_sorted;
    out[p] = b;
  }
}

struct Ctx {
  float qx, qy, qz;
  double ex, ey, ez;  // exact query coordinates
  const float4* pts;
  const double* pts64;
  const uint32_t* perm;
  int scene_inexact;
  float rho, e_abs, floor2;
};

__device__ __forceinline__ double exact_d2(const Ctx& c, uint32_t i) {
  double sx, sy, sz;
  if (c.scene_inexact) {
    const double* p = c.pts64 + 3ull * i;
    sx = p[0];
    sy = p[1];
    sz = p[2];
  } else {
    const float4 p = __ldg(&c.pts[i]);
    sx = p.x;
    sy = p.y;
    sz = p.z;
  }
  const double dx = __dsub_rn(sx, c.ex), dy = __dsub_rn(sy, c.ey), dz = __dsub_rn(sz, c.ez);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ float key_tol(const Ctx& c, float m) {
  float t = c.rho * m + c.floor2;
  if (c.e_abs > 0.f) t += 2.f * sqrtf(m) * c.e_abs + c.e_abs * c.e_abs;
  return t;
}

__device__ __forceinline__ double exact_d2_at(double ex, double ey, double ez, const float4* pts, const double* pts64,
                                              int inexact, uint32_t i) {
  double sx, sy, sz;
  if (inexact) {
    const double* p = pts64 + 3ull * i;
    sx = p[0];
    sy = p[1];
    sz = p[2];
  } else {
    const float4 p = __ldg(&pts[i]);
    sx = p.x;
    sy = p.y;
    sz = p.z;
  }
  const double dx = __dsub_rn(sx, ex), dy = __dsub_rn(sy, ey), dz = __dsub_rn(sz, ez);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Exact comparison of two candidates by the reference's sort key.  Out of
// line and with scalar arguments, so the caller's query context stays in
// registers.
__device__ __noinline__ bool exact_before(double ex, double ey, double ez, const float4* pts, const double* pts64,
                                          const uint32_t* perm, int inexact, uint32_t ia, uint32_t ib) {
  const double da = __dsqrt_rn(exact_d2_at(ex, ey, ez, pts, pts64, inexact, ia));
  const double db = __dsqrt_rn(exact_d2_at(ex, ey, ez, pts, pts64, inexact, ib));
  if (da != db) return da < db;
  const uint32_t na = __float_as_uint(__ldg(&pts[ia].w)), nb = __float_as_uint(__ldg(&pts[ib].w));
  if (na != nb) return na < nb;
  return __ldg(&perm[ia]) < __ldg(&perm[ib]);
}

// True when candidate a orders strictly before candidate b.  FP32 keys decide
// whenever they are further apart than the error band; otherwise FP64 does.
__device__ __forceinline__ bool before(const Ctx& c, float ka, uint32_t ia, float kb, uint32_t ib) {
  const float d = kb - ka;
  const float t = key_tol(c, fmaxf(ka, kb));
  if (d > t) return true;
  if (-d > t) return false;
  return exact_before(c.ex, c.ey, c.ez, c.pts, c.pts64, c.perm, c.scene_inexact, ia, ib);
}

// Every point in a box whose FP32 key lower bound is kbox orders after the
// candidate with key klast.
__device__ __forceinline__ bool box_beyond(const Ctx& c, float kbox, float klast) {
  const float k = kbox * (1.f - 8.f * kU);
  return (k - klast) > key_tol(c, k);
}

__device__ __forceinline__ float box_d2(float qx, float qy, float qz, const float4& lo, const float4& hi) {
  const float dx = fmaxf(fmaxf(lo.x - qx, qx - hi.x), 0.f);
  const float dy = fmaxf(fmaxf(lo.y - qy, qy - hi.y), 0.f);
  const float dz = fmaxf(fmaxf(lo.z - qz, qz - hi.z), 0.f);
  return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

struct Pass1Params {
  SceneView S;
  const float4* qpts;
  const double* qraw;
  int qstride;
  const uint32_t* qorder;
  uint32_t nq;
  uint32_t kmax;
  int L;
  const DevBands* bands;
  uint32_t* temp;
  uint32_t* counts;
  uint8_t* flags;
  uint32_t* heavy_list;
  uint32_t* heavy_m;
  unsigned int* heavy_count;
  unsigned int* error;
  unsigned long long* stats;  // kStatCount counters, only with STATS
  const uint32_t* qcodes;     // KNN: query Morton codes in processing order (seeds the list)
  const uint32_t* scodes;     // KNN: the scene's sorted Morton codes
};

// Traversal counters gathered by the STATS instantiation (diagnostics).
enum Stat { kStatNodes, kStatLeafPoints, kStatInRadius, kStatInserts, kStatShifts, kStatBand, kStatMaxLeafPoints,
            kStatGenericQueries, kStatLargeQueries, kStatLeafPairs, kStatEmitFixups, kStatRefined, kStatCount };

// One thread per query, queries in Morton order so a warp walks neighbouring
// subtrees.  KNN == false: radius-limited (fixed_radius_neighbors and
// bounded_knn_rows); KNN == true: k nearest.  Every lane keeps its own list.
// WALK: kWalkLane -- each lane walks the rope-linked records alone;
// kWalkRope -- the warp walks them together in pre-order, entering a node
// when any lane's current k-th bound reaches it; kWalkNear -- the warp walks
// nearer child first with a stack (fewer nodes for longer lists, a dearer
// step: 14% faster than kWalkRope at k = 16, 10% slower at k = 1 on the
// benchmark's clustered 1M x 1M sets).  In the packet forms each lane tests a
// leaf only when its own bound reaches it, so lists and rows are the
// per-lane walk's.
constexpr int kWalkLane = 0, kWalkRope = 1, kWalkNear = 2;
// Half-width of the Morton window that seeds a nearest list of length L
// before its walk (2w points, inserted by every lane at once): a wider window
// tightens the k-th bound the divergent walk starts from, at the cost of the
// window's own tests.  Measured on the clustered 1M x 1M sets (packets in
// Morton order): k = 16 walk 3.69 / 3.69 / 3.71 / 3.84 ms at w = 2L / 3L /
// 4L / 6L; k = 1 0.82 / 0.79 / 0.82 / 0.90 ms at w = 8 / 16 / 32 / 64 (the
// 4M x 4M uniform 2D Hausdorff nearest: 1.48 / 1.52 / 1.68 / 2.08 ms).
__host__ __device__ constexpr int seed_half_width(int L) { return L * 2 < 16 ? 16 : L * 2; }
// Lists at least this long take kWalkNear (k = 4: 1.40 ms pre-order against
// 1.46 ms nearer first).
constexpr int kNearFirstMinList = 5;
// A leaf at most this many lanes need is visited point-major (visit_leaf_pm).
// With 24-point buckets: k = 1 walk 0.56 ms with 8 (0.60 with 4), the 4M x 4M
// Hausdorff nearest 1.21 ms (1.23), k = 16 3.44 ms with 4 (3.48 with 2); with
// 8-point buckets lane-major visits of every leaf took 0.79, 1.52 and 3.69 ms.
__host__ __device__ constexpr int point_major_max(int L) { return L <= 4 ? 8 : 4; }
// Held to 64 registers (32 resident warps at 128 threads per block): the
// k = 16 walk ran 2.8% faster than at its natural 72 (28 warps); at 48
// registers the spills cost more than the occupancy gained.
template <bool KNN, bool STATS, int WALK = kWalkLane>
__global__ void __launch_bounds__(256, 4) k_pass1(Pass1Params P) {
  extern __shared__ uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int L = P.L;
  uint32_t* lkey = smem + (size_t)warp * 64 * L;
  uint32_t* lidx = lkey + 32 * L;
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  constexpr bool PACKET = WALK != kWalkLane;
  if (PACKET ? !__any_sync(0xffffffffu, t0 < P.nq) : t0 >= P.nq) return;
  const bool active = t0 < P.nq;  // PACKET: lanes past the end take part in the warp's walk only
  const uint32_t t = active ? t0 : P.nq - 1;
  const uint32_t qin = P.qorder[t];
  const float4 q = P.qpts[qin];
  const DevBands B = *P.bands;
  const SceneView& S = P.S;
  Ctx c;
  c.qx = q.x;
  c.qy = q.y;
  c.qz = q.z;
  {
    const double* r = P.qraw + (size_t)qin * P.qstride;
    c.ex = r[1];
    c.ey = r[2];
    c.ez = P.qstride == 4 ? r[3] : 0.0;
  }
  c.pts = S.pts;
  c.pts64 = S.pts64;
  c.perm = S.perm;
  c.scene_inexact = *S.inexact;
  c.rho = B.rho;
  c.e_abs = B.e_abs;
  c.floor2 = B.floor2;

  const uint32_t kmax = P.kmax;
  uint32_t count = 0;
  int len = 0;
  bool heavy = false;
  bool prune = false;  // the list is complete: only candidates ordering before its last entry matter
  float klast = INFINITY;
  uint32_t ilast = kNone;
  unsigned long long st_nodes = 0, st_points = 0, st_inserts = 0, st_shifts = 0, st_band = 0;
  int win_lo = 0, win_hi = 0;  // seeded window (already in the list)

  auto insert = [&](float key, uint32_t idx) {
    int pos;
    if (len < L) {
      pos = len++;
    } else {
      pos = L - 1;
    }
    while (pos > 0) {
      const float pk = __uint_as_float(lkey[(pos - 1) * 32 + lane]);
      const uint32_t pi = lidx[(pos - 1) * 32 + lane];
      if (!before(c, key, idx, pk, pi)) break;
      lkey[pos * 32 + lane] = __float_as_uint(pk);
      lidx[pos * 32 + lane] = pi;
      --pos;
      if (STATS) ++st_shifts;
    }
    if (STATS) ++st_inserts;
    lkey[pos * 32 + lane] = __float_as_uint(key);
    lidx[pos * 32 + lane] = idx;
    if (len == L) {
      klast = __uint_as_float(lkey[(L - 1) * 32 + lane]);
      ilast = lidx[(L - 1) * 32 + lane];
    }
  };

  auto visit_leaf = [&](int first, int cnt) {
    if (STATS) st_points += cnt;
    for (int i = first; i < first + cnt; ++i) {
      if (KNN && i >= win_lo && i < win_hi) continue;
      const float4 p = __ldg(&S.pts[i]);
      const float dx = p.x - c.qx, dy = p.y - c.qy, dz = p.z - c.qz;
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      if (!KNN) {
        if (d2 > B.hi2) continue;
        if (prune && !before(c, d2, (uint32_t)i, klast, ilast)) continue;
        if (d2 >= B.lo2) {
          if (STATS) ++st_band;
          if (exact_d2(c, (uint32_t)i) > B.r2) continue;
        }
        ++count;
        if (heavy) continue;
        if (len < L) {
          insert(d2, (uint32_t)i);
        } else if ((uint32_t)L == kmax) {
          // more than k_max neighbors: keep the k_max nearest, then prune
          prune = true;
          if (before(c, d2, (uint32_t)i, klast, ilast)) insert(d2, (uint32_t)i);
        } else {
          heavy = true;  // needs more rows than the shared-memory list holds
        }
      } else {
        if (len == L && !before(c, d2, (uint32_t)i, klast, ilast)) continue;
        insert(d2, (uint32_t)i);
        ++count;
      }
    }
  };

  // Point-major visit of a leaf few lanes need (nearest lists): lane j holds
  // point first + j and the needing lanes are taken in turn; a point passes
  // when it may order before that lane's current last entry (the FP32 side
  // of `before`, a superset of what it accepts), and the owning lane then
  // inserts the passing points one by one, exactly as visit_leaf would.
  auto visit_leaf_pm = [&](int first, int cnt, unsigned int needers) {
    const bool has = lane < cnt;
    const uint32_t pi = (uint32_t)(first + (has ? lane : 0));
    const float4 p = __ldg(&S.pts[pi]);
    while (needers) {
      const int q = __ffs(needers) - 1;
      needers &= needers - 1u;
      const float qx = __shfl_sync(0xffffffffu, c.qx, q), qy = __shfl_sync(0xffffffffu, c.qy, q),
                  qz = __shfl_sync(0xffffffffu, c.qz, q);
      const float kl = __shfl_sync(0xffffffffu, klast, q);
      const bool full_list = __shfl_sync(0xffffffffu, (int)(len == L), q) != 0;
      const int wlo = __shfl_sync(0xffffffffu, win_lo, q), whi = __shfl_sync(0xffffffffu, win_hi, q);
      const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      bool pass = has && !((int)pi >= wlo && (int)pi < whi);
      if (full_list) pass = pass && d2 - kl <= key_tol(c, fmaxf(d2, kl));
      unsigned int passing = __ballot_sync(0xffffffffu, pass);
      if (STATS && lane == q) st_points += cnt;
      while (passing) {
        const int j = __ffs(passing) - 1;
        passing &= passing - 1u;
        const float key = __shfl_sync(0xffffffffu, d2, j);
        if (lane == q) {
          const uint32_t idx = (uint32_t)(first + j);
          if (!(len == L && !before(c, key, idx, klast, ilast))) {
            insert(key, idx);
            ++count;
          }
        }
      }
    }
  };

  auto box_ok = [&](float kb) -> bool {
    if (!KNN && kb > B.box_hi2) return false;
    const bool full = KNN ? (len == L) : prune;
    if (full && box_beyond(c, kb, klast)) return false;
    return true;
  };

  // KNN: seed the list with the scene points around the query's Morton code
  // (a window in the sorted order), so the walk starts with a tight k-th
  // bound; the walk skips the window's points.
  if (KNN && S.n > 0 && P.scodes != nullptr) {
    const uint32_t code = P.qcodes[t];
    uint32_t lo = 0, hi = S.n;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(&P.scodes[mid]) < code) lo = mid + 1;
      else hi = mid;
    }
    const int w = seed_half_width(L);
    int a = (int)lo - w;
    if (a < 0) a = 0;
    int b = a + 2 * w;
    if (b > (int)S.n) {
      b = (int)S.n;
      a = b - 2 * w < 0 ? 0 : b - 2 * w;
    }
    if (L >= kNearFirstMinList) {
      // outward from the query's position (lo, lo - 1, lo + 1, ...): points
      // nearer in the curve tend to be nearer in space, so more inserts land
      // at the list's end instead of shifting it (k = 16: 178 shifts per
      // query instead of 249); the list is the same
      int right = (int)lo < a ? a : (int)lo < b ? (int)lo : b - 1, left = right - 1;
      for (int j = a; j < b; ++j) {
        const bool take_right = right < b && (((j - a) & 1) == 0 || left < a);
        visit_leaf(take_right ? right : left, 1);
        if (take_right) ++right;
        else --left;
      }
    } else {
      visit_leaf(a, b - a);
    }
    win_lo = a;
    win_hi = b;
  }
  // depth-first walk over the pre-order records
  int cur = S.n > 0 ? 0 : kRopeEnd;
  if constexpr (WALK == kWalkRope) {
    while (cur != kRopeEnd) {
      const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
      if (STATS) ++st_nodes;
      const int hit = __float_as_int(a.w);
      const bool need = active && box_ok(box_d2(c.qx, c.qy, c.qz, a, b));
      if (__ballot_sync(0xffffffffu, need)) {
        if (hit >= 0) {
          ++cur;  // internal node: its left child is the next record
          continue;
        }
        const unsigned int nm = __ballot_sync(0xffffffffu, need);
        if (KNN && __popc(nm) <= point_major_max(L)) visit_leaf_pm(leaf_first(hit), leaf_count(hit), nm);
        else if (need) visit_leaf(leaf_first(hit), leaf_count(hit));
      }
      cur = __float_as_int(b.w);
    }
    if (!active) return;
  } else if constexpr (WALK == kWalkNear) {
    // Nearer child first.  A node's two children are tested together, by the
    // lanes that needed the node; the packet enters the child that most of
    // those lanes find nearer and keeps the other, if any lane needs it, on a
    // warp-uniform stack in shared memory.  A kept child is tested again when
    // it comes off the stack, against bounds that have shrunk meanwhile (a
    // child's box lies inside its parent's, so a lane that did not need the
    // parent never needs the child).  The right child of an internal record
    // is its left child's rope; the depth, and so the stack, stays below
    // kStackDepth (30 code bits plus 32 index bits).
    __shared__ int stack_all[256 / 32][kStackDepth];
    int* stack = stack_all[warp];
    int sp = 0;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
    bool need = false;
    if (cur != kRopeEnd) {
      a = __ldg(&S.nodes[0]);
      b = __ldg(&S.nodes[1]);
      if (STATS) ++st_nodes;
      need = active && box_ok(box_d2(c.qx, c.qy, c.qz, a, b));
      if (!__any_sync(0xffffffffu, need)) cur = kRopeEnd;
    }
    // at the loop top (a, b) is cur's record, `need` this lane's test of it,
    // and some lane needs it
    while (cur != kRopeEnd) {
      const int hit = __float_as_int(a.w);
      bool descended = false;
      if (hit < 0) {
        const unsigned int nm = __ballot_sync(0xffffffffu, need);
        if (KNN && __popc(nm) <= point_major_max(L)) visit_leaf_pm(leaf_first(hit), leaf_count(hit), nm);
        else if (need) visit_leaf(leaf_first(hit), leaf_count(hit));
      } else {
        const int left = cur + 1;
        const float4 la = __ldg(&S.nodes[2 * left]), lb = __ldg(&S.nodes[2 * left + 1]);
        const int right = __float_as_int(lb.w);
        const float4 ra = __ldg(&S.nodes[2 * right]), rb = __ldg(&S.nodes[2 * right + 1]);
        if (STATS) st_nodes += 2;
        const float dl = box_d2(c.qx, c.qy, c.qz, la, lb), dr = box_d2(c.qx, c.qy, c.qz, ra, rb);
        const bool nl = need && box_ok(dl), nr = need && box_ok(dr);
        const unsigned int bl = __ballot_sync(0xffffffffu, nl), br = __ballot_sync(0xffffffffu, nr);
        if (bl | br) {
          bool right_first = br != 0;
          if (bl && br) {
            const unsigned int vote_r = __ballot_sync(0xffffffffu, nr && (!nl || dr < dl));
            right_first = 2 * __popc(vote_r) > __popc(bl | br);
            if (sp == kStackDepth) {  // cannot happen for a valid tree; the call reports it
              if (lane == 0) atomicOr(P.error, 8u);
              break;
            }
            if (lane == 0) stack[sp] = right_first ? left : right;
            ++sp;
          }
          cur = right_first ? right : left;
          a = right_first ? ra : la;
          b = right_first ? rb : lb;
          need = right_first ? nr : nl;
          descended = true;
        }
      }
      if (!descended) {  // the next kept node some lane still needs
        cur = kRopeEnd;
        while (sp > 0) {
          __syncwarp();
          const int k = stack[--sp];
          __syncwarp();
          a = __ldg(&S.nodes[2 * k]);
          b = __ldg(&S.nodes[2 * k + 1]);
          if (STATS) ++st_nodes;
          need = active && box_ok(box_d2(c.qx, c.qy, c.qz, a, b));
          if (__any_sync(0xffffffffu, need)) {
            cur = k;
            break;
          }
        }
      }
    }
    if (!active) return;
  } else {
    while (cur != kRopeEnd) {
      const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
      if (STATS) ++st_nodes;
      const int hit = __float_as_int(a.w);
      if (box_ok(box_d2(c.qx, c.qy, c.qz, a, b))) {
        if (hit >= 0) {
          ++cur;  // internal node: its left child is the next record
          continue;
        }
        visit_leaf(leaf_first(hit), leaf_count(hit));
      }
      cur = __float_as_int(b.w);
    }
  }

  if (STATS) {
    atomicAdd(&P.stats[kStatNodes], st_nodes);
    atomicAdd(&P.stats[kStatLeafPoints], st_points);
    atomicAdd(&P.stats[kStatInRadius], (unsigned long long)count);
    atomicAdd(&P.stats[kStatInserts], st_inserts);
    atomicAdd(&P.stats[kStatShifts], st_shifts);
    atomicAdd(&P.stats[kStatBand], st_band);
    atomicMax(&P.stats[kStatMaxLeafPoints], st_points);
  }
  uint8_t fl = 0;
  if (!KNN) {
    P.counts[qin] = count < kmax ? count : kmax;
    if (count > kmax) fl |= 1;
  } else {
    P.counts[qin] = (uint32_t)len;
  }
  if (heavy) {
    fl |= 2;
    const unsigned int h = atomicAdd(P.heavy_count, 1u);
    P.heavy_list[h] = qin;
    P.heavy_m[h] = count;
    P.temp[(size_t)qin * L] = h;
  } else {
    uint32_t* dst = P.temp + (size_t)qin * L;
    for (int j = 0; j < len; ++j) dst[j] = lidx[j * 32 + lane];
  }
  P.flags[qin] = fl;
}

// ---- fixed-radius collect pass ----------------------------------------------
// One thread per query in Morton order.  In-radius candidates are appended
// unsorted to the query's slab (capacity kSlab) as one 8-byte entry each; the
// exact in-radius count is kept, so the overflow flag and the row offsets are
// exact without any per-query list.
constexpr int kSlab = 256;  // candidates kept per query
constexpr unsigned int kStrideBlocks = kSmCount * 8;  // grid of the kernels that stride over device counts

// Candidate slab: query-major, kSlab entries for the query at processing rank
// t starting at t * kSlab.  An entry is (FP32 sort key bits << 32) | sorted
// point index, so a lane appends one candidate with one 8-byte store and a
// warp reads a query's candidates with contiguous loads.
__host__ __device__ __forceinline__ size_t slab_base(uint32_t t) { return (size_t)t * kSlab; }

__device__ __forceinline__ unsigned long long slab_entry(float key, uint32_t i) {
  return ((unsigned long long)__float_as_uint(key) << 32) | i;
}

// Per-query record written by the collect pass at the query's processing rank
// and read by the emit kernels, so they find the query's exact coordinates,
// id and candidate count with one load.
struct QueryInfo {
  double ex, ey, ez;  // exact query coordinates (z = 0 in 2D)
  uint32_t qid;
  uint32_t meta;      // candidate count (<= kSlab), the kQuery* bits and the query's kmax (<= 64)
};
constexpr uint32_t kQueryCountMask = 0xFFFFu;
constexpr uint32_t kQueryGeneric = 1u << 16;   // more than kSlab candidates: generic path
constexpr uint32_t kQueryBig = 1u << 17;       // 65..kSlab candidates, or refined: k_emit_list
constexpr uint32_t kQueryOverflow = 1u << 18;  // more in-radius points than kmax
constexpr int kQueryKmaxShift = 19;            // bits 19..25: kmax
__device__ __forceinline__ int query_kmax(uint32_t meta) { return (int)((meta >> kQueryKmaxShift) & 127u); }

struct CollectParams {
  SceneView S;
  const float4* qpts;
  const double* qraw;
  int qstride;
  const uint32_t* qorder;    // processing rank -> query input index (kNone: padding of a problem batch)
  uint32_t nq;               // processing ranks (a batch pads every problem to whole warps)
  uint32_t kmax;
  const DevBands* bands;     // one per problem (one in all for a single problem)
  const uint32_t* warp_prob; // problem batch: the problem of each warp of processing ranks (nullptr: single)
  const uint32_t* prob_kmax; // problem batch: kmax per problem
  unsigned long long* slab;  // kSlab entries per query, see slab_base()
  uint32_t* counts;          // min(count, kmax), query input order
  QueryInfo* qinfo;          // by processing rank
  uint8_t* flags;            // bit0: count > kmax, bit1: count > kSlab (generic path), bit2: count > 64
  uint32_t* heavy_list;
  uint32_t* heavy_m;
  uint32_t* heavy_t;         // processing rank of each heavy_list entry (optional)
  uint32_t* mid_list;        // processing ranks of the queries with 65..128 candidates (or refined, <= 128)
  uint32_t* big_list;        // processing ranks of the queries with 129..kSlab candidates
  unsigned int* small;       // [0] generic-path query count, [1] error bits, [2] mid_list length,
                             // [3] big_list length, [4] emit fixup queue length
  uint8_t* overflow_out;     // optional: 1 per query (input order) when count > kmax
  unsigned long long* stats;
};

// Per-query state of the collect pass and its accept / finish steps, shared by
// the per-lane and the per-warp (packet) traversals.
struct CollectLane {
  uint32_t t, qin;
  float4 q;
  uint32_t count;
  unsigned long long* out;  // this query's slab entries
  unsigned long long st_nodes, st_points, st_band, st_pairs;
};

// The query's exact coordinates, read when needed (the band's FP64 test and
// the query record) rather than held in registers through the walk.
__device__ __forceinline__ void query_exact(const CollectParams& P, uint32_t qin, double& ex, double& ey,
                                            double& ez) {
  const double* r = P.qraw + (size_t)qin * P.qstride;
  ex = r[1];
  ey = r[2];
  ez = P.qstride == 4 ? r[3] : 0.0;
}

// Tests sorted point i against the lane's query and appends it when it is in
// radius: FP32 decides outside the band, FP64 inside.  The stored key is the
// FP32 d2 for FP32-exact inputs, else the exact FP64 d2 rounded to FP32.
template <bool STATS>
__device__ __forceinline__ void collect_point(const CollectParams& P, const DevBands& B, int scene_inexact,
                                              CollectLane& L, uint32_t i, const float4& p) {
  const float dx = p.x - L.q.x, dy = p.y - L.q.y, dz = p.z - L.q.z;
  float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  if (d2 > B.hi2) return;
  if (d2 >= B.lo2 || B.any_inexact) {
    if (STATS && d2 >= B.lo2) ++L.st_band;
    double ex, ey, ez;
    query_exact(P, L.qin, ex, ey, ez);
    const double e2 = exact_d2_at(ex, ey, ez, P.S.pts, P.S.pts64, scene_inexact, i);
    if (d2 >= B.lo2 && e2 > B.r2) return;
    if (B.any_inexact) d2 = __double2float_rn(e2);
  }
  if (L.count < (uint32_t)kSlab) L.out[L.count] = slab_entry(d2, i);
  ++L.count;
}

template <bool STATS>
__device__ __forceinline__ void collect_finish(const CollectParams& P, const CollectLane& L, uint32_t kmax) {
  if (STATS) {
    atomicAdd(&P.stats[kStatNodes], L.st_nodes);
    atomicAdd(&P.stats[kStatLeafPoints], L.st_points);
    atomicAdd(&P.stats[kStatInRadius], (unsigned long long)L.count);
    atomicAdd(&P.stats[kStatBand], L.st_band);
    atomicAdd(&P.stats[kStatLeafPairs], L.st_pairs);
    atomicMax(&P.stats[kStatMaxLeafPoints], (unsigned long long)L.count);
  }
  const uint32_t count = L.count;
  P.counts[L.qin] = count < kmax ? count : kmax;
  uint8_t fl = count > kmax ? 1 : 0;
  if (count > (uint32_t)kSlab) {
    fl |= 2;
    const unsigned int h = atomicAdd(&P.small[0], 1u);
    P.heavy_list[h] = L.qin;
    P.heavy_m[h] = count;
    if (P.heavy_t) P.heavy_t[h] = L.t;
  } else if (count > 128u) {
    fl |= 4;
    P.big_list[atomicAdd(&P.small[3], 1u)] = L.t;
  } else if (count > 64u) {
    fl |= 4;
    P.mid_list[atomicAdd(&P.small[2], 1u)] = L.t;
  }
  QueryInfo qi;
  query_exact(P, L.qin, qi.ex, qi.ey, qi.ez);
  qi.qid = __float_as_uint(L.q.w);
  qi.meta = (count < (uint32_t)kSlab ? count : (uint32_t)kSlab) | ((fl & 1) ? kQueryOverflow : 0u) |
            ((fl & 2) ? kQueryGeneric : 0u) | ((fl & 4) ? kQueryBig : 0u) | (kmax << kQueryKmaxShift);
  P.qinfo[L.t] = qi;
  P.flags[L.qin] = fl;
  if (P.overflow_out) P.overflow_out[L.qin] = fl & 1;
}

__device__ __forceinline__ void collect_init(const CollectParams& P, uint32_t t, CollectLane& L) {
  L.t = t;
  L.qin = P.qorder[t];
  L.q = P.qpts[L.qin];
  L.count = 0;
  L.out = P.slab + slab_base(t);
  L.st_nodes = L.st_points = L.st_band = L.st_pairs = 0;
}

// Tests the points of leaf bucket [first, first + cnt) against the lane's
// query.  `test` false: the lane only takes part in the (warp-uniform) loads.
// Four point loads are issued before their tests (more loads in flight per
// warp; measured 6% faster at the 32-register budget than one at a time).
template <bool STATS>
__device__ __forceinline__ void collect_leaf(const CollectParams& P, const DevBands& B, int scene_inexact,
                                             CollectLane& L, int first, int cnt, bool test) {
  constexpr int kGroup = 4;
  int i = first;
  const int end = first + cnt;
  for (; i + kGroup <= end; i += kGroup) {
    float4 p[kGroup];
#pragma unroll
    for (int u = 0; u < kGroup; ++u) p[u] = __ldg(&P.S.pts[i + u]);
    if (test) {
#pragma unroll
      for (int u = 0; u < kGroup; ++u) collect_point<STATS>(P, B, scene_inexact, L, (uint32_t)(i + u), p[u]);
    }
  }
  for (; i < end; ++i) {
    const float4 p = __ldg(&P.S.pts[i]);
    if (test) collect_point<STATS>(P, B, scene_inexact, L, (uint32_t)i, p);
  }
}

// Point-major form of collect_leaf for a packet: lane j holds point
// first + j of the bucket (cnt <= 32), and the warp takes the queries whose
// sphere reaches the bucket (`active`, one bit per lane) one at a time: the
// query's coordinates are broadcast, every lane tests its point, and the hits
// go to consecutive entries of that query's slab row (one coalesced store).
// The loop runs once per reaching query instead of once per point, and lanes
// whose query misses the bucket cost nothing.  The decisions are
// collect_point's (FP32 outside the band, FP64 inside); only the order of a
// query's slab entries differs, which the emit's sort does not see.
template <bool STATS>
__device__ __forceinline__ void collect_leaf_pm(const CollectParams& P, const DevBands& B, int scene_inexact,
                                                CollectLane& L, uint32_t t0, int lane, int first, int cnt,
                                                unsigned int active) {
  const bool has = lane < cnt;
  const uint32_t i = (uint32_t)(first + (has ? lane : 0));
  const float4 p = __ldg(&P.S.pts[i]);
  const unsigned int lt_mask = (1u << lane) - 1u;
  if (STATS) {
    L.st_points += cnt;
    if ((active >> lane) & 1u) L.st_pairs += cnt;
  }
  while (active) {
    const int q = __ffs(active) - 1;
    active &= active - 1u;
    const float qx = __shfl_sync(0xffffffffu, L.q.x, q);
    const float qy = __shfl_sync(0xffffffffu, L.q.y, q);
    const float qz = __shfl_sync(0xffffffffu, L.q.z, q);
    const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
    float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    bool hit = has && d2 <= B.hi2;
    const bool check = hit && (d2 >= B.lo2 || B.any_inexact);
    if (__any_sync(0xffffffffu, check)) {
      const uint32_t qin = __shfl_sync(0xffffffffu, L.qin, q);
      if (check) {
        double ex, ey, ez;
        query_exact(P, qin, ex, ey, ez);
        if (STATS && d2 >= B.lo2) ++L.st_band;
        const double e2 = exact_d2_at(ex, ey, ez, P.S.pts, P.S.pts64, scene_inexact, i);
        if (d2 >= B.lo2 && e2 > B.r2)
          hit = false;
        else if (B.any_inexact)
          d2 = __double2float_rn(e2);
      }
    }
    const unsigned int hits = __ballot_sync(0xffffffffu, hit);
    if (hits) {
      const uint32_t c0 = __shfl_sync(0xffffffffu, L.count, q);
      if (hit) {
        const uint32_t pos = c0 + (uint32_t)__popc(hits & lt_mask);
        if (pos < (uint32_t)kSlab) P.slab[slab_base(t0 + (uint32_t)q) + pos] = slab_entry(d2, i);
      }
      if (lane == q) L.count = c0 + (uint32_t)__popc(hits);
    }
  }
}

// One thread per query, queries in Morton order.  Stackless walk over the
// rope-linked nodes, while-while style: a lane advances through internal
// nodes until it stands on an overlapping leaf bucket, then the lanes test
// their buckets together.
template <bool STATS>
__global__ void __launch_bounds__(256) k_collect(CollectParams P) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.nq) return;
  const DevBands B = *P.bands;
  const SceneView& S = P.S;
  const int scene_inexact = *S.inexact;
  CollectLane L;
  collect_init(P, t, L);
  int cur = S.n > 0 ? 0 : kRopeEnd;
  while (cur != kRopeEnd) {
    int first = 0, cnt = 0;
    while (cur != kRopeEnd) {
      const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
      if (STATS) ++L.st_nodes;
      const int hit = __float_as_int(a.w);
      const bool over = box_d2(L.q.x, L.q.y, L.q.z, a, b) <= B.box_hi2;
      if (over && hit >= 0) {
        ++cur;  // internal node: its left child is the next record
        continue;
      }
      cur = __float_as_int(b.w);
      if (over) {
        first = leaf_first(hit);
        cnt = leaf_count(hit);
        break;
      }
    }
    if (STATS) {
      L.st_points += cnt;
      L.st_pairs += cnt;
    }
    collect_leaf<STATS>(P, B, scene_inexact, L, first, cnt, true);
  }
  collect_finish<STATS>(P, L, P.kmax);
}

// One warp per 32 Morton-consecutive queries (packet traversal): the warp
// walks the rope-linked nodes once, entering a node when any lane's query
// sphere overlaps it.  Node and point loads are warp-uniform (one request
// each) and the control flow never diverges; each lane tests leaf points
// against its own query.  CUBE: internal nodes are tested against the
// query's bounding cube (six compares against bounds rounded outward; it
// never rejects a node the sphere test accepts), leaf buckets against the
// sphere.  BATCH: several problems (a problem batch, or several requests on
// one scene): each warp walks its problem's subtree with its problem's bands
// and kmax; kept out of the single-problem instantiation, whose registers it
// would cost.
// LEAF: how a reached leaf bucket is tested -- 0 lane-major (collect_leaf:
// every lane loops over the bucket's points), 1 point-major (collect_leaf_pm:
// the warp loops over the reaching queries), 2 either, chosen per bucket
// (warp-uniform): point-major when at most kHybridRatio reaching queries per
// point, i.e. when few of the packet's spheres reach the bucket.
constexpr int kLeafLaneMajor = 0, kLeafPointMajor = 1, kLeafHybrid = 2;
// The packet walk for processing ranks t & ~31 .. (t & ~31) + 31 (lane t & 31).
template <bool STATS, bool CUBE, bool BATCH, int LEAF>
__device__ __forceinline__ void collect_packet_body(const CollectParams& P, uint32_t t) {
  // a problem batch pads every problem to whole warps, so a warp has one problem
  const uint32_t prob = BATCH ? P.warp_prob[t >> 5] : 0u;
  const bool valid = t < P.nq && (!BATCH || P.qorder[t] != kNone);
  if (BATCH && !valid && t < P.nq) P.qinfo[t] = QueryInfo{0.0, 0.0, 0.0, 0u, 0u};  // padding: nothing to emit
  const DevBands B = P.bands[prob];
  const SceneView& S = P.S;
  const int scene_inexact = *S.inexact;
  CollectLane L;
  if (valid) {
    collect_init(P, t, L);
  } else {
    L.q = make_float4(INFINITY, INFINITY, INFINITY, 0.f);  // never overlaps
    L.count = 0;
    L.out = nullptr;
    L.st_nodes = L.st_points = L.st_band = L.st_pairs = 0;
  }
  float3 clo, chi;  // query cube, CUBE only
  if (CUBE) {
    const float h = sqrtf(B.box_hi2) * (1.0f + 4.0f * kU);  // >= the sphere radius
    clo = make_float3(__fsub_rd(L.q.x, h), __fsub_rd(L.q.y, h), __fsub_rd(L.q.z, h));
    chi = make_float3(__fadd_ru(L.q.x, h), __fadd_ru(L.q.y, h), __fadd_ru(L.q.z, h));
  }
  // the walk covers the problem's subtree: from its root to the root's rope
  int cur = S.n > 0 ? 0 : kRopeEnd, end = kRopeEnd;
  if (BATCH) {
    cur = S.prob_root[prob];
    if (cur != kRopeEnd) end = __float_as_int(__ldg(&S.nodes[2 * cur + 1]).w);
  }
  while (cur != end) {
    const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
    if (STATS) ++L.st_nodes;
    const int hit = __float_as_int(a.w);
    bool over;
    if (CUBE && hit >= 0)
      over = valid && a.x <= chi.x && b.x >= clo.x && a.y <= chi.y && b.y >= clo.y && a.z <= chi.z && b.z >= clo.z;
    else
      over = valid && box_d2(L.q.x, L.q.y, L.q.z, a, b) <= B.box_hi2;
    const unsigned int reach = __ballot_sync(0xffffffffu, over);
    if (reach) {
      if (hit >= 0) {
        ++cur;  // internal node: its left child is the next record
        continue;
      }
      const int first = leaf_first(hit), cnt = leaf_count(hit);
      const bool pm = LEAF == kLeafPointMajor || (LEAF == kLeafHybrid && 2 * __popc(reach) <= cnt);
      if (pm) {
        collect_leaf_pm<STATS>(P, B, scene_inexact, L, t & ~31u, (int)(threadIdx.x & 31), first, cnt, reach);
      } else {
        if (STATS) {
          L.st_points += cnt;
          if (over) L.st_pairs += cnt;
        }
        collect_leaf<STATS>(P, B, scene_inexact, L, first, cnt, over);
      }
    }
    cur = __float_as_int(b.w);
  }
  if (valid) collect_finish<STATS>(P, L, BATCH ? P.prob_kmax[prob] : P.kmax);
}

template <bool STATS, bool CUBE, bool BATCH, int MIN_BLOCKS, int LEAF = kLeafLaneMajor>
__global__ void __launch_bounds__(256, MIN_BLOCKS) k_collect_packet(CollectParams P) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!__any_sync(0xffffffffu, t < P.nq)) return;  // whole warp past the end
  collect_packet_body<STATS, CUBE, BATCH, LEAF>(P, t);
}

// ---- heavy queries: radius refinement -------------------------------------------
// A query with more than kSlab points in radius needs only its kmax (<= 64)
// nearest.  If at least kmax points lie within a smaller radius r', those kmax
// nearest are all among them, so the query is collected again at r' and then
// sorted and emitted like any other query (its rows and counts still refer to
// the original radius: the kmax nearest within r).  r' is chosen from the
// in-radius count (cube-root scaling towards ~2 kmax points) inside a bracket
// [lo, hi] that every pass narrows; queries still unresolved after a few
// passes (for instance many points at one distance) take the generic path.

// The bands of DevBands recomputed for another radius (same formulas; the
// FP32 e_abs is rounded up, which only widens them).
__device__ __forceinline__ DevBands bands_at_radius(const DevBands& base, double radius) {
  DevBands b = base;
  const double rho = (double)base.rho, e_abs = (double)base.e_abs;
  const double r_hi = radius * (1.0 + rho) + e_abs + 1.0e-18;
  const double r_lo = radius * (1.0 - rho) - e_abs;
  float hi2 = __double2float_ru(r_hi * r_hi);
  if (hi2 < b.floor2) hi2 = b.floor2;
  b.hi2 = hi2;
  b.lo2 = r_lo > 0.0 ? __double2float_rd(r_lo * r_lo) : 0.0f;
  b.box_hi2 = __double2float_ru((double)hi2 * (1.0 + 1.0e-6));
  b.r2 = radius * radius;
  return b;
}

struct RefineParams {
  CollectParams C;         // scene, queries, processing order, bands, slab
  const uint32_t* qprob;   // problem of each query (input order); nullptr: one problem
  const uint32_t* work;    // processing ranks to collect again
  const double* rad;       // their radii
  uint32_t nwork;
  uint32_t* cnt;           // out: in-radius count at rad (all of them, not only the kSlab stored)
  // device-driven form (captured graphs): the count is read from *nwork_dev, the
  // packet kernel runs when it is >= packet_min and the warp kernel otherwise,
  // and both stride over the work with whatever grid they were given
  const unsigned int* nwork_dev;
  uint32_t packet_min;
};

__device__ __forceinline__ uint32_t refine_count(const RefineParams& R, bool packet_kernel) {
  if (!R.nwork_dev) return R.nwork;
  const uint32_t n = *R.nwork_dev;
  return (n >= R.packet_min) == packet_kernel ? n : 0u;
}

// One warp per work item: the warp walks the query's subtree once (node
// tests warp-uniform) and its lanes test a leaf bucket's points together,
// appending accepted points with a ballot prefix.  The accept rule is
// collect_point's (FP32 outside the band, FP64 inside).  Heavy queries are few
// and scattered, so a packet of 32 of them would walk the union of 32 regions.
__device__ __forceinline__ void collect_refine_warp(const RefineParams& R, uint32_t j, int lane, int scene_inexact) {
  const CollectParams& P = R.C;
  const SceneView& S = P.S;
  const uint32_t t = R.work[j], qin = P.qorder[t];
  const uint32_t prob = R.qprob ? R.qprob[qin] : 0u;
  const DevBands LB = bands_at_radius(P.bands[prob], R.rad[j]);
  const float4 q = P.qpts[qin];
  const double* rq = P.qraw + (size_t)qin * P.qstride;
  const double ex = rq[1], ey = rq[2], ez = P.qstride == 4 ? rq[3] : 0.0;
  unsigned long long* out = P.slab + slab_base(t);
  int cur = S.n > 0 ? 0 : kRopeEnd, end = kRopeEnd;
  if (S.prob_root) {
    cur = S.prob_root[prob];
    if (cur != kRopeEnd) end = __float_as_int(__ldg(&S.nodes[2 * cur + 1]).w);
  }
  const unsigned int lt = (1u << lane) - 1u;
  uint32_t count = 0;
  while (cur != end) {
    const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
    const int hit = __float_as_int(a.w);
    if (box_d2(q.x, q.y, q.z, a, b) <= LB.box_hi2) {
      if (hit >= 0) {
        ++cur;
        continue;
      }
      const int first = leaf_first(hit), cnt = leaf_count(hit);
      bool acc = false;
      float key = 0.f;
      const uint32_t i = (uint32_t)(first + lane);
      if (lane < cnt) {
        const float4 p = __ldg(&S.pts[i]);
        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
        key = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        acc = key <= LB.hi2;
        if (acc && (key >= LB.lo2 || LB.any_inexact)) {
          const double e2 = exact_d2_at(ex, ey, ez, S.pts, S.pts64, scene_inexact, i);
          if (key >= LB.lo2 && e2 > LB.r2) acc = false;
          if (LB.any_inexact) key = __double2float_rn(e2);
        }
      }
      const unsigned int m = __ballot_sync(0xffffffffu, acc);
      if (acc) {
        const uint32_t pos = count + __popc(m & lt);
        if (pos < (uint32_t)kSlab) out[pos] = slab_entry(key, i);
      }
      count += __popc(m);
    }
    cur = __float_as_int(b.w);
  }
  if (lane == 0) R.cnt[j] = count;
}

__global__ void __launch_bounds__(256) k_collect_refine(RefineParams R) {
  const uint32_t n = refine_count(R, false);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t j = (uint32_t)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (j >= n) return;  // whole warp
  const int scene_inexact = *R.C.S.inexact;
  for (; j < n; j += warps) collect_refine_warp(R, j, threadIdx.x & 31, scene_inexact);
}

// One thread per work item, warp-packet walks (the form for many heavy
// queries, which then cluster in space): the lanes of a warp that share a
// subtree root walk it together (a problem batch can mix roots in a warp).
__device__ __forceinline__ void collect_refine_packet(const RefineParams& R, uint32_t j, bool valid,
                                                      int scene_inexact) {
  const CollectParams& P = R.C;
  const SceneView& S = P.S;
  CollectLane L;
  uint32_t prob = 0;
  DevBands LB = P.bands[0];
  int root = kRopeEnd, end = kRopeEnd;
  if (valid) {
    collect_init(P, R.work[j], L);
    prob = R.qprob ? R.qprob[L.qin] : 0u;
    LB = bands_at_radius(P.bands[prob], R.rad[j]);
    root = S.prob_root ? S.prob_root[prob] : (S.n > 0 ? 0 : kRopeEnd);
    if (root != kRopeEnd) end = __float_as_int(__ldg(&S.nodes[2 * root + 1]).w);
  } else {
    L.q = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    L.count = 0;
    L.out = nullptr;
  }
  bool todo = valid && root != kRopeEnd;
  while (true) {
    const unsigned int pending = __ballot_sync(0xffffffffu, todo);
    if (!pending) break;
    const int leader = __ffs(pending) - 1;
    const int r0 = __shfl_sync(0xffffffffu, root, leader), e0 = __shfl_sync(0xffffffffu, end, leader);
    const bool mine = todo && root == r0;
    int cur = r0;
    while (cur != e0) {
      const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
      const int hit = __float_as_int(a.w);
      const bool over = mine && box_d2(L.q.x, L.q.y, L.q.z, a, b) <= LB.box_hi2;
      if (__any_sync(0xffffffffu, over)) {
        if (hit >= 0) {
          ++cur;
          continue;
        }
        collect_leaf<false>(P, LB, scene_inexact, L, leaf_first(hit), leaf_count(hit), over);
      }
      cur = __float_as_int(b.w);
    }
    todo = todo && !mine;
  }
  if (valid) R.cnt[j] = L.count;
}

// The same walk for one scene without problem subtrees (many heavy queries of a
// plain or prepared scene): no per-lane roots, and close to the collect's occupancy.
__global__ void __launch_bounds__(256, 6) k_collect_refine_packet_scene(RefineParams R) {
  const uint32_t n = refine_count(R, true);
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;  // warp-uniform
  if (base >= n) return;  // whole warp
  const CollectParams& P = R.C;
  const SceneView& S = P.S;
  const int scene_inexact = *S.inexact;
  for (; base < n; base += stride) {
    const uint32_t j = base + (threadIdx.x & 31);
    const bool valid = j < n;
    CollectLane L;
    DevBands LB = P.bands[0];
    if (valid) {
      collect_init(P, R.work[j], L);
      LB = bands_at_radius(P.bands[0], R.rad[j]);
    } else {
      L.q = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
      L.count = 0;
      L.out = nullptr;
    }
    int cur = S.n > 0 ? 0 : kRopeEnd;
    while (cur != kRopeEnd) {
      const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
      const int hit = __float_as_int(a.w);
      const bool over = valid && box_d2(L.q.x, L.q.y, L.q.z, a, b) <= LB.box_hi2;
      if (__any_sync(0xffffffffu, over)) {
        if (hit >= 0) {
          ++cur;
          continue;
        }
        collect_leaf<false>(P, LB, scene_inexact, L, leaf_first(hit), leaf_count(hit), over);
      }
      cur = __float_as_int(b.w);
    }
    if (valid) R.cnt[j] = L.count;
  }
}

__global__ void __launch_bounds__(256) k_collect_refine_packet(RefineParams R) {
  const uint32_t n = refine_count(R, true);
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;  // warp-uniform
  if (base >= n) return;  // whole warp
  const int scene_inexact = *R.C.S.inexact;
  for (; base < n; base += stride) {
    const uint32_t j = base + (threadIdx.x & 31);
    collect_refine_packet(R, j, j < n, scene_inexact);
  }
}

struct RefineUpdate {
  const uint32_t* qorder;
  const uint32_t* qprob;      // nullptr: one problem
  const uint32_t* prob_kmax;  // nullptr: kmax below
  uint32_t kmax;
  QueryInfo* qinfo;
  uint8_t* flags;
  uint32_t* mid_list;
  uint32_t* big_list;
  unsigned int* small;        // [2] mid_list length, [3] big_list length
  // this pass
  const uint32_t* work;
  const double* rad;
  const double* lo;
  const double* hi;
  const uint32_t* full;       // in-radius count at radius frad (at least kmax points)
  const double* frad;         // the original radius, or a smaller tested one that held more than kSlab
  const uint32_t* cnt;
  uint32_t nwork;
  // next pass (or, on the last pass, the generic path's list)
  uint32_t* next_work;
  double* next_rad;
  double* next_lo;
  double* next_hi;
  uint32_t* next_full;
  double* next_frad;
  unsigned int* next_count;
  uint32_t* generic_qin;      // last pass: unresolved queries (input index), their counts at
  uint32_t* generic_m;        // generic_rad: the generic path gathers within that radius
  double* generic_rad;
  int last;
  const unsigned int* nwork_dev;  // non-null: the count is read here (captured graphs)
};

// One work item: resolves it (emit lists), lists it for the generic path (last
// pass), or returns true with its next-pass radius, bracket and bound.
__device__ __forceinline__ bool refine_update_one(const RefineUpdate& U, uint32_t j, uint32_t& t, double& est,
                                                  double& l, double& h, uint32_t& f, double& fr) {
  t = U.work[j];
  const uint32_t qin = U.qorder[t], c = U.cnt[j];
  const uint32_t kmax = U.prob_kmax ? U.prob_kmax[U.qprob ? U.qprob[qin] : 0u] : U.kmax;
  if (c >= kmax && c <= (uint32_t)kSlab) {  // resolved: the slab holds every point within rad
    // A resolved query goes to a list kernel whatever its count (k_emit_list<4>
    // sorts up to 128): k_emit may run while the refinement does, and it skips
    // the query under both the collect's record (generic) and this one (big).
    uint8_t fl = (uint8_t)((U.flags[qin] & ~6u) | (c > 64u ? 4u : 0u));
    U.flags[qin] = fl;
    U.qinfo[t].meta = c | ((fl & 1) ? kQueryOverflow : 0u) | kQueryBig | (kmax << kQueryKmaxShift);
    if (c > 128u)
      U.big_list[atomicAdd(&U.small[3], 1u)] = t;
    else
      U.mid_list[atomicAdd(&U.small[2], 1u)] = t;
    return false;
  }
  // a tested radius with more than kSlab (>= kmax) points in it also holds the
  // kmax nearest; the smallest such radius bounds the generic path's gather
  f = U.full[j];
  fr = U.frad[j];
  if (c > (uint32_t)kSlab && c < f) {
    f = c;
    fr = U.rad[j];
  }
  if (U.last) {
    const unsigned int k = atomicAdd(U.next_count, 1u);
    U.generic_qin[k] = qin;
    U.generic_m[k] = f;
    U.generic_rad[k] = fr;
    return false;
  }
  const double r = U.rad[j];
  l = U.lo[j];
  h = U.hi[j];
  if (c < kmax) l = r; else h = r;
  est = r * cbrt(2.0 * kmax / (double)(c > 0u ? c : 1u));
  if (!(est > l && est < h)) est = 0.5 * (l + h);
  return true;
}

// The next pass's work keeps each warp's items in their order (one atomic per
// warp): items come in processing (Morton) order, so a packet of the next pass
// still walks one region.
__global__ void k_refine_update(RefineUpdate U) {
  const uint32_t n = U.nwork_dev ? *U.nwork_dev : U.nwork;
  const int lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += stride) {  // warp-uniform
    const uint32_t j = base + lane;
    uint32_t t = 0, f = 0;
    double est = 0.0, l = 0.0, h = 0.0, fr = 0.0;
    const bool next = j < n && refine_update_one(U, j, t, est, l, h, f, fr);
    const unsigned int m = __ballot_sync(0xffffffffu, next);
    if (!m) continue;
    unsigned int first = 0;
    if (lane == 0) first = atomicAdd(U.next_count, (unsigned int)__popc(m));
    first = __shfl_sync(0xffffffffu, first, 0);
    if (next) {
      const unsigned int k = first + __popc(m & ((1u << lane) - 1u));
      U.next_work[k] = t;
      U.next_rad[k] = est;
      U.next_lo[k] = l;
      U.next_hi[k] = h;
      U.next_full[k] = f;
      U.next_frad[k] = fr;
    }
  }
}

// The first refinement pass's work: the collect pass's heavy queries (listed
// by input index with their full counts), radius scaled from the full count.
__global__ void k_refine_init(const uint32_t* heavy_qin, const uint32_t* heavy_m, const uint32_t* heavy_t,
                              uint32_t H, const uint32_t* qprob, const double* prob_radius, double radius,
                              const uint32_t* prob_kmax, uint32_t kmax, uint32_t* work, double* rad, double* lo,
                              double* hi, uint32_t* full, double* frad, const unsigned int* H_dev) {
  if (H_dev) H = *H_dev;  // captured graphs: the collect pass's heavy count
  for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < H; h += gridDim.x * blockDim.x) {
    const uint32_t qin = heavy_qin[h], p = qprob ? qprob[qin] : 0u;
    const uint32_t m = heavy_m[h];
    work[h] = heavy_t[h];
    const double r = prob_radius ? prob_radius[p] : radius;
    const uint32_t k = prob_kmax ? prob_kmax[p] : kmax;
    rad[h] = r * cbrt(2.0 * k / (double)m);
    hi[h] = r;
    frad[h] = r;
    lo[h] = 0.0;
    full[h] = m;
  }
}


// ---- emit: warp per query -----------------------------------------------------
// Emitted row writer.
struct RowSink {
  void* rows;
  unsigned long long capacity;
  int ranked;
  __device__ __forceinline__ void put(unsigned long long row, uint32_t qid, uint32_t nid, double dist,
                                      uint32_t rank) const {
    if (row >= capacity) return;
    const unsigned long long db = (unsigned long long)__double_as_longlong(dist);
    if (!ranked) {
      reinterpret_cast<uint4*>(rows)[row] = make_uint4(qid, nid, (uint32_t)db, (uint32_t)(db >> 32));
    } else {
      uint2* out = reinterpret_cast<uint2*>(static_cast<char*>(rows) + row * 24);
      out[0] = make_uint2(qid, nid);
      out[1] = make_uint2((uint32_t)db, (uint32_t)(db >> 32));
      out[2] = make_uint2(rank, 0u);
    }
  }
};

struct EmitParams {
  SceneView S;
  uint32_t nq;
  unsigned long long* slab;
  const QueryInfo* qinfo;     // by processing rank
  const unsigned long long* poff;  // first row of each query, by processing rank
  RowSink sink;
  uint32_t* fix_list;         // processing ranks queued for k_emit_fixup
  unsigned int* fix_count;
  // Emission of one range [out_lo, out_hi) of output ranks (rows copied to the
  // host range by range): k_emit takes the range's queries through `order`
  // (output rank -> processing rank), k_emit_list the range's part
  // [list_start[range], list_start[range + 1]) of its list partitioned by
  // range, and the fix-up the queue from `*fix_begin`.  All null: every
  // query at once.
  const uint32_t* order = nullptr;
  const unsigned int* list_start = nullptr;
  const unsigned int* fix_begin = nullptr;
  uint32_t out_lo = 0, out_hi = 0;
  int range = 0;
};

// A deferred query's sorted packed keys live in slab entries its candidates do
// not use: from entry 64 for at most 64 candidates, from entry 128 for at most
// 128 (room for 256 keys).
__device__ __forceinline__ uint32_t* deferred_keys(unsigned long long* slab, uint32_t t, int n) {
  return reinterpret_cast<uint32_t*>(slab + slab_base(t) + (n <= 64 ? 64 : 128));
}

// Packed sort element: the FP32 d2 key with its low SHIFT mantissa bits
// replaced by the slab slot.  Valid keys are below 0x80000000, so the padding
// value 0xFFFFFFFF sorts last.  Two elements whose truncated keys differ by two
// units or more are in exact order (the FP32 keys are within a few ulps of
// the exact FP64 d2, far less than 2^SHIFT ulps); closer pairs are re-decided
// exactly.
template <int SHIFT>
__device__ __forceinline__ uint32_t pack_key(uint32_t key_bits, uint32_t slot) {
  return (key_bits & ~((1u << SHIFT) - 1u)) | slot;
}

// Bitonic sort across the warp of 32 * E packed elements in a striped layout
// (element i = r * 32 + lane): exchanges at distance >= 32 stay in a lane's
// registers, shorter ones take one shuffle per register.  Ascending.
template <int E>
__device__ __forceinline__ void warp_bitonic_striped(uint32_t (&v)[E], int lane) {
#pragma unroll
  for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int rj = j >> 5;
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const int pr = r ^ rj;
          if (pr > r) {
            const bool up = (((r << 5) | lane) & k) == 0;
            const uint32_t a = v[r], b = v[pr];
            v[r] = up ? min(a, b) : max(a, b);
            v[pr] = up ? max(a, b) : min(a, b);
          }
        }
      } else {
        const bool lower = (lane & j) == 0;
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const bool up = (((r << 5) | lane) & k) == 0;
          const uint32_t other = __shfl_xor_sync(0xffffffffu, v[r], j);
          v[r] = (lower == up) ? min(v[r], other) : max(v[r], other);
        }
      }
    }
  }
}

// Odd-even transposition over a warp's sorted buffer, one thread, restricted
// to neighbours whose truncated keys differ by at most one unit, until no swap
// happens (bounded by n passes).  Runs only when such a pair exists.
__device__ __noinline__ void exact_fixup_sorted(uint32_t* buf, int n, int shift, const unsigned long long* ent,
                                                SceneView S, int inexact, double ex, double ey, double ez) {
  const uint32_t mask = (1u << shift) - 1u;
  for (int pass = 0; pass < n; ++pass) {
    bool changed = false;
    for (int parity = 0; parity < 2; ++parity) {
      for (int i = parity; i + 1 < n; i += 2) {
        const uint32_t a = buf[i], b = buf[i + 1];
        if ((b >> shift) - (a >> shift) > 1u) continue;
        if (exact_before(ex, ey, ez, S.pts, S.pts64, S.perm, inexact, (uint32_t)ent[b & mask],
                         (uint32_t)ent[a & mask])) {
          buf[i] = b;
          buf[i + 1] = a;
          changed = true;
        }
      }
    }
    if (!changed) break;
  }
}

// Only the first kk of a query's n sorted candidates become rows.  An element
// whose truncated key is two units or more above that of element kk - 1
// orders after every element up to kk - 1 exactly as well, so the exact
// re-decision of near ties only has to cover the first m elements: those
// within one unit of element kk - 1 or below it (m = n when kk = n).  `v`
// holds the warp-sorted packed keys in the striped layout (padding
// 0xFFFFFFFF); every lane returns the same m.
template <int E, int SHIFT>
__device__ __forceinline__ int exact_window(const uint32_t (&v)[E], int n, int kk, int lane) {
  if (kk >= n) return n;
  const int c = kk - 1;
  uint32_t vc = v[0];
#pragma unroll
  for (int r = 1; r < E; ++r)
    if ((c >> 5) == r) vc = v[r];
  const uint32_t limit = (__shfl_sync(0xffffffffu, vc, c & 31) >> SHIFT) + 1u;
  int m = 0;
#pragma unroll
  for (int r = 0; r < E; ++r) m += __popc(__ballot_sync(0xffffffffu, v[r] != 0xFFFFFFFFu && (v[r] >> SHIFT) <= limit));
  return m;
}

// The window of exact_window for keys sorted in a shared-memory buffer (k_emit_fixup).
__device__ __forceinline__ int exact_window_sorted(const uint32_t* keys, int n, int kk, int shift) {
  if (kk >= n) return n;
  const uint32_t limit = (keys[kk - 1] >> shift) + 1u;
  int m = kk;
  while (m < n && (keys[m] >> shift) <= limit) ++m;
  return m;
}

// What a warp needs of one query before it sorts: three independent loads
// (the query's record, its first row and slab entry `lane`), so a query costs
// one memory round trip before the sort and one (the point gather) after it.
struct EmitQuery {
  QueryInfo qi;
  unsigned long long base;  // first row of the query
  unsigned long long e0;    // slab entry `lane` (read before the count is known; unused beyond it)
};

__device__ __forceinline__ void emit_load(const EmitParams& P, uint32_t t, int lane, EmitQuery& q) {
  q.qi = P.qinfo[t];
  q.base = P.poff[t];
  q.e0 = P.slab[slab_base(t) + lane];  // inside the query's kSlab entries whatever its count
}

// Sorts the query's n <= 32 * E candidates by the reference's key and writes
// its first min(n, kmax) rows; lane l writes rows l, l + 32, ... so each store
// instruction covers 32 consecutive rows.  When two neighbours need the exact
// comparison, DEFER == false re-decides them here through `wbuf` (shared
// memory); DEFER == true leaves the sorted list in the query's spare slab
// entries and queues the query for k_emit_fixup, which keeps this kernel free
// of the exact comparison's call (and of the registers that call needs).
template <int E, bool DEFER>
__device__ __forceinline__ void emit_query(const EmitParams& P, uint32_t t, const EmitQuery& q, int n, int lane,
                                           uint32_t* wbuf) {
  constexpr int SHIFT = E == 1 ? 5 : E == 2 ? 6 : E == 4 ? 7 : 8;
  constexpr uint32_t kMask = (1u << SHIFT) - 1u;
  const unsigned long long* ent = P.slab + slab_base(t);
  uint32_t v[E], ids[E];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int s = (r << 5) | lane;
    if (s < n) {
      const unsigned long long e = r == 0 ? q.e0 : ent[s];
      v[r] = pack_key<SHIFT>((uint32_t)(e >> 32), (uint32_t)s);
      ids[r] = (uint32_t)e;
    } else {
      v[r] = 0xFFFFFFFFu;
      ids[r] = 0u;
    }
  }
  warp_bitonic_striped<E>(v, lane);
  const int kmax = query_kmax(q.qi.meta);
  const int kk = n < kmax ? n : kmax;
  const int m = exact_window<E, SHIFT>(v, n, kk, lane);
  // ambiguous neighbours inside the window: element i and i + 1 within one truncated unit
  bool amb = false;
#pragma unroll
  for (int r = 0; r < E; ++r) {
    uint32_t nx = __shfl_down_sync(0xffffffffu, v[r], 1);
    const uint32_t wrap = __shfl_sync(0xffffffffu, v[r + 1 < E ? r + 1 : r], 0);
    if (lane == 31) nx = r + 1 < E ? wrap : 0xFFFFFFFFu;
    amb |= ((r << 5) | lane) + 1 < m && (nx >> SHIFT) - (v[r] >> SHIFT) <= 1u;
  }
  const double ex = q.qi.ex, ey = q.qi.ey, ez = q.qi.ez;
  const int inexact = *P.S.inexact;
  if (__any_sync(0xffffffffu, amb)) {
    if constexpr (DEFER) {
      static_assert(E <= 4, "a deferred query needs spare slab entries");
      uint32_t* spare = deferred_keys(P.slab, t, n);
#pragma unroll
      for (int r = 0; r < E; ++r) spare[(r << 5) | lane] = v[r];
      if (lane == 0) P.fix_list[atomicAdd(P.fix_count, 1u)] = t;
      return;
    } else {
#pragma unroll
      for (int r = 0; r < E; ++r) wbuf[(r << 5) | lane] = v[r];
      __syncwarp();
      if (lane == 0) exact_fixup_sorted(wbuf, m, SHIFT, ent, P.S, inexact, ex, ey, ez);
      __syncwarp();
#pragma unroll
      for (int r = 0; r < E; ++r) v[r] = wbuf[(r << 5) | lane];
      __syncwarp();
    }
  }
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = (r << 5) | lane;
    const uint32_t slot = v[r] & kMask;
    uint32_t idx;
    if (E <= 2) {  // the entry of slot s sits in lane s % 32, register s / 32
      idx = __shfl_sync(0xffffffffu, ids[0], slot & 31);
      if (E == 2) {
        const uint32_t hi = __shfl_sync(0xffffffffu, ids[E - 1], slot & 31);
        if (slot >= 32) idx = hi;
      }
    } else {
      idx = i < kk ? (uint32_t)ent[slot] : 0u;
    }
    if (i < kk) {
      const float4 p = __ldg(&P.S.pts[idx]);
      double sx, sy, sz;
      if (inexact) {
        const double* pp = P.S.pts64 + 3ull * idx;
        sx = pp[0];
        sy = pp[1];
        sz = pp[2];
      } else {
        sx = p.x;
        sy = p.y;
        sz = p.z;
      }
      const double dx = __dsub_rn(sx, ex), dy = __dsub_rn(sy, ey), dz = __dsub_rn(sz, ez);
      const double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
      P.sink.put(q.base + i, q.qi.qid, __float_as_uint(p.w), dist, (uint32_t)i + 1);
    }
  }
}

// Warp per query in processing (Morton) order for the queries with at most
// 64 candidates; queries with 65..kSlab candidates are k_emit_list's, those on
// the generic path get their rows from k_expand.
constexpr int kEmitThreads = 256;

// The grid fills the GPU once (emit_grid) and each warp strides over the
// queries: a warp takes its next query as soon as it is done with one,
// instead of short blocks of eight queries retiring and launching.
constexpr int kEmitBlocksPerSm = 8;

__global__ void __launch_bounds__(kEmitThreads, kEmitBlocksPerSm) k_emit(EmitParams P) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (kEmitThreads / 32);
  const uint32_t total = P.order ? P.out_hi - P.out_lo : P.nq;  // P.order: one range of output ranks
  for (uint32_t w = blockIdx.x * (kEmitThreads / 32) + (threadIdx.x >> 5); w < total; w += warps) {
    const uint32_t t = P.order ? P.order[P.out_lo + w] : w;
    EmitQuery q;
    emit_load(P, t, lane, q);
    const uint32_t meta = q.qi.meta;
    const int n = (int)(meta & kQueryCountMask);
    if ((meta & (kQueryGeneric | kQueryBig)) || n == 0) continue;
    if (n <= 32)
      emit_query<1, true>(P, t, q, n, lane, nullptr);
    else
      emit_query<2, true>(P, t, q, n, lane, nullptr);
  }
}

// Blocks of k_emit for `queries` warps of work: one resident wave at most.
inline unsigned int emit_grid(uint64_t queries) {
  const uint64_t blocks = div_up(queries * 32, (uint64_t)kEmitThreads);
  const uint64_t cap = (uint64_t)kSmCount * kEmitBlocksPerSm;
  return (unsigned int)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

// The queries the emit kernels queued, one warp per query: the sorted keys go
// to shared memory, the warp runs odd-even transposition over them (the
// pairs of one parity are disjoint, so the lanes take them in parallel)
// re-deciding neighbours within one truncated unit exactly, until a pass
// swaps nothing; then it writes the rows.  The queue length is read on the
// device, so no host round trip is needed.
constexpr int kFixupThreads = 128;

__global__ void __launch_bounds__(kFixupThreads) k_emit_fixup(EmitParams P) {
  __shared__ uint32_t sk[kFixupThreads / 32][128];
  const unsigned int m = *P.fix_count;
  const unsigned int first = P.fix_begin ? *P.fix_begin : 0u;
  const int lane = threadIdx.x & 31;
  uint32_t* keys = sk[threadIdx.x >> 5];
  const int inexact = *P.S.inexact;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t j = first + (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); j < m; j += warps) {
    const uint32_t t = P.fix_list[j];
    const QueryInfo qi = P.qinfo[t];
    const int n = (int)(qi.meta & kQueryCountMask);  // <= 128 for a deferred query
    const int shift = n <= 32 ? 5 : n <= 64 ? 6 : 7;
    const uint32_t mask = (1u << shift) - 1u;
    const unsigned long long* ent = P.slab + slab_base(t);
    const uint32_t* src = deferred_keys(P.slab, t, n);
    for (int i = lane; i < n; i += 32) keys[i] = src[i];
    __syncwarp();
    const int kmax = query_kmax(qi.meta);
    const int kk = n < kmax ? n : kmax;
    const int w = exact_window_sorted(keys, n, kk, shift);  // the elements the first kk rows can come from
    for (int pass = 0; pass < w; ++pass) {
      bool changed = false;
      for (int parity = 0; parity < 2; ++parity) {
        for (int i = parity + 2 * lane; i + 1 < w; i += 64) {
          const uint32_t a = keys[i], b = keys[i + 1];
          if ((b >> shift) - (a >> shift) > 1u) continue;
          if (exact_before(qi.ex, qi.ey, qi.ez, P.S.pts, P.S.pts64, P.S.perm, inexact, (uint32_t)ent[b & mask],
                           (uint32_t)ent[a & mask])) {
            keys[i] = b;
            keys[i + 1] = a;
            changed = true;
          }
        }
        __syncwarp();
      }
      if (!__any_sync(0xffffffffu, changed)) break;
    }
    const unsigned long long base = P.poff[t];
    for (int i = lane; i < kk; i += 32) {
      const uint32_t idx = (uint32_t)ent[keys[i] & mask];
      const float4 p = __ldg(&P.S.pts[idx]);
      const double dist = __dsqrt_rn(exact_d2_at(qi.ex, qi.ey, qi.ez, P.S.pts, P.S.pts64, inexact, idx));
      P.sink.put(base + i, qi.qid, __float_as_uint(p.w), dist, (uint32_t)i + 1);
    }
    __syncwarp();
  }
}

// ---- ranked summaries ----------------------------------------------------------
// One warp per query in output order reads the query's rows (contiguous) and
// reduces them to the reference's ranked summary: count, first and last row,
// and the distances added one by one in row order (so the sum is the one a
// sequential loop over the rows gives).  Each block also writes its queries'
// partial aggregate (in warp order), which k_summary_final reduces in block
// order: the aggregate is the same on every run.
struct SummaryPartial {
  unsigned long long count, nearest, kth;
  double sum;
};

// ---- nearest in-radius witness (k_max 1, one row per query) -------------------
// offsets[o] = input index of output rank o, offsets[nq] = nq: the emit then
// writes a query's first row at its input position.
__global__ void k_witness_offsets(const uint32_t* oorder, const unsigned int* identity, uint32_t nq,
                                  unsigned long long* offsets) {
  const bool ident = *identity != 0;
  for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o <= nq; o += (uint64_t)gridDim.x * blockDim.x)
    offsets[o] = o == nq ? nq : (ident ? o : oorder[o]);
}

// The row of a query without a neighbour in radius (rtdl_optix_core.cpp:6043-6090:
// neighbor id 0xFFFFFFFF, distance FLT_MAX).
__global__ void k_witness_fill(const float4* qpts, uint32_t nq, RtdlFixedRadiusNeighborRow* rows,
                               unsigned long long capacity) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq && i < capacity;
       i += (uint64_t)gridDim.x * blockDim.x)
    rows[i] = RtdlFixedRadiusNeighborRow{__float_as_uint(qpts[i].w), 0xFFFFFFFFu, 3.4028234663852886e38};
}

// ---- fixed-radius count with a threshold --------------------------------------
// The reference's generic count (generic_primitives.py:198-227): a query's
// in-radius points are counted (radius inclusive, FP64 distances) until the
// threshold is reached; threshold 0 counts them all.  Here the count uses the
// collect's accept rule (FP32 outside the band, FP64 inside) on a packet walk,
// and a lane stops testing once its query reaches the threshold; the walk ends
// when every lane of the warp has.
struct CountParams {
  SceneView S;
  const float4* qpts;
  const double* qraw;
  int qstride;
  const uint32_t* qorder;       // processing rank -> input index
  uint32_t nq;
  const DevBands* bands;
  uint32_t threshold;
  uint32_t* ids_out;            // per query, input order (each optional)
  uint32_t* counts_out;
  uint32_t* flags_out;
  RtdlFixedRadiusCountRow* rows_out;
  unsigned long long* reached;  // optional: queries that reached the threshold
  // point groups (optional): a candidate also needs its group's box within radius
  const uint32_t* group_of;     // group of each scene point (scene input order)
  const double* group_boxes;    // min_x, min_y, max_x, max_y per group
};

// The reference's group test (rtdl_optix_core.cpp:6143-6147) in FP64: the
// squared distance from the query to the group's box, within radius.
__device__ __forceinline__ bool group_box_ok(const CountParams& P, const SceneView& S, uint32_t qin, uint32_t i,
                                             double r2) {
  const double* rq = P.qraw + (size_t)qin * P.qstride;
  const double qx = rq[1], qy = rq[2];
  const double* g = P.group_boxes + 4ull * P.group_of[S.perm[i]];
  const double dx = qx < g[0] ? __dsub_rn(g[0], qx) : (qx > g[2] ? __dsub_rn(qx, g[2]) : 0.0);
  const double dy = qy < g[1] ? __dsub_rn(g[1], qy) : (qy > g[3] ? __dsub_rn(qy, g[3]) : 0.0);
  return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= r2;
}

__global__ void __launch_bounds__(256) k_count_packet(CountParams P) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!__any_sync(0xffffffffu, t < P.nq)) return;  // whole warp past the end
  const bool valid = t < P.nq;
  const DevBands B = *P.bands;
  const SceneView& S = P.S;
  const int scene_inexact = *S.inexact;
  uint32_t qin = 0;
  float4 q = make_float4(INFINITY, INFINITY, INFINITY, 0.f);  // never overlaps
  if (valid) {
    qin = P.qorder[t];
    q = P.qpts[qin];
  }
  const uint32_t thr = P.threshold;
  uint32_t count = 0;
  bool active = valid;
  int cur = S.n > 0 ? 0 : kRopeEnd;
  while (cur != kRopeEnd) {
    const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
    const int hit = __float_as_int(a.w);
    const bool over = active && box_d2(q.x, q.y, q.z, a, b) <= B.box_hi2;
    if (__any_sync(0xffffffffu, over)) {
      if (hit >= 0) {
        ++cur;  // internal node: its left child is the next record
        continue;
      }
      const int first = leaf_first(hit), cnt = leaf_count(hit);
      bool test = over;
      for (int i = first; i < first + cnt; ++i) {
        const float4 p = __ldg(&S.pts[i]);
        if (!test) continue;
        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
        const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        if (d2 > B.hi2) continue;
        if (d2 >= B.lo2) {
          const double* rq = P.qraw + (size_t)qin * P.qstride;
          const double e2 = exact_d2_at(rq[1], rq[2], P.qstride == 4 ? rq[3] : 0.0, S.pts, S.pts64, scene_inexact,
                                        (uint32_t)i);
          if (e2 > B.r2) continue;
        }
        if (P.group_of && !group_box_ok(P, S, qin, (uint32_t)i, B.r2)) continue;
        ++count;
        if (thr != 0u && count >= thr) {
          active = false;
          test = false;
        }
      }
      if (!__any_sync(0xffffffffu, active)) break;  // every query of the warp reached its threshold
    }
    cur = __float_as_int(b.w);
  }
  const bool reached = valid && thr != 0u && count >= thr;
  if (valid) {
    const uint32_t id = __float_as_uint(q.w);
    if (P.ids_out) P.ids_out[qin] = id;
    if (P.counts_out) P.counts_out[qin] = count;
    if (P.flags_out) P.flags_out[qin] = reached ? 1u : 0u;
    if (P.rows_out) P.rows_out[qin] = RtdlFixedRadiusCountRow{id, count, reached ? 1u : 0u};
  }
  if (P.reached) {
    const unsigned int m = __ballot_sync(0xffffffffu, reached);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(P.reached, (unsigned long long)__popc(m));
  }
}

// Point groups: the nearest point within radius whose group box is also within
// radius, by exact FP64 distance then smaller id (rtdl_optix_core.cpp:6215-6306);
// one row per query at its input index, 0xFFFFFFFF / FLT_MAX when none.
__global__ void __launch_bounds__(256) k_group_nearest_packet(CountParams P, RtdlFixedRadiusNeighborRow* rows) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!__any_sync(0xffffffffu, t < P.nq)) return;  // whole warp past the end
  const bool valid = t < P.nq;
  const DevBands B = *P.bands;
  const SceneView& S = P.S;
  const int scene_inexact = *S.inexact;
  uint32_t qin = 0;
  float4 q = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
  if (valid) {
    qin = P.qorder[t];
    q = P.qpts[qin];
  }
  double best = 0.0;
  uint32_t best_id = 0xFFFFFFFFu;
  bool found = false;
  int cur = S.n > 0 ? 0 : kRopeEnd;
  while (cur != kRopeEnd) {
    const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
    const int hit = __float_as_int(a.w);
    const bool over = valid && box_d2(q.x, q.y, q.z, a, b) <= B.box_hi2;
    if (__any_sync(0xffffffffu, over)) {
      if (hit >= 0) {
        ++cur;
        continue;
      }
      const int first = leaf_first(hit), cnt = leaf_count(hit);
      for (int i = first; i < first + cnt; ++i) {
        const float4 p = __ldg(&S.pts[i]);
        if (!over) continue;
        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
        if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) > B.hi2) continue;
        const double* rq = P.qraw + (size_t)qin * P.qstride;
        const double e2 = exact_d2_at(rq[1], rq[2], P.qstride == 4 ? rq[3] : 0.0, S.pts, S.pts64, scene_inexact,
                                      (uint32_t)i);
        if (e2 > B.r2) continue;
        if (P.group_of && !group_box_ok(P, S, qin, (uint32_t)i, B.r2)) continue;
        const uint32_t id = __float_as_uint(p.w);
        if (!found || e2 < best || (e2 == best && id < best_id)) {
          best = e2;
          best_id = id;
          found = true;
        }
      }
    }
    cur = __float_as_int(b.w);
  }
  if (valid)
    rows[qin] = RtdlFixedRadiusNeighborRow{__float_as_uint(q.w), found ? best_id : 0xFFFFFFFFu,
                                           found ? __dsqrt_rn(best) : 3.4028234663852886e38};
}

// The witness row of largest distance, ties to the smaller query id then
// neighbour id; a query without a witness counts as infinitely far
// (rtdl_optix_core.cpp:6310-6358).  One block.
__device__ __forceinline__ bool witness_after(const RtdlFixedRadiusNeighborRow& c, const RtdlFixedRadiusNeighborRow& b) {
  if (c.distance != b.distance) return c.distance > b.distance;
  if (c.query_id != b.query_id) return c.query_id < b.query_id;
  return c.neighbor_id < b.neighbor_id;
}

__global__ void __launch_bounds__(1024) k_witness_max(const RtdlFixedRadiusNeighborRow* rows, uint32_t n,
                                                      RtdlFixedRadiusNeighborRow* out) {
  __shared__ RtdlFixedRadiusNeighborRow sb[1024];
  RtdlFixedRadiusNeighborRow best{0xFFFFFFFFu, 0xFFFFFFFFu, -1.0};
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    RtdlFixedRadiusNeighborRow r = rows[i];
    if (r.neighbor_id == 0xFFFFFFFFu || !isfinite(r.distance)) r.distance = INFINITY;
    if (witness_after(r, best)) best = r;
  }
  sb[threadIdx.x] = best;
  __syncthreads();
  for (unsigned int stride = blockDim.x >> 1; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride && witness_after(sb[threadIdx.x + stride], sb[threadIdx.x]))
      sb[threadIdx.x] = sb[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sb[0];
}

// The 3-D device-output contract with threshold 0 (rtdl_optix_core.cpp:4189-4201):
// every query reaches it with a count of 0, and no walk is needed.
__global__ void k_count_trivial(const float4* qpts, uint32_t nq, uint32_t* ids_out, uint32_t* counts_out,
                                uint32_t* flags_out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    ids_out[i] = __float_as_uint(qpts[i].w);
    counts_out[i] = 0u;
    flags_out[i] = 1u;
  }
}

struct SummarySpec {
  RtdlFixedRadiusRankedNeighborSummary* summaries_dev;  // per query, input order (optional)
  RtdlFixedRadiusRankedNeighborAggregate* aggregate_host;
};


constexpr int kSummaryThreads = 256;

__global__ void __launch_bounds__(kSummaryThreads)
    k_summarize(const RtdlFixedRadiusNeighborRow* rows, const unsigned long long* offsets, const uint32_t* oorder,
                const unsigned int* identity, const float4* qpts, uint32_t nq,
                RtdlFixedRadiusRankedNeighborSummary* summaries, SummaryPartial* partial) {
  __shared__ SummaryPartial wsum[kSummaryThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t j = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  SummaryPartial mine{0ull, 0ull, 0ull, 0.0};
  if (j < nq) {  // warp-uniform
    const uint32_t qin = *identity ? (uint32_t)j : oorder[j];
    const unsigned long long a = offsets[j], b = offsets[j + 1];
    const int cnt = (int)(b - a);  // at most 64
    double d0 = 0.0, d1 = 0.0;
    if (lane < cnt) d0 = rows[a + lane].distance;
    if (lane + 32 < cnt) d1 = rows[a + 32 + lane].distance;
    double sum = 0.0;
    for (int i = 0; i < cnt; ++i) sum += __shfl_sync(0xffffffffu, i < 32 ? d0 : d1, i & 31);
    RtdlFixedRadiusRankedNeighborSummary sm;
    sm.query_id = __float_as_uint(qpts[qin].w);
    sm.neighbor_count = (uint32_t)cnt;
    sm.nearest_neighbor_id = cnt ? rows[a].neighbor_id : 0xFFFFFFFFu;
    sm.kth_neighbor_id = cnt ? rows[b - 1].neighbor_id : 0xFFFFFFFFu;
    sm.nearest_distance = cnt ? rows[a].distance : 0.0;
    sm.kth_distance = cnt ? rows[b - 1].distance : 0.0;
    sm.sum_distance = sum;
    if (lane == 0) {
      if (summaries) summaries[qin] = sm;
      mine = SummaryPartial{(unsigned long long)cnt, sm.nearest_neighbor_id, sm.kth_neighbor_id, sum};
    }
  }
  if (lane == 0) wsum[warp] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    SummaryPartial acc{0ull, 0ull, 0ull, 0.0};
    for (int w = 0; w < kSummaryThreads / 32; ++w) {
      acc.count += wsum[w].count;
      acc.nearest += wsum[w].nearest;
      acc.kth += wsum[w].kth;
      acc.sum += wsum[w].sum;
    }
    partial[blockIdx.x] = acc;
  }
}

// One block: thread t adds partials t, t + blockDim, ... in order, then a
// fixed tree over the threads.
__global__ void __launch_bounds__(1024) k_summary_final(const SummaryPartial* partial, uint32_t m, uint32_t nq,
                                                        RtdlFixedRadiusRankedNeighborAggregate* out) {
  __shared__ SummaryPartial sp[1024];
  SummaryPartial acc{0ull, 0ull, 0ull, 0.0};
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    acc.count += partial[i].count;
    acc.nearest += partial[i].nearest;
    acc.kth += partial[i].kth;
    acc.sum += partial[i].sum;
  }
  sp[threadIdx.x] = acc;
  __syncthreads();
  for (unsigned int stride = blockDim.x >> 1; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) {
      sp[threadIdx.x].count += sp[threadIdx.x + stride].count;
      sp[threadIdx.x].nearest += sp[threadIdx.x + stride].nearest;
      sp[threadIdx.x].kth += sp[threadIdx.x + stride].kth;
      sp[threadIdx.x].sum += sp[threadIdx.x + stride].sum;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out->query_count = nq;
    out->bounded_neighbor_count = sp[0].count;
    out->nearest_id_checksum = sp[0].nearest;
    out->kth_id_checksum = sp[0].kth;
    out->sum_distance = sp[0].sum;
  }
}

// Row offsets in processing order: poff[t] = offsets[qrank[qorder[t]]].
__global__ void k_proc_offsets(const uint32_t* qorder, const uint32_t* qrank, const unsigned long long* offsets,
                               uint32_t nq, unsigned long long* poff) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t qin = qorder[t];
    poff[t] = qin == kNone ? 0ull : offsets[qrank[qin]];
  }
}

// One warp per query of a work list (processing ranks): E = 4 for 65..128
// candidates (exact fixups deferred to k_emit_fixup), E = 8 for 129..kSlab
// (fixups in place through shared memory).
constexpr int kEmitListThreads = 128;

template <int E, bool DEFER>
// nwork_dev non-null (captured graphs): the list length is read there and the
// warps stride over the list.
__global__ void __launch_bounds__(kEmitListThreads)
    k_emit_list(EmitParams P, const uint32_t* work, uint32_t nwork, const unsigned int* nwork_dev) {
  __shared__ uint32_t wbuf[DEFER ? 1 : kEmitListThreads / 32][DEFER ? 1 : 32 * E];
  const int lane = threadIdx.x & 31;
  if (nwork_dev) nwork = *nwork_dev;
  uint32_t begin = 0;
  if (P.list_start) {  // one range of output ranks
    begin = P.list_start[P.range];
    nwork = P.list_start[P.range + 1];
  }
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t j = begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); j < nwork; j += warps) {  // whole warps
    const uint32_t t = work[j];
    EmitQuery q;
    emit_load(P, t, lane, q);
    const int n = (int)(q.qi.meta & kQueryCountMask);
    emit_query<E, DEFER>(P, t, q, n, lane, DEFER ? nullptr : wbuf[threadIdx.x >> 5]);
  }
}

// Output rank -> processing rank map for emission range by range (padding
// ranks hold no query).
__global__ void k_emit_order(const uint32_t* qorder, const uint32_t* qrank, uint32_t np, uint32_t* order) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x) {
    const uint32_t qin = qorder[t];
    if (qin != kNone) order[qrank[qin]] = t;
  }
}

// The download range of output rank r: the c with nq*c/C <= r < nq*(c+1)/C
// (integer division, as the range bounds are cut).
__device__ __forceinline__ uint32_t download_range(uint32_t r, uint32_t nq, uint32_t chunks) {
  return (uint32_t)((((uint64_t)r + 1) * chunks - 1) / nq);
}

// A work list of processing ranks partitioned by download range (a counting
// sort; the order inside a range is arbitrary, which the per-query emit does
// not see).  part[0..C) counts, part[C..2C] the range starts, part[2C+1..3C]
// the scatter cursors.
__global__ void k_range_count(const uint32_t* list, const unsigned int* n_dev, const uint32_t* qorder,
                              const uint32_t* qrank, uint32_t nq, uint32_t chunks, unsigned int* part) {
  const unsigned int n = *n_dev;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    atomicAdd(&part[download_range(qrank[qorder[list[j]]], nq, chunks)], 1u);
}

__global__ void k_range_starts(uint32_t chunks, unsigned int* part) {
  unsigned int sum = 0;
  for (uint32_t c = 0; c < chunks; ++c) {
    part[chunks + c] = sum;
    part[2 * chunks + 1 + c] = sum;
    sum += part[c];
  }
  part[2 * chunks] = sum;
}

__global__ void k_range_scatter(const uint32_t* list, const unsigned int* n_dev, const uint32_t* qorder,
                                const uint32_t* qrank, uint32_t nq, uint32_t chunks, unsigned int* part,
                                uint32_t* out) {
  const unsigned int n = *n_dev;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t t = list[j];
    const uint32_t c = download_range(qrank[qorder[t]], nq, chunks);
    out[atomicAdd(&part[2 * chunks + 1 + c], 1u)] = t;
  }
}

// First row of each range of output ranks [c * nq / chunks, ...), and the total.
__global__ void k_chunk_rows(const unsigned long long* offsets, uint32_t nq, int chunks, unsigned long long* out) {
  const int c = threadIdx.x;
  if (c <= chunks) out[c] = offsets[(uint64_t)nq * (uint32_t)c / (uint32_t)chunks];
}

// The next range's fix-ups start after this range's.
__global__ void k_fix_advance(unsigned int* fix_begin, const unsigned int* fix_count) { *fix_begin = *fix_count; }

__global__ void k_fill_i32(int* out, uint32_t n, int v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = v;
}

// Problem batch: *flag stays nonzero while every problem's query ids ascend.
__global__ void k_batch_ids_sorted(const float4* qpts, const uint32_t* qprob, uint32_t n, unsigned int* flag) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (qprob[i] == qprob[i - 1] && __float_as_uint(qpts[i].w) < __float_as_uint(qpts[i - 1].w)) *flag = 0u;
}

// Problem batch: one block per problem copies its sorted queries to the padded
// processing order (kNone fills the last warp) and records each warp's problem.
__global__ void k_batch_pad(const unsigned long long* qoff, const unsigned long long* pstart, const uint32_t* sorted,
                            uint32_t* qorder, uint32_t* warp_prob) {
  const uint32_t p = blockIdx.x;
  const unsigned long long a = qoff[p], nqp = qoff[p + 1] - a, base = pstart[p], padded = pstart[p + 1] - base;
  for (unsigned long long j = threadIdx.x; j < padded; j += blockDim.x) {
    qorder[base + j] = j < nqp ? sorted[a + j] : kNone;
    if ((j & 31) == 0) warp_prob[(base + j) >> 5] = p;
  }
}

// keys[j] = src[order[j]] (skipped when *skip is nonzero).
__global__ void k_gather_u32(const uint32_t* src, const uint32_t* order, uint32_t n, const unsigned int* skip,
                             uint32_t* keys) {
  if (*skip) return;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    keys[j] = src[order[j]];
}

// out[p] = offsets[qoff[p]]: the first row of each problem (and the total).
__global__ void k_problem_rows(const unsigned long long* offsets, const unsigned long long* qoff, uint32_t m,
                               unsigned long long* out) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p <= m; p += gridDim.x * blockDim.x) out[p] = offsets[qoff[p]];
}

__global__ void k_invert(const uint32_t* order, uint32_t n, const unsigned int* identity_flag, uint32_t* inv) {
  const bool ident = *identity_flag != 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    inv[ident ? j : order[j]] = (uint32_t)j;
}

// k > 64 KNN: every query takes the generic path.
__global__ void k_mark_all_heavy(const uint32_t* qorder, uint32_t nq, uint32_t n, uint32_t k, uint32_t* counts,
                                 uint8_t* flags, uint32_t* temp, uint32_t* heavy_list, uint32_t* heavy_m) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t qin = qorder[t];
    heavy_list[t] = qin;
    heavy_m[t] = n;
    counts[qin] = k < n ? k : n;
    flags[qin] = 2;
    temp[qin] = (uint32_t)t;
  }
}

__global__ void k_extract_ids(const float4* qpts, uint32_t n, uint32_t* ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    ids[i] = __float_as_uint(qpts[i].w);
}

struct HeavyEntry {
  unsigned long long key;  // bits of the FP64 distance (non-negative: bit order == value order)
  uint32_t nid;
  uint32_t sidx;
};

__device__ __forceinline__ Ctx make_ctx(const SceneView& S, const float4* qpts, const double* qraw, int qstride,
                                        uint32_t qin, const DevBands& B) {
  Ctx c;
  const float4 q = qpts[qin];
  c.qx = q.x;
  c.qy = q.y;
  c.qz = q.z;
  const double* r = qraw + (size_t)qin * qstride;
  c.ex = r[1];
  c.ey = r[2];
  c.ez = qstride == 4 ? r[3] : 0.0;
  c.pts = S.pts;
  c.pts64 = S.pts64;
  c.perm = S.perm;
  c.scene_inexact = *S.inexact;
  c.rho = B.rho;
  c.e_abs = B.e_abs;
  c.floor2 = B.floor2;
  return c;
}

__global__ void __launch_bounds__(kHeavyThreads)
    k_heavy_gather(SceneView S, const float4* qpts, const double* qraw, int qstride, const uint32_t* heavy_list,
                   const unsigned long long* seg_off, const uint32_t* seg_size, int knn, const DevBands* bands,
                   HeavyEntry* scratch, unsigned int* error) {
  __shared__ unsigned int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  const uint32_t h = blockIdx.x;
  const uint32_t qin = heavy_list[h];
  const DevBands B = *bands;
  const Ctx c = make_ctx(S, qpts, qraw, qstride, qin, B);
  HeavyEntry* seg = scratch + seg_off[h];
  const uint32_t P2 = seg_size[h];
  for (uint32_t i = threadIdx.x; i < S.n; i += blockDim.x) {
    if (!knn) {
      const float4 p = __ldg(&S.pts[i]);
      const float dx = p.x - c.qx, dy = p.y - c.qy, dz = p.z - c.qz;
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      if (d2 > B.hi2) continue;
      if (d2 >= B.lo2 && exact_d2(c, i) > B.r2) continue;
    }
    const double dist = __dsqrt_rn(exact_d2(c, i));
    const unsigned int pos = atomicAdd(&cnt, 1u);
    if (pos < P2) {
      HeavyEntry e;
      e.key = (unsigned long long)__double_as_longlong(dist);
      e.nid = __float_as_uint(__ldg(&S.pts[i].w));
      e.sidx = i;
      seg[pos] = e;
    } else {
      atomicOr(error, 2u);
    }
  }
  __syncthreads();
  for (uint32_t i = cnt + threadIdx.x; i < P2; i += blockDim.x) {
    HeavyEntry e;
    e.key = ~0ull;
    e.nid = kNone;
    e.sidx = kNone;
    seg[i] = e;
  }
}

// Generic-path gather for a radius query with more than kSlab candidates: one
// warp per query walks the BVH with a warp-uniform stack; the lanes test a leaf
// bucket's points together and append in-radius candidates with a ballot
// prefix (no atomics).
__global__ void __launch_bounds__(32)
    k_heavy_gather_bvh(SceneView S, const float4* qpts, const double* qraw, int qstride, const uint32_t* heavy_list,
                       const unsigned long long* seg_off, const uint32_t* seg_size, const DevBands* bands,
                       const uint32_t* qprob, const double* item_rad, HeavyEntry* scratch, unsigned int* error) {
  const int lane = threadIdx.x;
  const uint32_t h = blockIdx.x;
  const uint32_t qin = heavy_list[h];
  const uint32_t prob = qprob ? qprob[qin] : 0u;
  // item_rad: the radius this query gathers within (a tested radius that holds its rows)
  const DevBands B = item_rad ? bands_at_radius(bands[prob], item_rad[h]) : bands[prob];
  const Ctx c = make_ctx(S, qpts, qraw, qstride, qin, B);
  HeavyEntry* seg = scratch + seg_off[h];
  const uint32_t P2 = seg_size[h];
  const unsigned int lt_mask = (1u << lane) - 1u;
  uint32_t cnt = 0;
  int cur = S.n > 0 ? 0 : kRopeEnd, end = kRopeEnd;
  if (S.prob_root) {  // problem batch: the query's problem subtree only
    cur = S.prob_root[prob];
    if (cur != kRopeEnd) end = __float_as_int(__ldg(&S.nodes[2 * cur + 1]).w);
  }
  while (cur != end) {  // warp-uniform: every lane follows the same nodes
    const float4 a = __ldg(&S.nodes[2 * cur]), b = __ldg(&S.nodes[2 * cur + 1]);
    const int hit = __float_as_int(a.w);
    if (box_d2(c.qx, c.qy, c.qz, a, b) <= B.box_hi2) {
      if (hit >= 0) {
        ++cur;  // internal node: its left child is the next record
        continue;
      }
      const int first = leaf_first(hit), leaf = leaf_count(hit);
      bool acc = false;
      const uint32_t i = (uint32_t)(first + lane);
      if (lane < leaf) {
        const float4 p = __ldg(&S.pts[i]);
        const float dx = p.x - c.qx, dy = p.y - c.qy, dz = p.z - c.qz;
        const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        acc = d2 <= B.hi2 && (d2 < B.lo2 || exact_d2(c, i) <= B.r2);
      }
      const unsigned int m = __ballot_sync(0xffffffffu, acc);
      if (acc) {
        const uint32_t pos = cnt + __popc(m & lt_mask);
        if (pos < P2) {
          HeavyEntry en;
          en.key = (unsigned long long)__double_as_longlong(__dsqrt_rn(exact_d2(c, i)));
          en.nid = __float_as_uint(__ldg(&S.pts[i].w));
          en.sidx = i;
          seg[pos] = en;
        } else {
          atomicOr(error, 2u);
        }
      }
      cnt += __popc(m);
    }
    cur = __float_as_int(b.w);
  }
  for (uint32_t i = cnt + lane; i < P2; i += 32) {
    HeavyEntry en;
    en.key = ~0ull;
    en.nid = kNone;
    en.sidx = kNone;
    seg[i] = en;
  }
}

__device__ __forceinline__ bool heavy_greater(const HeavyEntry& a, const HeavyEntry& b, const uint32_t* perm) {
  if (a.key != b.key) return a.key > b.key;
  if (a.nid != b.nid) return a.nid > b.nid;
  if (a.sidx == kNone || b.sidx == kNone) return a.sidx == kNone && b.sidx != kNone;
  return perm[a.sidx] > perm[b.sidx];
}

constexpr uint32_t kHeavySmemEntries = 2048;  // 32 KiB of 16-B entries per block

template <typename Ptr>
__device__ __forceinline__ void bitonic_block(Ptr e, uint32_t P2, const uint32_t* perm) {
  for (uint32_t k = 2; k <= P2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const HeavyEntry a = e[i], b = e[ixj];
          const bool up = (i & k) == 0;
          if (heavy_greater(a, b, perm) == up) {
            e[i] = b;
            e[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Block-per-query bitonic sort of a segment by (distance, neighbor id, search
// input index); in shared memory up to 2,048 entries, in global memory above.
__global__ void __launch_bounds__(kHeavyThreads)
    k_heavy_sort(const unsigned long long* seg_off, const uint32_t* seg_size, HeavyEntry* scratch,
                 const uint32_t* perm) {
  extern __shared__ HeavyEntry heavy_smem[];
  HeavyEntry* e = scratch + seg_off[blockIdx.x];
  const uint32_t P2 = seg_size[blockIdx.x];
  if (P2 <= kHeavySmemEntries) {
    for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) heavy_smem[i] = e[i];
    __syncthreads();
    bitonic_block(heavy_smem, P2, perm);
    for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) e[i] = heavy_smem[i];
  } else {
    bitonic_block(e, P2, perm);
  }
}

__global__ void k_heavy_emit(const unsigned long long* seg_off, const unsigned long long* out_off,
                             const uint32_t* out_count, const HeavyEntry* scratch, uint32_t* heavy_out) {
  const HeavyEntry* e = scratch + seg_off[blockIdx.x];
  uint32_t* dst = heavy_out + out_off[blockIdx.x];
  const uint32_t k = out_count[blockIdx.x];
  for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) dst[j] = e[j].sidx;
}

struct ExpandParams {
  SceneView S;
  const float4* qpts;
  const double* qraw;
  int qstride;
  const uint32_t* oorder;
  const DevBands* bands;
  uint32_t nq;
  int L;
  const uint32_t* counts;
  const uint8_t* flags;
  const uint32_t* temp;
  const uint32_t* heavy_out;
  const unsigned long long* heavy_out_off;
  const unsigned long long* offsets;
  void* rows;
  unsigned long long capacity;
  int ranked;
  uint8_t* overflow_out;
  unsigned int* error;
  const uint32_t* work_list;  // optional: process only these queries (input indices)
  const uint32_t* qrank;      // with work_list: input index -> output rank
};

// G consecutive threads per query (G = 32: a warp) write its rows with the
// exact FP64 distance: all queries in output order, or the queries of
// `work_list`.  G is at least the longest row list when it is known to be
// short (nearest lists of k <= 16 rows), so a warp serves 32 / G queries and
// their rows, consecutive in output order, with one set of stores.
template <int G>
__global__ void __launch_bounds__(kExpandThreads) k_expand(ExpandParams P) {
  const int lane = threadIdx.x & (G - 1);
  const uint64_t groups = ((uint64_t)gridDim.x * blockDim.x) / G;
  const bool ids_sorted = P.bands->ids_sorted != 0;
  const bool scene_inexact = *P.S.inexact != 0;
  for (uint64_t j = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; j < P.nq; j += groups) {
    const uint32_t qin = P.work_list ? P.work_list[j] : (ids_sorted ? (uint32_t)j : P.oorder[j]);
    const uint32_t cnt = P.counts[qin];
    const uint8_t fl = P.flags[qin];
    if (P.overflow_out != nullptr && lane == 0) P.overflow_out[qin] = fl & 1;
    if (cnt == 0 || P.rows == nullptr) continue;
    const unsigned long long base = P.offsets[P.work_list ? P.qrank[qin] : (uint32_t)j];
    const uint32_t qid = __float_as_uint(P.qpts[qin].w);
    const double* r = P.qraw + (size_t)qin * P.qstride;
    const double ex = r[1], ey = r[2], ez = P.qstride == 4 ? r[3] : 0.0;
    const uint32_t* src = P.work_list ? P.heavy_out + P.heavy_out_off[j]
                          : (fl & 2) ? P.heavy_out + P.heavy_out_off[P.temp[(size_t)qin * P.L]]
                                     : P.temp + (size_t)qin * P.L;
    for (uint32_t s = lane; s < cnt; s += G) {
      const uint32_t sidx = src[s];
      if (sidx >= P.S.n) {  // never expected: a generic-path slot without a candidate
        atomicOr(P.error, 4u);
        continue;
      }
      const float4 p = __ldg(&P.S.pts[sidx]);
      double sx, sy, sz;
      if (scene_inexact) {
        const double* pp = P.S.pts64 + 3ull * sidx;
        sx = pp[0];
        sy = pp[1];
        sz = pp[2];
      } else {
        sx = p.x;
        sy = p.y;
        sz = p.z;
      }
      const double dx = __dsub_rn(sx, ex), dy = __dsub_rn(sy, ey), dz = __dsub_rn(sz, ez);
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      const double dist = __dsqrt_rn(d2);
      const unsigned long long row = base + s;
      if (row >= P.capacity) continue;
      const uint32_t nid = __float_as_uint(p.w);
      const unsigned long long db = (unsigned long long)__double_as_longlong(dist);
      if (!P.ranked) {
        reinterpret_cast<uint4*>(P.rows)[row] = make_uint4(qid, nid, (uint32_t)db, (uint32_t)(db >> 32));
      } else {
        uint2* out = reinterpret_cast<uint2*>(static_cast<char*>(P.rows) + row * 24);
        out[0] = make_uint2(qid, nid);
        out[1] = make_uint2((uint32_t)db, (uint32_t)(db >> 32));
        out[2] = make_uint2(s + 1, 0u);
      }
    }
  }
}

// ---- directed Hausdorff: FP64 max over per-query nearest distances ---------
struct Witness {
  unsigned long long dist;  // FP64 bits
  uint32_t qid, nid;
};
// max by (distance, -query_id, -neighbor_id)
__device__ __forceinline__ bool witness_better(const Witness& a, const Witness& b) {
  if (a.dist != b.dist) return a.dist > b.dist;
  if (a.qid != b.qid) return a.qid < b.qid;
  return a.nid < b.nid;
}

__global__ void __launch_bounds__(256)
    k_nearest_reduce(SceneView S, const float4* qpts, const double* qraw, int qstride, uint32_t nq,
                     const uint32_t* temp, double* nearest_dist, uint32_t* nearest_id, Witness* partial) {
  __shared__ Witness warp_best[8];
  Witness best{0ull, kNone, kNone};
  bool have = false;
  const bool scene_inexact = *S.inexact != 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t sidx = temp[i];
    const float4 p = __ldg(&S.pts[sidx]);
    const double* r = qraw + i * qstride;
    double sx, sy, sz;
    if (scene_inexact) {
      const double* pp = S.pts64 + 3ull * sidx;
      sx = pp[0];
      sy = pp[1];
      sz = pp[2];
    } else {
      sx = p.x;
      sy = p.y;
      sz = p.z;
    }
    const double dx = __dsub_rn(sx, r[1]), dy = __dsub_rn(sy, r[2]), dz = __dsub_rn(sz, qstride == 4 ? r[3] : 0.0);
    const double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    const Witness w{(unsigned long long)__double_as_longlong(dist), __float_as_uint(qpts[i].w), __float_as_uint(p.w)};
    if (nearest_dist) nearest_dist[i] = dist;
    if (nearest_id) nearest_id[i] = w.nid;
    if (!have || witness_better(w, best)) {
      best = w;
      have = true;
    }
  }
  if (!have) best = Witness{0ull, kNone, kNone};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Witness other;
    other.dist = __shfl_xor_sync(0xffffffffu, best.dist, o);
    other.qid = __shfl_xor_sync(0xffffffffu, best.qid, o);
    other.nid = __shfl_xor_sync(0xffffffffu, best.nid, o);
    if (witness_better(other, best)) best = other;
  }
  if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    Witness b = warp_best[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (witness_better(warp_best[w], b)) b = warp_best[w];
    partial[blockIdx.x] = b;
  }
}

__global__ void k_witness_final(const Witness* partial, int n, Witness* out) {
  if (threadIdx.x != 0) return;
  Witness b = partial[0];
  for (int i = 1; i < n; ++i)
    if (witness_better(partial[i], b)) b = partial[i];
  *out = b;
}

bool stats_enabled() {
  static const bool on = std::getenv("RTDL_B200_STATS") != nullptr;
  return on;
}



}  // namespace

std::vector<unsigned long long>& last_stats() {
  thread_local std::vector<unsigned long long> v(kStatCount, 0ull);
  return v;
}

namespace {

// Ranges of output ranks whose rows are copied to the host as each completes.
constexpr int kDownloadChunks = 8;

struct Readback {
  unsigned long long rows;
  unsigned int heavy;  // these four are copied together from the `small` device counters
  unsigned int error;
  unsigned int mid;
  unsigned int big;
  unsigned int scene_bad;
  unsigned int query_bad;
  unsigned int fixups;
  unsigned int refine_left;  // heavy queries still unresolved after a refinement pass
  unsigned long long chunk_rows[kDownloadChunks + 1];  // first row of each download range
};

// Pinned and mapped into the device address space, so small reads of device
// counters can be written into it by a kernel (SmallReads) instead of being
// copied by the copy engine.
Readback* pinned_readback() {
  thread_local Readback* rb = nullptr;
  if (rb == nullptr)
    RTDL_CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&rb), sizeof(Readback),
                                  cudaHostAllocMapped | cudaHostAllocPortable));
  return rb;
}

// Small reads of device counters into the thread's Readback, written by one
// kernel of one warp.  Kernel stores do not queue behind copies: a call whose
// rows are being copied to the host (the copy engine busy for milliseconds)
// reads its counts at once instead of after those copies.  Sources and
// fields are 4-byte words; the host reads the fields after the stream has
// been synchronized.
struct SmallRead {
  static constexpr int kMax = 6;
  const uint32_t* src[kMax];
  uint32_t* dst[kMax];
  uint32_t words[kMax];
  int n;
};

__global__ void k_read_small(SmallRead r) {
  for (int k = 0; k < r.n; ++k)
    for (uint32_t i = threadIdx.x; i < r.words[k]; i += blockDim.x) r.dst[k][i] = r.src[k][i];
}

class SmallReads {
 public:
  explicit SmallReads(Readback* rb) : rb_(rb) {
    void* alias = nullptr;
    RTDL_CUDA_CHECK(cudaHostGetDevicePointer(&alias, rb, 0));
    alias_ = static_cast<char*>(alias);
    r_.n = 0;
  }
  // `field` is a member of the Readback given at construction.
  void add(void* field, const void* dev, size_t bytes) {
    if (r_.n == SmallRead::kMax) throw std::runtime_error("too many small reads in one launch");
    r_.src[r_.n] = static_cast<const uint32_t*>(dev);
    r_.dst[r_.n] = reinterpret_cast<uint32_t*>(alias_ + (static_cast<char*>(field) - reinterpret_cast<char*>(rb_)));
    r_.words[r_.n] = (uint32_t)(bytes / 4);
    ++r_.n;
  }
  void launch(cudaStream_t s) {
    k_read_small<<<1, 32, 0, s>>>(r_);
    RTDL_LAUNCHED(1);
    r_.n = 0;
  }

 private:
  Readback* rb_;
  char* alias_;
  SmallRead r_;
};

inline unsigned int grid_for(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  const uint64_t cap = (uint64_t)kSmCount * 32;
  return (unsigned int)(b < cap ? b : cap);
}

inline uint32_t next_pow2(uint32_t v) {
  uint32_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

struct QueryPrep {
  PointStats* qst = nullptr;
  float4* qpts = nullptr;
  DevBands* bands = nullptr;   // one, or one per problem of a batch
  uint32_t* qorder = nullptr;  // processing rank -> input index (a batch pads problems to whole warps: kNone)
  uint32_t* qcodes = nullptr;  // Morton codes in processing order (qcodes[t] belongs to qorder[t]); single only
  uint32_t* oorder = nullptr;
  uint32_t nproc = 0;          // processing ranks
  const unsigned int* order_identity = nullptr;  // device flag: output order == input order
  // problem batch only
  uint32_t* qprob = nullptr;      // problem of each query (input order)
  uint32_t* warp_prob = nullptr;  // problem of each warp of processing ranks
  uint32_t* prob_kmax = nullptr;
  unsigned int* sorted_flag = nullptr;
  unsigned long long* qoff = nullptr;  // device copy of the query offsets
  double* prob_radius = nullptr;       // radius of each problem
  int* shared_roots = nullptr;         // requests against one plain scene: every problem's root is the scene's
  SceneView view{};                    // the scene as the traversal kernels see it
  const PreparedQueries* borrowed = nullptr;  // set: the query-side buffers belong to a prepared query set
};

// The call-side view of a prepared query set: its buffers are borrowed, only
// the bands (scene and query statistics, this radius) are computed.
QueryPrep borrow_prepared(Scene* sc, const PreparedQueries* pq, double radius, cudaStream_t s) {
  QueryPrep qp;
  qp.borrowed = pq;
  qp.qst = pq->qst;
  qp.qpts = pq->qpts;
  qp.qorder = pq->qorder;
  qp.oorder = pq->oorder;
  qp.nproc = pq->n;
  qp.order_identity = pq->identity;
  qp.view = sc->view();
  qp.bands = static_cast<DevBands*>(dev_alloc(sizeof(DevBands), s));
  k_bands<<<1, 32, 0, s>>>(sc->stats, pq->qst, radius, 1, qp.bands);
  RTDL_LAUNCHED(1);
  return qp;
}



QueryPrep prepare_queries(Scene* sc, const void* queries_dev, uint32_t nq, bool has_radius, double radius,
                          bool want_output_order, cudaStream_t s) {
  QueryPrep qp;
  qp.qst = static_cast<PointStats*>(dev_alloc(sizeof(PointStats), s));
  qp.qpts = static_cast<float4*>(dev_alloc(sizeof(float4) * nq, s));
  qp.bands = static_cast<DevBands*>(dev_alloc(sizeof(DevBands), s));
  qp.qorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  reset_stats(qp.qst, s);
  prep_points(queries_dev, nq, sc->dim, qp.qpts, qp.qst, s);
  k_bands<<<1, 32, 0, s>>>(sc->stats, qp.qst, radius, has_radius ? 1 : 0, qp.bands);
  RTDL_LAUNCHED(1);
  qp.nproc = nq;
  qp.order_identity = &qp.bands->ids_sorted;
  qp.view = sc->view();
  qp.qcodes = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  morton_codes(qp.qpts, nq, sc->dim, sc->stats, qp.qcodes, s);
  iota_u32(qp.qorder, nq, s);
  radix_sort_pairs(qp.qcodes, qp.qorder, nq, 0, sc->dim == 3 ? 30 : 32, nullptr, &qp.qst->bad, s);
  if (want_output_order) {
    qp.oorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
    uint32_t* ids = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
    k_extract_ids<<<grid_for(nq, 256), 256, 0, s>>>(qp.qpts, nq, ids);
    RTDL_LAUNCHED(1);
    iota_u32(qp.oorder, nq, s);
    radix_sort_pairs(ids, qp.oorder, nq, 0, 32, &qp.bands->ids_sorted, &qp.qst->bad, s);
    dev_free(ids, s);
  }
  return qp;
}

// A problem batch's query preparation: per-query problem ids, per-problem
// bands and kmax, composite (problem, Morton) sort, processing order padded
// so each warp holds queries of one problem, and the output order (problem,
// then query id, stable).
QueryPrep prepare_queries_batch(Scene* sc, const void* queries_dev, uint32_t nq, const BatchSpec& bs,
                                cudaStream_t s) {
  const uint32_t P = bs.problems;
  QueryPrep qp;
  const bool shared = sc->problems == 0;  // several requests against one plain scene
  qp.view = sc->view();
  if (shared) {
    qp.shared_roots = static_cast<int*>(dev_alloc(sizeof(int) * P, s));
    k_fill_i32<<<div_up(P, 256), 256, 0, s>>>(qp.shared_roots, P, sc->n > 0 ? 0 : kRopeEnd);
    RTDL_LAUNCHED(1);
    qp.view.prob_root = qp.shared_roots;
  }
  std::vector<unsigned long long> pstart(P + 1, 0);
  for (uint32_t p = 0; p < P; ++p) pstart[p + 1] = pstart[p] + (bs.qoff[p + 1] - bs.qoff[p] + 31) / 32 * 32;
  if (pstart[P] > 0xFFFFFFFFull - 32) throw std::runtime_error("problem batch has too many queries");
  qp.nproc = (uint32_t)pstart[P];
  qp.qst = static_cast<PointStats*>(dev_alloc(sizeof(PointStats), s));
  qp.qpts = static_cast<float4*>(dev_alloc(sizeof(float4) * (nq ? nq : 1), s));
  qp.bands = static_cast<DevBands*>(dev_alloc(sizeof(DevBands) * P, s));
  qp.qorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (qp.nproc ? qp.nproc : 1), s));
  qp.qprob = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (nq ? nq : 1), s));
  qp.warp_prob = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (qp.nproc / 32 + 1), s));
  qp.prob_kmax = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * P, s));
  qp.sorted_flag = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int), s));
  qp.qoff = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (P + 1), s));
  qp.order_identity = qp.sorted_flag;
  unsigned long long* d_pstart = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (P + 1), s));
  qp.prob_radius = static_cast<double*>(dev_alloc(sizeof(double) * P, s));
  double* d_radius = qp.prob_radius;
  RTDL_CUDA_CHECK(cudaMemcpyAsync(qp.qoff, bs.qoff, sizeof(unsigned long long) * (P + 1), cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(d_pstart, pstart.data(), sizeof(unsigned long long) * (P + 1),
                                  cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(d_radius, bs.radius, sizeof(double) * P, cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(qp.prob_kmax, bs.kmax, sizeof(uint32_t) * P, cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemsetAsync(qp.sorted_flag, 0xFF, sizeof(unsigned int), s));  // nonzero: sorted
  reset_stats(qp.qst, s);
  prep_points(queries_dev, nq, sc->dim, qp.qpts, qp.qst, s);
  batch_problem_ids(qp.qoff, P, nq, qp.qprob, s);
  if (nq > 1) {
    k_batch_ids_sorted<<<grid_for(nq, 256), 256, 0, s>>>(qp.qpts, qp.qprob, nq, qp.sorted_flag);
    RTDL_LAUNCHED(1);
  }
  k_bands_batch<<<div_up(P, 128), 128, 0, s>>>(sc->stats, qp.qst, d_radius, P, qp.sorted_flag, qp.bands);
  RTDL_LAUNCHED(1);
  // processing order: composite (problem, Morton in the problem's box) sort, padded per problem
  uint32_t* codes = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (nq ? nq : 1), s));
  uint32_t* sorted = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (nq ? nq : 1), s));
  if (shared)
    batch_codes(qp.qpts, qp.qprob, nq, sc->dim, sc->stats, 0, batch_code_bits(P, sc->dim), codes, s);
  else
    batch_codes(qp.qpts, qp.qprob, nq, sc->dim, sc->prob_stats, 1, sc->code_bits, codes, s);
  iota_u32(sorted, nq, s);
  radix_sort_pairs(codes, sorted, nq, 0, 32, nullptr, &qp.qst->bad, s);
  k_batch_pad<<<P, 256, 0, s>>>(qp.qoff, d_pstart, sorted, qp.qorder, qp.warp_prob);
  RTDL_LAUNCHED(1);
  // output order: by query id, then (stable) by problem; skipped when every
  // problem's ids are already ascending
  qp.oorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (nq ? nq : 1), s));
  iota_u32(qp.oorder, nq, s);
  k_extract_ids<<<grid_for(nq, 256), 256, 0, s>>>(qp.qpts, nq, codes);
  RTDL_LAUNCHED(1);
  radix_sort_pairs(codes, qp.oorder, nq, 0, 32, qp.sorted_flag, &qp.qst->bad, s);
  k_gather_u32<<<grid_for(nq, 256), 256, 0, s>>>(qp.qprob, qp.oorder, nq, qp.sorted_flag, codes);
  RTDL_LAUNCHED(1);
  radix_sort_pairs(codes, qp.oorder, nq, 0, batch_problem_bits(P), qp.sorted_flag, &qp.qst->bad, s);
  dev_free(codes, s);
  dev_free(sorted, s);
  dev_free(d_pstart, s);
  return qp;
}

void free_prep(QueryPrep& qp, cudaStream_t s) {
  if (qp.borrowed) {
    dev_free(qp.bands, s);
    return;
  }
  dev_free(qp.qst, s);
  dev_free(qp.qpts, s);
  dev_free(qp.bands, s);
  dev_free(qp.qorder, s);
  dev_free(qp.qcodes, s);
  dev_free(qp.oorder, s);
  dev_free(qp.qprob, s);
  dev_free(qp.warp_prob, s);
  dev_free(qp.prob_kmax, s);
  dev_free(qp.sorted_flag, s);
  dev_free(qp.qoff, s);
  dev_free(qp.shared_roots, s);
  dev_free(qp.prob_radius, s);
}

}  // namespace

namespace {

// Output of the generic (block/warp-per-query) path: sorted candidate indices
// per query, located through heavy_out_off[h] (h = the query's generic slot).
struct GenericOut {
  uint32_t* heavy_out = nullptr;
  unsigned long long* heavy_out_off = nullptr;
  void release(cudaStream_t s) {
    dev_free(heavy_out, s);
    dev_free(heavy_out_off, s);
    heavy_out = nullptr;
    heavy_out_off = nullptr;
  }
};

// Runs the generic path for H queries listed in heavy_list with candidate
// counts heavy_m (read back here).  knn: gather every scene point (brute
// force); otherwise gather in-radius candidates through the BVH.
GenericOut run_generic_path(Scene* sc, const QueryPrep& qp, const void* queries_dev, int qstride, uint32_t H,
                            const uint32_t* heavy_list, const uint32_t* heavy_m, uint32_t limit, bool knn,
                            unsigned int* error, cudaStream_t s, const double* item_rad = nullptr) {
  GenericOut g;
  std::vector<uint32_t> hm(H);
  RTDL_CUDA_CHECK(cudaMemcpyAsync(hm.data(), heavy_m, sizeof(uint32_t) * H, cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  std::vector<unsigned long long> seg_off(H), out_off(H);
  std::vector<uint32_t> seg_size(H), out_cnt(H);
  unsigned long long seg_total = 0, out_total = 0;
  for (uint32_t h = 0; h < H; ++h) {
    seg_size[h] = next_pow2(hm[h] ? hm[h] : 1);
    seg_off[h] = seg_total;
    seg_total += seg_size[h];
    out_cnt[h] = hm[h] < limit ? hm[h] : limit;
    out_off[h] = out_total;
    out_total += out_cnt[h];
  }
  const unsigned long long kScratchLimit = 1ull << 28;  // entries (4 GiB of 16-B sort entries)
  if (seg_total > kScratchLimit)
    throw std::runtime_error(
        "b200 backend: the generic path for limits above 64 needs more than 4 GiB of sort scratch; "
        "reduce k/k_max or split the query set");
  unsigned long long* d_seg_off = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * H, s));
  uint32_t* d_seg_size = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * H, s));
  g.heavy_out_off = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * H, s));
  uint32_t* d_out_cnt = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * H, s));
  HeavyEntry* scratch = static_cast<HeavyEntry*>(dev_alloc(sizeof(HeavyEntry) * seg_total, s));
  g.heavy_out = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (out_total ? out_total : 1), s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(d_seg_off, seg_off.data(), sizeof(unsigned long long) * H, cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(d_seg_size, seg_size.data(), sizeof(uint32_t) * H, cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(g.heavy_out_off, out_off.data(), sizeof(unsigned long long) * H,
                                  cudaMemcpyHostToDevice, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(d_out_cnt, out_cnt.data(), sizeof(uint32_t) * H, cudaMemcpyHostToDevice, s));
  if (knn)
    k_heavy_gather<<<H, kHeavyThreads, 0, s>>>(sc->view(), qp.qpts, static_cast<const double*>(queries_dev), qstride,
                                               heavy_list, d_seg_off, d_seg_size, 1, qp.bands, scratch, error);
  else
    k_heavy_gather_bvh<<<H, 32, 0, s>>>(qp.view, qp.qpts, static_cast<const double*>(queries_dev), qstride,
                                        heavy_list, d_seg_off, d_seg_size, qp.bands, qp.qprob, item_rad, scratch,
                                        error);
  k_heavy_sort<<<H, kHeavyThreads, sizeof(HeavyEntry) * kHeavySmemEntries, s>>>(d_seg_off, d_seg_size, scratch,
                                                                                sc->perm);
  k_heavy_emit<<<H, kHeavyThreads, 0, s>>>(d_seg_off, g.heavy_out_off, d_out_cnt, scratch, g.heavy_out);
  RTDL_LAUNCHED(3);
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // the host vectors above are read by the copies
  dev_free(d_seg_off, s);
  dev_free(d_seg_size, s);
  dev_free(d_out_cnt, s);
  dev_free(scratch, s);
  return g;
}

// Host side of the radius refinement (see k_collect_refine): up to kRefinePasses
// passes over the unresolved heavy queries, each followed by an update that
// resolves queries or narrows their radius; after the last pass the
// unresolved ones are listed for the generic path.
constexpr int kRefinePasses = 6;

struct RefineOut {
  uint32_t generic = 0, mid = 0, big = 0;
  const uint32_t* generic_qin = nullptr;
  const uint32_t* generic_m = nullptr;
  const double* generic_rad = nullptr;  // the radius each generic query gathers within
  std::vector<void*> buffers;  // released by the caller once the rows are out
};

RefineOut refine_heavy(const CollectParams& C, const QueryPrep& qp, double radius, uint32_t kmax, uint32_t H,
                       const uint32_t* heavy_list, const uint32_t* heavy_m, const uint32_t* heavy_t,
                       QueryInfo* qinfo, uint8_t* flags, uint32_t* mid_list, uint32_t* big_list, unsigned int* small,
                       cudaStream_t s, const std::function<void()>& after_first_pass = {}) {
  RefineOut out;
  auto alloc = [&](size_t bytes) {
    void* p = dev_alloc(bytes ? bytes : 1, s);
    out.buffers.push_back(p);
    return p;
  };
  uint32_t* work[2];
  double *rad[2], *lo[2], *hi[2], *frad[2];
  uint32_t* full[2];
  for (int b = 0; b < 2; ++b) {
    work[b] = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * H));
    rad[b] = static_cast<double*>(alloc(sizeof(double) * H));
    lo[b] = static_cast<double*>(alloc(sizeof(double) * H));
    hi[b] = static_cast<double*>(alloc(sizeof(double) * H));
    full[b] = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * H));
    frad[b] = static_cast<double*>(alloc(sizeof(double) * H));
  }
  double* gen_rad = static_cast<double*>(alloc(sizeof(double) * H));
  uint32_t* cnt = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * H));
  uint32_t* gen_qin = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * H));
  uint32_t* gen_m = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * H));
  unsigned int* next_count = static_cast<unsigned int*>(alloc(sizeof(unsigned int)));
  k_refine_init<<<div_up(H, 256), 256, 0, s>>>(heavy_list, heavy_m, heavy_t, H, qp.qprob, qp.prob_radius, radius,
                                               qp.prob_kmax, kmax, work[0], rad[0], lo[0], hi[0], full[0],
                                               frad[0], nullptr);
  RTDL_LAUNCHED(1);
  Readback* rb = pinned_readback();
  uint32_t n = H;
  int cur = 0;
  for (int pass = 0; pass < kRefinePasses && n > 0; ++pass) {
    const bool last = pass == kRefinePasses - 1;

    RefineParams R;
    R.C = C;
    R.qprob = qp.qprob;
    R.work = work[cur];
    R.rad = rad[cur];
    R.nwork = n;
    R.cnt = cnt;
    R.nwork_dev = nullptr;
    R.packet_min = 0;
    const bool scene_packet = n >= qp.nproc / 8 && !qp.qprob && !qp.view.prob_root;
    if (n >= qp.nproc / 8) {  // many heavy queries: they cluster, a packet of them walks one region
      if (scene_packet)
        k_collect_refine_packet_scene<<<div_up(n, 256), 256, 0, s>>>(R);
      else
        k_collect_refine_packet<<<div_up(n, 256), 256, 0, s>>>(R);
    } else
      k_collect_refine<<<div_up((uint64_t)n * 32, 256), 256, 0, s>>>(R);
    RTDL_CUDA_CHECK(cudaMemsetAsync(next_count, 0, sizeof(unsigned int), s));
    RefineUpdate U;
    U.qorder = qp.qorder;
    U.qprob = qp.qprob;
    U.prob_kmax = qp.prob_kmax;
    U.kmax = kmax;
    U.qinfo = qinfo;
    U.flags = flags;
    U.mid_list = mid_list;
    U.big_list = big_list;
    U.small = small;
    U.work = work[cur];
    U.rad = rad[cur];
    U.lo = lo[cur];
    U.hi = hi[cur];
    U.full = full[cur];
    U.frad = frad[cur];
    U.cnt = cnt;
    U.nwork = n;
    U.nwork_dev = nullptr;
    U.next_work = work[cur ^ 1];
    U.next_rad = rad[cur ^ 1];
    U.next_lo = lo[cur ^ 1];
    U.next_hi = hi[cur ^ 1];
    U.next_full = full[cur ^ 1];
    U.next_frad = frad[cur ^ 1];
    U.next_count = next_count;
    U.generic_qin = gen_qin;
    U.generic_m = gen_m;
    U.generic_rad = gen_rad;
    U.last = last ? 1 : 0;
    k_refine_update<<<div_up(n, 256), 256, 0, s>>>(U);
    RTDL_LAUNCHED(2);
    if (pass == 0 && after_first_pass) after_first_pass();  // work the caller queues before the first wait

    SmallReads reads(rb);
    reads.add(&rb->refine_left, next_count, sizeof(unsigned int));
    reads.launch(s);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    n = rb->refine_left;
    if (last) out.generic = n;
    cur ^= 1;
  }
  out.generic_qin = gen_qin;
  out.generic_m = gen_m;
  out.generic_rad = gen_rad;
  SmallReads reads(rb);
  reads.add(&rb->mid, small + 2, sizeof(unsigned int) * 2);
  reads.launch(s);
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  out.mid = rb->mid;
  out.big = rb->big;
  return out;
}

// The collect pass, by the tuning's traversal (a problem batch walks in packets).
void launch_collect(const CollectParams& C, uint32_t np, uint32_t nq, bool batch, bool stats, cudaStream_t s) {
  const int threads = tuning().block_threads;
  const bool packet = tuning().traversal != 1 || batch;
  if (packet) {
    const unsigned int grid = div_up(np, threads);
    const bool cube = tuning().traversal == 2;
    // occupancy bounds chosen so neither variant spills (32 and 40 registers)
    if (batch)  // several problems (traversal counters are not gathered here)
      tuning().traversal == 4 ? k_collect_packet<false, false, true, 5, kLeafHybrid><<<grid, threads, 0, s>>>(C)
                              : k_collect_packet<false, false, true, 5><<<grid, threads, 0, s>>>(C);
    else if (tuning().traversal == 3)
      stats ? k_collect_packet<true, false, false, 1, kLeafPointMajor><<<grid, threads, 0, s>>>(C)
            : k_collect_packet<false, false, false, 6, kLeafPointMajor><<<grid, threads, 0, s>>>(C);
    else if (tuning().traversal == 4)
      stats ? k_collect_packet<true, false, false, 1, kLeafHybrid><<<grid, threads, 0, s>>>(C)
            : k_collect_packet<false, false, false, 6, kLeafHybrid><<<grid, threads, 0, s>>>(C);
    else if (stats)
      cube ? k_collect_packet<true, true, false, 1><<<grid, threads, 0, s>>>(C)
           : k_collect_packet<true, false, false, 1><<<grid, threads, 0, s>>>(C);
    else
      cube ? k_collect_packet<false, true, false, 6><<<grid, threads, 0, s>>>(C)
           : k_collect_packet<false, false, false, 7><<<grid, threads, 0, s>>>(C);
  } else {
    if (stats)
      k_collect<true><<<div_up(nq, threads), threads, 0, s>>>(C);
    else
      k_collect<false><<<div_up(nq, threads), threads, 0, s>>>(C);
  }
  RTDL_LAUNCHED(1);
}

// Buffers of the device-driven refinement (worst case: every processing rank).
struct RefineDevice {
  uint32_t* work[2];
  double *rad[2], *lo[2], *hi[2], *frad[2];
  uint32_t* full[2];
  uint32_t *cnt, *gen_qin, *gen_m;
  double* gen_rad;
  unsigned int* pass_count;  // kRefinePasses: work left after each pass (after the last: the generic count)
};

// The radius refinement without host reads (captured graphs): every pass is
// launched, each kernel reads its work count on the device and strides over it,
// and both walk
// forms are launched (the one the host-driven loop would not pick exits).
// small[0] holds the collect pass's heavy count; D.pass_count[kRefinePasses-1]
// ends with the number of queries left for the generic path.
void enqueue_refine_device(const CollectParams& C, const uint32_t* qprob, const double* prob_radius, double radius,
                           const uint32_t* prob_kmax, uint32_t kmax, uint32_t nproc, bool one_scene,
                           QueryInfo* qinfo, uint8_t* flags, unsigned int* small, const RefineDevice& D,
                           cudaStream_t s) {
  RTDL_CUDA_CHECK(cudaMemsetAsync(D.pass_count, 0, sizeof(unsigned int) * kRefinePasses, s));
  k_refine_init<<<kSmCount * 4, 256, 0, s>>>(C.heavy_list, C.heavy_m, C.heavy_t, 0, qprob, prob_radius, radius,
                                             prob_kmax, kmax, D.work[0], D.rad[0], D.lo[0], D.hi[0], D.full[0],
                                             D.frad[0], small);
  RTDL_LAUNCHED(1);
  int cur = 0;
  for (int pass = 0; pass < kRefinePasses; ++pass) {
    const unsigned int* n_dev = pass == 0 ? small : D.pass_count + pass - 1;
    RefineParams R;
    R.C = C;
    R.qprob = qprob;
    R.work = D.work[cur];
    R.rad = D.rad[cur];
    R.nwork = 0;
    R.cnt = D.cnt;
    R.nwork_dev = n_dev;
    R.packet_min = nproc / 8;  // the host-driven loop's choice between the two forms
    if (one_scene)
      k_collect_refine_packet_scene<<<kStrideBlocks, 256, 0, s>>>(R);
    else
      k_collect_refine_packet<<<kStrideBlocks, 256, 0, s>>>(R);
    k_collect_refine<<<kStrideBlocks, 256, 0, s>>>(R);
    RefineUpdate U;
    U.qorder = C.qorder;
    U.qprob = qprob;
    U.prob_kmax = prob_kmax;
    U.kmax = kmax;
    U.qinfo = qinfo;
    U.flags = flags;
    U.mid_list = C.mid_list;
    U.big_list = C.big_list;
    U.small = small;
    U.work = D.work[cur];
    U.rad = D.rad[cur];
    U.lo = D.lo[cur];
    U.hi = D.hi[cur];
    U.full = D.full[cur];
    U.frad = D.frad[cur];
    U.cnt = D.cnt;
    U.nwork = 0;
    U.next_work = D.work[cur ^ 1];
    U.next_rad = D.rad[cur ^ 1];
    U.next_lo = D.lo[cur ^ 1];
    U.next_hi = D.hi[cur ^ 1];
    U.next_full = D.full[cur ^ 1];
    U.next_frad = D.frad[cur ^ 1];
    U.next_count = D.pass_count + pass;
    U.generic_qin = D.gen_qin;
    U.generic_m = D.gen_m;
    U.generic_rad = D.gen_rad;
    U.last = pass == kRefinePasses - 1 ? 1 : 0;
    U.nwork_dev = n_dev;
    k_refine_update<<<kSmCount * 4, 256, 0, s>>>(U);
    RTDL_LAUNCHED(3);
    cur ^= 1;
  }
}

void check_readback(const Readback& r) {
  throw_if_bad(r.scene_bad | r.query_bad);
  if (r.error & 1u) throw std::runtime_error("BVH traversal stack overflow");
}

// fixed_radius_neighbors / bounded_knn_rows: collect, scan, emit.
QueryResult run_radius_query(Scene* sc, const void* queries_dev, uint32_t nq, int predicate, double radius,
                             uint32_t kmax, void* rows_dev, size_t rows_capacity, void** rows_alloc,
                             uint8_t* overflow_dev, cudaStream_t s, PhaseTimer* timer, const BatchSpec* bs = nullptr,
                             const SummarySpec* ss = nullptr, const PreparedQueries* pq = nullptr,
                             bool witness = false, RowDownload* dl = nullptr) {
  // witness (k_max 1): one row per query at its input position, pre-filled
  // with the no-witness row; the nearest in-radius neighbour overwrites it.
  QueryResult res;
  void* summary_rows = nullptr;  // ranked summaries: the rows stay internal
  if (ss) rows_alloc = &summary_rows;
  if (pq) queries_dev = pq->raw;
  const int qstride = sc->dim == 3 ? 4 : 3;
  if (bs) {  // the largest kmax bounds the generic path's output
    kmax = 1;
    for (uint32_t p = 0; p < bs->problems; ++p) kmax = bs->kmax[p] > kmax ? bs->kmax[p] : kmax;
  }
  QueryPrep qp = pq   ? borrow_prepared(sc, pq, radius, s)
                 : bs ? prepare_queries_batch(sc, queries_dev, nq, *bs, s)
                      : prepare_queries(sc, queries_dev, nq, true, radius, true, s);
  const uint32_t np = qp.nproc;  // processing ranks
  const size_t nq1 = nq ? nq : 1, np1 = np ? np : 1;
  uint32_t* qrank = pq ? pq->qrank : static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq1, s));
  if (!pq) {
    k_invert<<<grid_for(nq, 256), 256, 0, s>>>(qp.oorder, nq, qp.order_identity, qrank);
    RTDL_LAUNCHED(1);
  }
  if (timer) timer->mark("query_prep");
  unsigned long long* slab =
      static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * slab_base((uint32_t)np1), s));
  uint32_t* counts = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq1, s));
  QueryInfo* qinfo = static_cast<QueryInfo*>(dev_alloc(sizeof(QueryInfo) * np1, s));
  uint8_t* flags = static_cast<uint8_t*>(dev_alloc(nq1, s));
  uint32_t* heavy_list = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq1, s));
  uint32_t* heavy_m = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq1, s));
  uint32_t* heavy_t = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq1, s));
  uint32_t* mid_list = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * np1, s));
  uint32_t* big_list = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * np1, s));
  uint32_t* fix_list = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * np1, s));
  unsigned int* small = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int) * 8, s));
  unsigned long long* offsets = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (nq + 1), s));
  unsigned long long* poff = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * np1, s));
  unsigned long long* prob_rows =
      bs ? static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (bs->problems + 1), s)) : nullptr;
  RTDL_CUDA_CHECK(cudaMemsetAsync(small, 0, sizeof(unsigned int) * 8, s));
  GenericOut g;
  std::vector<void*> refine_bufs;
  auto cleanup = [&]() {
    g.release(s);
    for (void* p : refine_bufs) dev_free(p, s);
    dev_free(prob_rows, s);
    dev_free(poff, s);
    if (!pq) dev_free(qrank, s);
    dev_free(slab, s);
    dev_free(counts, s);
    dev_free(qinfo, s);
    dev_free(flags, s);
    dev_free(heavy_list, s);
    dev_free(heavy_m, s);
    dev_free(heavy_t, s);
    dev_free(mid_list, s);
    dev_free(big_list, s);
    dev_free(fix_list, s);
    dev_free(small, s);
    dev_free(offsets, s);
    free_prep(qp, s);
  };
  try {
    CollectParams C;
    C.S = qp.view;
    C.qpts = qp.qpts;
    C.qraw = static_cast<const double*>(queries_dev);
    C.qstride = qstride;
    C.qorder = qp.qorder;
    C.nq = np;
    C.kmax = kmax;
    C.bands = qp.bands;
    C.warp_prob = qp.warp_prob;
    C.prob_kmax = qp.prob_kmax;
    C.slab = slab;
    C.counts = counts;
    C.qinfo = qinfo;
    C.flags = flags;
    C.heavy_list = heavy_list;
    C.heavy_m = heavy_m;
    C.heavy_t = heavy_t;
    C.mid_list = mid_list;
    C.big_list = big_list;
    C.small = small;
    C.overflow_out = overflow_dev;
    C.stats = nullptr;
    const bool stats = stats_enabled();
    if (stats) {
      C.stats = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * kStatCount, s));
      RTDL_CUDA_CHECK(cudaMemsetAsync(C.stats, 0, sizeof(unsigned long long) * kStatCount, s));
    }
    if (timer) timer->mark("setup");
    launch_collect(C, np, nq, bs != nullptr, stats, s);
    if (stats) {
      RTDL_CUDA_CHECK(cudaMemcpyAsync(last_stats().data(), C.stats, sizeof(unsigned long long) * kStatCount,
                                      cudaMemcpyDeviceToHost, s));
      dev_free(C.stats, s);
    }
    if (timer) timer->mark("traverse");
    if (witness) {
      k_witness_offsets<<<grid_for(nq + 1, 256), 256, 0, s>>>(qp.oorder, qp.order_identity, nq, offsets);
      RTDL_LAUNCHED(1);
    } else {
      scan_counts_u64(counts, qp.oorder, qp.order_identity, nq, offsets, s);
    }
    if (bs) {
      k_problem_rows<<<div_up(bs->problems + 1, 256), 256, 0, s>>>(offsets, qp.qoff, bs->problems, prob_rows);
      RTDL_LAUNCHED(1);
      RTDL_CUDA_CHECK(cudaMemcpyAsync(bs->row_offsets, prob_rows, sizeof(unsigned long long) * (bs->problems + 1),
                                      cudaMemcpyDeviceToHost, s));
    }
    if (timer) timer->mark("scan");
    auto launch_expand = [&](uint32_t n_generic, const uint32_t* list) {
      ExpandParams X;
      X.S = sc->view();
      X.qpts = qp.qpts;
      X.qraw = static_cast<const double*>(queries_dev);
      X.qstride = qstride;
      X.oorder = qp.oorder;
      X.bands = qp.bands;
      X.nq = n_generic;
      X.L = kSlab;
      X.counts = counts;
      X.flags = flags;
      X.temp = nullptr;  // unused with a work list
      X.heavy_out = g.heavy_out;
      X.heavy_out_off = g.heavy_out_off;
      X.offsets = offsets;
      X.rows = rows_dev;
      X.capacity = rows_dev ? rows_capacity : 0;
      X.ranked = predicate == kFrn ? 0 : 1;
      X.overflow_out = nullptr;
      X.error = small + 1;
      X.work_list = list;
      X.qrank = qrank;
      k_expand<32><<<grid_for((uint64_t)n_generic * 32, kExpandThreads), kExpandThreads, 0, s>>>(X);
      RTDL_LAUNCHED(1);
    };
    // Rows only counted: the total is known after the scan (no refinement, no emit).
    const bool count_only = rows_alloc == nullptr && rows_dev == nullptr && !bs && !ss && !witness;
    Readback* rb = pinned_readback();
    if (count_only) {
      SmallReads reads(rb);
      reads.add(&rb->rows, offsets + nq, sizeof(unsigned long long));
      reads.add(&rb->heavy, small, sizeof(unsigned int) * 4);
      reads.add(&rb->scene_bad, &sc->stats->bad, sizeof(unsigned int));
      reads.add(&rb->query_bad, &qp.qst->bad, sizeof(unsigned int));
      reads.launch(s);
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      check_readback(*rb);
      res.rows = rb->rows;
    } else {
      // rows copied to the host range by range as they are emitted
      bool chunked = dl != nullptr && (dl->alloc != nullptr || dl->host_fixed != nullptr) && rows_alloc != nullptr &&
                     !bs && !ss && !witness &&
                     nq >= (uint32_t)kDownloadChunks * 1024u;
      SmallReads reads(rb);
      if (chunked) {
        unsigned long long* chunk_dev =
            static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (kDownloadChunks + 1), s));
        refine_bufs.push_back(chunk_dev);
        k_chunk_rows<<<1, 32, 0, s>>>(offsets, nq, kDownloadChunks, chunk_dev);
        RTDL_LAUNCHED(1);
        reads.add(rb->chunk_rows, chunk_dev, sizeof(unsigned long long) * (kDownloadChunks + 1));
      }
      reads.add(&rb->rows, offsets + nq, sizeof(unsigned long long));
      reads.add(&rb->heavy, small, sizeof(unsigned int) * 4);
      reads.add(&rb->scene_bad, &sc->stats->bad, sizeof(unsigned int));
      reads.add(&rb->query_bad, &qp.qst->bad, sizeof(unsigned int));
      reads.launch(s);
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      const Readback r = *rb;
      check_readback(r);
      res.rows = r.rows;
      if (res.rows == 0) chunked = false;
      uint32_t mid = r.mid, big = r.big, generic = r.heavy;
      const uint32_t* generic_list = heavy_list;
      const uint32_t* generic_m = heavy_m;
      const double* generic_rad = nullptr;
      auto emit_params = [&]() {
        EmitParams E;
        E.S = sc->view();
        E.nq = np;
        E.slab = slab;
        E.qinfo = qinfo;
        E.poff = poff;
        E.sink.rows = rows_dev;
        E.sink.capacity = rows_dev ? rows_capacity : 0;
        E.sink.ranked = predicate == kFrn ? 0 : 1;
        E.fix_list = fix_list;
        E.fix_count = small + 4;
        return E;
      };
      if (r.heavy > 0 && rows_alloc == nullptr && !witness) {
        // Rows into a given device buffer: the emit does not wait for the heavy
        // queries.  Three streams: the list kernels of the collect's 65..kSlab
        // candidate queries (their counts are final) are queued first on the
        // second stream, the first refinement pass on the third, then k_emit
        // on this one; the refinement's later passes (each reads its count
        // back to the host), the generic path and the list kernels of the
        // queries it resolved follow on the third stream.  k_emit skips a
        // heavy query whichever of its records it reads: the collect marked
        // it generic, the pass that resolves it marks it for a list kernel
        // and appends it to a list after the collect's entries.
        cudaStream_t ls = aux_stream(0), rs = aux_stream(1);
        static thread_local cudaEvent_t ev_offsets = nullptr, ev_lists = nullptr, ev_refined = nullptr;
        if (!ev_offsets) {
          RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_offsets, cudaEventDisableTiming));
          RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_lists, cudaEventDisableTiming));
          RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_refined, cudaEventDisableTiming));
        }
        k_proc_offsets<<<grid_for(np, 256), 256, 0, s>>>(qp.qorder, qrank, offsets, np, poff);
        RTDL_LAUNCHED(1);
        RTDL_CUDA_CHECK(cudaEventRecord(ev_offsets, s));
        RTDL_CUDA_CHECK(cudaStreamWaitEvent(ls, ev_offsets, 0));
        RTDL_CUDA_CHECK(cudaStreamWaitEvent(rs, ev_offsets, 0));
        const EmitParams E = emit_params();
        auto launch_lists = [&](uint32_t first_mid, uint32_t n_mid, uint32_t first_big, uint32_t n_big,
                                cudaStream_t st) {
          if (n_mid > 0) {
            k_emit_list<4, true><<<div_up((uint64_t)n_mid * 32, kEmitListThreads), kEmitListThreads, 0, st>>>(
                E, mid_list + first_mid, n_mid, nullptr);
            RTDL_LAUNCHED(1);
          }
          if (n_big > 0) {
            k_emit_list<8, false><<<div_up((uint64_t)n_big * 32, kEmitListThreads), kEmitListThreads, 0, st>>>(
                E, big_list + first_big, n_big, nullptr);
            RTDL_LAUNCHED(1);
          }
        };
        launch_lists(0, r.mid, 0, r.big, ls);
        RTDL_CUDA_CHECK(cudaEventRecord(ev_lists, ls));
        RefineOut ro = refine_heavy(C, qp, radius, kmax, r.heavy, heavy_list, heavy_m, heavy_t, qinfo, flags, mid_list,
                                    big_list, small, rs, [&]() {
                                      k_emit<<<emit_grid(np), kEmitThreads, 0, s>>>(E);
                                      RTDL_LAUNCHED(1);
                                    });
        refine_bufs = ro.buffers;
        generic = ro.generic;
        res.heavy = generic;
        if (stats) {
          last_stats()[kStatGenericQueries] = generic;
          last_stats()[kStatLargeQueries] = ro.mid + ro.big;
          last_stats()[kStatRefined] = r.heavy - generic;
        }
        // the gather is bounded by each query's smallest tested radius that holds its rows
        if (generic > 0)
          g = run_generic_path(sc, qp, queries_dev, qstride, generic, ro.generic_qin, ro.generic_m, kmax, false,
                               small + 1, rs, ro.generic_rad);
        launch_lists(r.mid, ro.mid - r.mid, r.big, ro.big - r.big, rs);
        RTDL_CUDA_CHECK(cudaEventRecord(ev_refined, rs));
        RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ev_lists, 0));
        RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ev_refined, 0));
        k_emit_fixup<<<kSmCount * 4, kFixupThreads, 0, s>>>(E);
        RTDL_LAUNCHED(1);
        if (generic > 0) launch_expand(generic, ro.generic_qin);
        if (timer) timer->mark("emit");
        SmallReads end_reads(rb);
        end_reads.add(&rb->error, small + 1, sizeof(unsigned int));
        end_reads.add(&rb->fixups, small + 4, sizeof(unsigned int));
        end_reads.launch(s);
        RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
        if (stats) last_stats()[kStatEmitFixups] = rb->fixups;
        if (rb->error & 6u) throw std::runtime_error("generic neighbor path produced an inconsistent candidate count");
      } else {
        if (r.heavy > 0) {
          // queries with more than kSlab points in radius: collect again at smaller radii
          RefineOut ro = refine_heavy(C, qp, radius, kmax, r.heavy, heavy_list, heavy_m, heavy_t, qinfo, flags, mid_list,
                                      big_list, small, s);
          refine_bufs = ro.buffers;
          generic = ro.generic;
          generic_list = ro.generic_qin;
          generic_m = ro.generic_m;
          generic_rad = ro.generic_rad;
          mid = ro.mid;
          big = ro.big;
          if (timer) timer->mark("refine");
        }
        res.heavy = generic;
        if (stats) {
          last_stats()[kStatGenericQueries] = generic;
          last_stats()[kStatLargeQueries] = mid + big;
          last_stats()[kStatRefined] = r.heavy - generic;
        }
        if (generic > 0) {
          // the gather is bounded by each query's smallest tested radius that holds its rows
          g = run_generic_path(sc, qp, queries_dev, qstride, generic, generic_list, generic_m, kmax, false, small + 1, s,
                               generic_rad);
          if (timer) timer->mark("generic_path");
        }
        if (rows_alloc != nullptr) {
          const size_t row_size = predicate == kFrn ? 16 : 24;
          rows_dev = res.rows ? dev_alloc(row_size * res.rows, s) : nullptr;
          rows_capacity = res.rows;
          *rows_alloc = rows_dev;
        }
        if (witness && rows_dev) {
          k_witness_fill<<<grid_for(nq, 256), 256, 0, s>>>(qp.qpts, nq, static_cast<RtdlFixedRadiusNeighborRow*>(rows_dev),
                                                           rows_capacity);
          RTDL_LAUNCHED(1);
        }
        k_proc_offsets<<<grid_for(np, 256), 256, 0, s>>>(qp.qorder, qrank, offsets, np, poff);
        RTDL_LAUNCHED(1);
        if (chunked) {
          const size_t row_size = predicate == kFrn ? 16 : 24;
          if (dl->host_fixed) {
            dl->host = dl->host_fixed;
            dl->pinned = true;
          } else {
            dl->host = dl->alloc(row_size * res.rows, &dl->pinned);
          }
        }
        EmitParams E = emit_params();
        if (chunked) {
          // Range by range in output order: each range's queries are emitted
          // (the list kernels and k_emit skip queries outside it), its deferred
          // queries fixed up, and the copy of its rows queued on the copy
          // stream, which overlaps the emission of the ranges after it.  The
          // generic queries' rows are written first.
          if (generic > 0) launch_expand(generic, generic_list);
          uint32_t* eorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq1, s));
          refine_bufs.push_back(eorder);
          k_emit_order<<<grid_for(np, 256), 256, 0, s>>>(qp.qorder, qrank, np, eorder);
          RTDL_LAUNCHED(1);
          // the two list kernels' work, partitioned by range (list lengths in small[2], small[3])
          constexpr uint32_t C = kDownloadChunks, kPart = 3 * C + 1;
          unsigned int* part = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int) * 2 * kPart, s));
          refine_bufs.push_back(part);
          RTDL_CUDA_CHECK(cudaMemsetAsync(part, 0, sizeof(unsigned int) * 2 * kPart, s));
          uint32_t* lists_by_range[2] = {nullptr, nullptr};
          const uint32_t list_len[2] = {mid, big};
          uint32_t* lists[2] = {mid_list, big_list};
          for (int l = 0; l < 2; ++l) {
            if (list_len[l] == 0) continue;
            lists_by_range[l] = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * list_len[l], s));
            refine_bufs.push_back(lists_by_range[l]);
            const unsigned int grid = grid_for(list_len[l], 256);
            k_range_count<<<grid, 256, 0, s>>>(lists[l], small + 2 + l, qp.qorder, qrank, nq, C, part + l * kPart);
            k_range_starts<<<1, 1, 0, s>>>(C, part + l * kPart);
            k_range_scatter<<<grid, 256, 0, s>>>(lists[l], small + 2 + l, qp.qorder, qrank, nq, C, part + l * kPart,
                                                 lists_by_range[l]);
            RTDL_LAUNCHED(3);
          }
          E.order = eorder;
          E.fix_begin = small + 5;
          static thread_local cudaEvent_t ev_range[kDownloadChunks] = {};
          unsigned long long first[kDownloadChunks + 1];
          for (int c = 0; c <= kDownloadChunks; ++c) first[c] = r.chunk_rows[c];
          if (first[kDownloadChunks] != res.rows) throw std::runtime_error("row ranges disagree with the row count");
          const size_t row_size = predicate == kFrn ? 16 : 24;
          for (int c = 0; c < (int)C; ++c) {
            if (first[c + 1] == first[c]) continue;  // no rows in this range
            E.out_lo = (uint32_t)((uint64_t)nq * (uint32_t)c / C);
            E.out_hi = (uint32_t)((uint64_t)nq * (uint32_t)(c + 1) / C);
            E.range = c;
            // the list kernels stride over the range's part: grids sized for an even split
            if (mid > 0) {
              E.list_start = part + C;
              k_emit_list<4, true><<<div_up((uint64_t)div_up(mid, C) * 32, kEmitListThreads), kEmitListThreads, 0, s>>>(
                  E, lists_by_range[0], 0, nullptr);
            }
            if (big > 0) {
              E.list_start = part + kPart + C;
              k_emit_list<8, false><<<div_up((uint64_t)div_up(big, C) * 32, kEmitListThreads), kEmitListThreads, 0,
                                      s>>>(E, lists_by_range[1], 0, nullptr);
            }
            E.list_start = nullptr;
            k_emit<<<emit_grid(E.out_hi - E.out_lo), kEmitThreads, 0, s>>>(E);
            k_emit_fixup<<<kSmCount * 4, kFixupThreads, 0, s>>>(E);
            k_fix_advance<<<1, 1, 0, s>>>(small + 5, small + 4);
            RTDL_LAUNCHED(5);
            if (!ev_range[c]) RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_range[c], cudaEventDisableTiming));
            RTDL_CUDA_CHECK(cudaEventRecord(ev_range[c], s));
            RTDL_CUDA_CHECK(cudaStreamWaitEvent(dl->copy, ev_range[c], 0));
            RTDL_CUDA_CHECK(cudaMemcpyAsync(static_cast<char*>(dl->host) + first[c] * row_size,
                                            static_cast<const char*>(rows_dev) + first[c] * row_size,
                                            (first[c + 1] - first[c]) * row_size, cudaMemcpyDeviceToHost, dl->copy));
            ++dl->copies;
          }
          if (timer) timer->mark("emit");
          SmallReads end_reads(rb);
          end_reads.add(&rb->error, small + 1, sizeof(unsigned int));
          end_reads.add(&rb->fixups, small + 4, sizeof(unsigned int));
          end_reads.launch(s);
          RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
          if (stats) last_stats()[kStatEmitFixups] = rb->fixups;
          if (rb->error & 6u) throw std::runtime_error("generic neighbor path produced an inconsistent candidate count");
          cleanup();
          return res;
        }
        // The list kernels (queries with 65..kSlab candidates: few warps, long
        // sorts) run on the second stream beside k_emit, so each fills the
        // other's partial waves; they write disjoint rows, and the fix-up waits
        // for both.
        static thread_local cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
        const bool side = mid > 0 || big > 0;
        cudaStream_t ls = s;
        if (side) {
          if (!ev_fork) {
            RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
            RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
          }
          ls = aux_stream();
          RTDL_CUDA_CHECK(cudaEventRecord(ev_fork, s));
          RTDL_CUDA_CHECK(cudaStreamWaitEvent(ls, ev_fork, 0));
        }
        if (mid > 0) {
          k_emit_list<4, true><<<div_up((uint64_t)mid * 32, kEmitListThreads), kEmitListThreads, 0, ls>>>(E, mid_list,
                                                                                                       mid, nullptr);
          RTDL_LAUNCHED(1);
        }
        if (big > 0) {
          k_emit_list<8, false><<<div_up((uint64_t)big * 32, kEmitListThreads), kEmitListThreads, 0, ls>>>(E, big_list,
                                                                                                        big, nullptr);
          RTDL_LAUNCHED(1);
        }
        k_emit<<<emit_grid(np), kEmitThreads, 0, s>>>(E);
        RTDL_LAUNCHED(1);
        if (side) {
          RTDL_CUDA_CHECK(cudaEventRecord(ev_join, ls));
          RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ev_join, 0));
        }
        k_emit_fixup<<<kSmCount * 4, kFixupThreads, 0, s>>>(E);
        RTDL_LAUNCHED(1);
        if (generic > 0) {
          launch_expand(generic, generic_list);
        }
        if (timer) timer->mark("emit");
        SmallReads end_reads(rb);
        end_reads.add(&rb->error, small + 1, sizeof(unsigned int));
        end_reads.add(&rb->fixups, small + 4, sizeof(unsigned int));
        end_reads.launch(s);
        RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
        if (stats) last_stats()[kStatEmitFixups] = rb->fixups;
        if (rb->error & 6u) throw std::runtime_error("generic neighbor path produced an inconsistent candidate count");
      }
    }
    if (ss) {
      const uint32_t blocks = div_up((uint64_t)nq * 32, kSummaryThreads);
      SummaryPartial* partial = static_cast<SummaryPartial*>(dev_alloc(sizeof(SummaryPartial) * blocks, s));
      RtdlFixedRadiusRankedNeighborAggregate* agg = static_cast<RtdlFixedRadiusRankedNeighborAggregate*>(
          dev_alloc(sizeof(RtdlFixedRadiusRankedNeighborAggregate), s));
      k_summarize<<<blocks, kSummaryThreads, 0, s>>>(static_cast<const RtdlFixedRadiusNeighborRow*>(summary_rows),
                                                    offsets, qp.oorder, qp.order_identity, qp.qpts, nq,
                                                    ss->summaries_dev, partial);
      k_summary_final<<<1, 1024, 0, s>>>(partial, blocks, nq, agg);
      RTDL_LAUNCHED(2);
      RTDL_CUDA_CHECK(cudaMemcpyAsync(ss->aggregate_host, agg, sizeof(*agg), cudaMemcpyDeviceToHost, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      dev_free(partial, s);
      dev_free(agg, s);
      if (timer) timer->mark("summarize");
    }
  } catch (...) {
    sync_quietly(s);
    sync_quietly(aux_stream(0));  // the refinement and the list kernels may run there
    sync_quietly(aux_stream(1));
    dev_free(summary_rows, s);
    cleanup();
    throw;
  }
  dev_free(summary_rows, s);
  cleanup();
  return res;
}

}  // namespace

QueryResult run_ranked_summaries(Scene* sc, const void* queries_dev, uint32_t nq, double radius, uint32_t kmax,
                                 RtdlFixedRadiusRankedNeighborSummary* summaries_dev,
                                 RtdlFixedRadiusRankedNeighborAggregate* aggregate_host, cudaStream_t s,
                                 PhaseTimer* timer, const PreparedQueries* pq) {
  if (pq) {
    if (pq->dim != sc->dim) throw std::runtime_error("prepared queries and scene differ in dimension");
    nq = pq->n;
  }
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  if (kmax < 1 || kmax > 64)
    throw std::runtime_error("prepared ranked fixed_radius_neighbors_3d aggregate currently supports k_max <= 64");
  *aggregate_host = RtdlFixedRadiusRankedNeighborAggregate{nq, 0u, 0u, 0u, 0.0};
  if (nq == 0) return QueryResult{};
  // an empty search set gives no summaries and a zero aggregate, as the
  // reference's wrappers do (optix_runtime.py:2555-2572, 2644-2651)
  if (sc->n == 0) return QueryResult{};
  if (timer) timer->mark("start");
  SummarySpec ss{summaries_dev, aggregate_host};
  return run_radius_query(sc, queries_dev, nq, kFrn, radius, kmax, nullptr, 0, nullptr, nullptr, s, timer, nullptr,
                          &ss, pq);
}

QueryResult run_query_prepared(Scene* sc, const PreparedQueries* pq, double radius, uint32_t kmax, void* rows_dev,
                               size_t rows_capacity, uint8_t* overflow_dev, cudaStream_t s, PhaseTimer* timer) {
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  if (pq->dim != sc->dim) throw std::runtime_error("prepared queries and scene differ in dimension");
  if (kmax < 1 || kmax > (uint32_t)kMaxList) throw std::runtime_error("prepared queries take k_max in [1, 64]");
  if (pq->n == 0) return QueryResult{};
  if (sc->n == 0) {
    if (overflow_dev) RTDL_CUDA_CHECK(cudaMemsetAsync(overflow_dev, 0, pq->n, s));
    return QueryResult{};
  }
  if (timer) timer->mark("start");
  return run_radius_query(sc, pq->raw, pq->n, kFrn, radius, kmax, rows_dev, rows_capacity, nullptr, overflow_dev, s,
                          timer, nullptr, nullptr, pq);
}

namespace {
// SoA point columns (partner-owned device buffers) -> RtdlPoint records.
__global__ void k_columns_to_records_2d(const uint32_t* ids, const double* x, const double* y, uint32_t n,
                                        RtdlPoint* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = RtdlPoint{ids[i], x[i], y[i]};
}
}  // namespace

void columns_to_records_2d(const uint32_t* ids, const double* x, const double* y, uint32_t n, void* out,
                           cudaStream_t s) {
  if (n == 0) return;
  k_columns_to_records_2d<<<grid_for(n, 256), 256, 0, s>>>(ids, x, y, n, static_cast<RtdlPoint*>(out));
  RTDL_LAUNCHED(1);
}

// ---- count with threshold, nearest witness --------------------------------------
namespace {
// The count (or, with nearest_rows, the point-group witness) walk over a scene;
// group_of / group_boxes restrict candidates to groups whose box is in radius.
void count_walk(Scene* sc, const void* queries_dev, uint32_t nq, double radius, uint32_t threshold,
                const CountOutputs& out, const uint32_t* group_of, const double* group_boxes,
                RtdlFixedRadiusNeighborRow* nearest_rows, cudaStream_t s) {
  if (nq == 0) return;
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  QueryPrep qp = prepare_queries(sc, queries_dev, nq, true, radius, false, s);
  unsigned long long* reached = nullptr;
  try {
    if (out.reached_host) {
      reached = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long), s));
      RTDL_CUDA_CHECK(cudaMemsetAsync(reached, 0, sizeof(unsigned long long), s));
    }
    CountParams P;
    P.S = sc->view();
    P.qpts = qp.qpts;
    P.qraw = static_cast<const double*>(queries_dev);
    P.qstride = sc->dim == 3 ? 4 : 3;
    P.qorder = qp.qorder;
    P.nq = nq;
    P.bands = qp.bands;
    P.threshold = threshold;
    P.ids_out = out.ids;
    P.counts_out = out.counts;
    P.flags_out = out.flags;
    P.rows_out = out.rows;
    P.reached = reached;
    P.group_of = group_of;
    P.group_boxes = group_boxes;
    if (nearest_rows)
      k_group_nearest_packet<<<div_up(nq, 256), 256, 0, s>>>(P, nearest_rows);
    else
      k_count_packet<<<div_up(nq, 256), 256, 0, s>>>(P);
    RTDL_LAUNCHED(1);
    Readback* rb = pinned_readback();
    RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->scene_bad, &sc->stats->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->query_bad, &qp.qst->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    if (reached)
      RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->rows, reached, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    check_readback(*rb);
    if (out.reached_host) *out.reached_host = rb->rows;
  } catch (...) {
    sync_quietly(s);
    dev_free(reached, s);
    free_prep(qp, s);
    throw;
  }
  dev_free(reached, s);
  free_prep(qp, s);
}
}  // namespace

void run_count_threshold(Scene* sc, const void* queries_dev, uint32_t nq, double radius, uint32_t threshold,
                         const CountOutputs& out, cudaStream_t s) {
  count_walk(sc, queries_dev, nq, radius, threshold, out, nullptr, nullptr, nullptr, s);
}

PointGroupScene* point_group_create(const RtdlPoint* points, size_t count, const RtdlPointGroupBounds2D* groups,
                                    size_t group_count, double max_radius, int leaf_size, cudaStream_t s) {
  size_t total = 0;
  for (size_t g = 0; g < group_count; ++g) {
    const RtdlPointGroupBounds2D& G = groups[g];
    if ((size_t)G.point_offset > count || (size_t)G.point_count > count - (size_t)G.point_offset)
      throw std::runtime_error("point_group_nearest_witness group span exceeds search point count");
    if (G.max_x < G.min_x || G.max_y < G.min_y)
      throw std::runtime_error("point_group_nearest_witness group bounds must be ordered");
    total += G.point_count;
  }
  if (total > (size_t)kMaxScenePoints) throw std::runtime_error("point groups reference more than 67,108,864 points");
  // the scene holds every group's points (a point in two groups twice), each tagged with its group
  std::vector<RtdlPoint> expanded(total);
  std::vector<uint32_t> group_of(total);
  std::vector<double> boxes(4 * group_count);
  size_t k = 0;
  for (size_t g = 0; g < group_count; ++g) {
    const RtdlPointGroupBounds2D& G = groups[g];
    for (uint32_t i = 0; i < G.point_count; ++i, ++k) {
      expanded[k] = points[G.point_offset + i];
      group_of[k] = (uint32_t)g;
    }
    boxes[4 * g] = G.min_x;
    boxes[4 * g + 1] = G.min_y;
    boxes[4 * g + 2] = G.max_x;
    boxes[4 * g + 3] = G.max_y;
  }
  PointGroupScene* pg = new PointGroupScene();
  pg->groups = (uint32_t)group_count;
  pg->points = (uint32_t)total;
  pg->max_radius = max_radius;
  void* d_pts = nullptr;
  try {
    d_pts = dev_alloc(sizeof(RtdlPoint) * (total ? total : 1), s);
    pg->group_of = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (total ? total : 1), s));
    pg->boxes = static_cast<double*>(dev_alloc(sizeof(double) * (boxes.empty() ? 4 : boxes.size()), s));
    if (total) {
      RTDL_CUDA_CHECK(cudaMemcpyAsync(d_pts, expanded.data(), sizeof(RtdlPoint) * total, cudaMemcpyHostToDevice, s));
      RTDL_CUDA_CHECK(cudaMemcpyAsync(pg->group_of, group_of.data(), sizeof(uint32_t) * total, cudaMemcpyHostToDevice,
                                      s));
    }
    if (!boxes.empty())
      RTDL_CUDA_CHECK(cudaMemcpyAsync(pg->boxes, boxes.data(), sizeof(double) * boxes.size(), cudaMemcpyHostToDevice, s));
    pg->sc = build_scene(d_pts, (uint32_t)total, 2, s, leaf_size);
    unsigned int bad = 0;
    RTDL_CUDA_CHECK(cudaMemcpyAsync(&bad, &pg->sc->stats->bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // the host vectors stay alive until the copies are done
    throw_if_bad(bad);
  } catch (...) {
    sync_quietly(s);
    dev_free(d_pts, s);
    point_group_destroy(pg);
    throw;
  }
  dev_free(d_pts, s);
  return pg;
}

void point_group_destroy(PointGroupScene* pg) {
  if (!pg) return;
  cudaStream_t s = pg->sc ? pg->sc->stream : nullptr;
  dev_free(pg->group_of, s);
  dev_free(pg->boxes, s);
  destroy_scene(pg->sc);
  if (s) cudaStreamSynchronize(s);
  delete pg;
}

void point_group_count(PointGroupScene* pg, const void* queries_dev, uint32_t nq, double radius, uint32_t threshold,
                       const CountOutputs& out, cudaStream_t s) {
  count_walk(pg->sc, queries_dev, nq, radius, threshold, out, pg->group_of, pg->boxes, nullptr, s);
}

void point_group_nearest(PointGroupScene* pg, const void* queries_dev, uint32_t nq, double radius,
                         RtdlFixedRadiusNeighborRow* rows_dev, RtdlFixedRadiusNeighborRow* max_row_host,
                         cudaStream_t s) {
  count_walk(pg->sc, queries_dev, nq, radius, 0, CountOutputs{}, pg->group_of, pg->boxes, rows_dev, s);
  if (max_row_host) {
    RtdlFixedRadiusNeighborRow* d_max =
        static_cast<RtdlFixedRadiusNeighborRow*>(dev_alloc(sizeof(RtdlFixedRadiusNeighborRow), s));
    k_witness_max<<<1, 1024, 0, s>>>(rows_dev, nq, d_max);
    RTDL_LAUNCHED(1);
    RTDL_CUDA_CHECK(cudaMemcpyAsync(max_row_host, d_max, sizeof(RtdlFixedRadiusNeighborRow), cudaMemcpyDeviceToHost, s));
    dev_free(d_max, s);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  }
}

void run_count_trivial(const void* queries_dev, uint32_t nq, int dim, const CountOutputs& out, cudaStream_t s) {
  if (nq == 0) return;
  float4* qpts = static_cast<float4*>(dev_alloc(sizeof(float4) * nq, s));
  PointStats* st = static_cast<PointStats*>(dev_alloc(sizeof(PointStats), s));
  reset_stats(st, s);
  prep_points(queries_dev, nq, dim, qpts, st, s);
  k_count_trivial<<<grid_for(nq, 256), 256, 0, s>>>(qpts, nq, out.ids, out.counts, out.flags);
  RTDL_LAUNCHED(1);
  dev_free(qpts, s);
  dev_free(st, s);
}

QueryResult run_nearest_witness(Scene* sc, const void* queries_dev, uint32_t nq, double radius, void** rows_alloc,
                                cudaStream_t s, PhaseTimer* timer) {
  if (rows_alloc) *rows_alloc = nullptr;
  if (nq == 0 || sc->n == 0) return QueryResult{};
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  return run_radius_query(sc, queries_dev, nq, kFrn, radius, 1, nullptr, 0, rows_alloc, nullptr, s, timer, nullptr,
                          nullptr, nullptr, true);
}

// ---- the plain per-call form: build and query in one call ---------------------
QueryResult run_build_and_query(const BuildQueryInputs& in, int predicate, double radius, uint32_t limit,
                                void* rows_dev, size_t rows_capacity, void** rows_alloc, uint8_t* overflow_dev,
                                cudaStream_t s, cudaStream_t aux, PhaseTimer* timer, Scene** scene_out,
                                void** query_owned, RowDownload* download) {
  *scene_out = nullptr;
  *query_owned = nullptr;
  const size_t qbytes = (in.dim == 3 ? sizeof(RtdlPoint3D) : sizeof(RtdlPoint)) * (size_t)in.nq;
  const bool overlap = predicate != kKnn && limit <= (uint32_t)kMaxList && in.nq > 0 && in.ns > 0 && aux != nullptr;
  if (!overlap) {
    const void* q = in.query_dev;
    if (in.query_host && in.nq) {
      *query_owned = dev_alloc(qbytes, s);
      RTDL_CUDA_CHECK(cudaMemcpyAsync(*query_owned, in.query_host, qbytes, cudaMemcpyHostToDevice, s));
      q = *query_owned;
    }
    Scene* sc = build_scene(in.search_dev, in.ns, in.dim, s, scene_leaf_size());
    *scene_out = sc;
    if (timer) timer->mark("build");
    return run_query(sc, q, in.nq, predicate, radius, limit, rows_dev, rows_capacity, rows_alloc, overflow_dev, s,
                     timer);
  }
  // the query side does not need the scene until its bands: it is prepared on
  // `aux` (own-box Morton order) while the scene builds on `s`
  static thread_local cudaEvent_t ev_start = nullptr, ev_ready = nullptr;
  if (!ev_start) {
    RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming));
    RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_ready, cudaEventDisableTiming));
  }
  RTDL_CUDA_CHECK(cudaEventRecord(ev_start, s));
  RTDL_CUDA_CHECK(cudaStreamWaitEvent(aux, ev_start, 0));  // whatever the caller queued on s comes first
  Scene* sc = build_scene(in.search_dev, in.ns, in.dim, s, scene_leaf_size());
  *scene_out = sc;
  const void* q = in.query_dev;
  if (in.query_host) {  // a pageable copy holds the host; the build is already queued
    *query_owned = dev_alloc(qbytes, aux);
    RTDL_CUDA_CHECK(cudaMemcpyAsync(*query_owned, in.query_host, qbytes, cudaMemcpyHostToDevice, aux));
    q = *query_owned;
  }
  PreparedQueries* pq = nullptr;
  try {
    pq = prepare_query_set(q, in.nq, in.dim, aux);
  } catch (...) {
    sync_quietly(aux);
    throw;
  }
  RTDL_CUDA_CHECK(cudaEventRecord(ev_ready, aux));
  RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ev_ready, 0));
  pq->stream = s;  // from here the set is used and released on s
  if (timer) timer->mark("build");
  QueryResult r;
  try {
    r = run_radius_query(sc, q, in.nq, predicate, radius, limit, rows_dev, rows_capacity, rows_alloc, overflow_dev, s,
                         timer, nullptr, nullptr, pq, false, download);
  } catch (...) {
    pq->raw = nullptr;
    destroy_query_set(pq);
    throw;
  }
  pq->raw = nullptr;  // the caller's records (or *query_owned)
  destroy_query_set(pq);
  return r;
}

// Rows to host memory with the query set cut into `chunks` ranges of its input
// order, answered one after another against one scene: each range's rows are
// copied to their place in `host_rows` (the ranges' rows follow one another
// in input order, as one call's would) range by range on `copy` while the
// next range is collected and emitted on `s`.  The transfer of the rows,
// which bounds such a call, so starts after the first range's query instead
// of after the whole set's.  Each range is an ordinary query: its rows are
// the rows a call with only those queries gives.
QueryResult run_build_and_query_chunked(const BuildQueryInputs& in, int predicate, double radius, uint32_t limit,
                                        cudaStream_t s, cudaStream_t copy, PhaseTimer* timer, Scene** scene_out,
                                        void* host_rows, unsigned long long host_capacity_rows, int chunks) {
  *scene_out = nullptr;
  const size_t rec = in.dim == 3 ? sizeof(RtdlPoint3D) : sizeof(RtdlPoint);
  const size_t row_size = predicate == kFrn ? sizeof(RtdlFixedRadiusNeighborRow) : sizeof(RtdlKnnNeighborRow);
  // Each range's query set is uploaded and prepared (Morton order, its own
  // statistics) on a third stream one range ahead: the first range's beside
  // the scene build, every later one beside the query of the range before it.
  cudaStream_t ps = aux_stream(1);
  std::vector<PreparedQueries*> sets(chunks, nullptr);
  std::vector<cudaEvent_t> ready(chunks, nullptr);
  auto range_of = [&](int c, uint32_t& q0, uint32_t& n) {
    q0 = (uint32_t)((uint64_t)in.nq * (uint32_t)c / (uint32_t)chunks);
    n = (uint32_t)((uint64_t)in.nq * (uint32_t)(c + 1) / (uint32_t)chunks) - q0;
  };
  auto prepare_range = [&](int c) {
    uint32_t q0, n;
    range_of(c, q0, n);
    void* d_q = dev_alloc(rec * n, ps);
    RTDL_CUDA_CHECK(cudaMemcpyAsync(d_q, static_cast<const char*>(in.query_host) + rec * q0, rec * n,
                                    cudaMemcpyHostToDevice, ps));
    PreparedQueries* pq = nullptr;
    try {
      pq = prepare_query_set(d_q, n, in.dim, ps);  // owns d_q from here
    } catch (...) {
      dev_free(d_q, ps);
      throw;
    }
    sets[c] = pq;
    RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ready[c], cudaEventDisableTiming));
    RTDL_CUDA_CHECK(cudaEventRecord(ready[c], ps));
  };
  // Every range keeps its device rows until all copies are done: a buffer
  // released behind its copies would make the pool order the next range's
  // allocation, and so its emission, after them.
  std::vector<void*> range_rows;
  auto release = [&]() {
    sync_quietly(ps);
    for (int c = 0; c < chunks; ++c) {
      if (sets[c]) {
        sets[c]->stream = s;
        destroy_query_set(sets[c]);
        sets[c] = nullptr;
      }
      if (ready[c]) {
        note_cleanup_error(cudaEventDestroy(ready[c]), "cudaEventDestroy");
        ready[c] = nullptr;
      }
    }
    for (void* p : range_rows) dev_free(p, s);
    range_rows.clear();
  };
  QueryResult total;
  try {
    // the query side waits for what the caller queued on s (the search set's upload)
    static thread_local cudaEvent_t ev_start = nullptr;
    if (!ev_start) RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming));
    RTDL_CUDA_CHECK(cudaEventRecord(ev_start, s));
    RTDL_CUDA_CHECK(cudaStreamWaitEvent(ps, ev_start, 0));
    prepare_range(0);
    Scene* sc = build_scene(in.search_dev, in.ns, in.dim, s, scene_leaf_size());
    *scene_out = sc;
    if (timer) timer->mark("build");
    for (int c = 0; c < chunks; ++c) {
      uint32_t q0, nqc;
      range_of(c, q0, nqc);
      if (total.rows + (unsigned long long)nqc * limit > host_capacity_rows)
        throw std::runtime_error("host row buffer too small for the query ranges");
      RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ready[c], 0));
      PreparedQueries* pq = sets[c];
      pq->stream = s;  // from here the set is used and released on s
      if (c + 1 < chunks) prepare_range(c + 1);
      void* d_rows = nullptr;
      RowDownload dl;
      dl.host_fixed = static_cast<char*>(host_rows) + total.rows * row_size;
      dl.copy = copy;
      QueryResult r;
      try {
        r = run_radius_query(sc, nullptr, nqc, predicate, radius, limit, nullptr, 0, &d_rows, nullptr, s, nullptr,
                             nullptr, nullptr, pq, false, &dl);
        if (r.rows && dl.copies == 0)  // a range too small to be copied piecewise: one copy after its emit
          RTDL_CUDA_CHECK(cudaMemcpyAsync(dl.host_fixed, d_rows, r.rows * row_size, cudaMemcpyDeviceToHost, s));
      } catch (...) {
        if (d_rows) range_rows.push_back(d_rows);
        throw;
      }
      range_rows.push_back(d_rows);
      destroy_query_set(pq);
      sets[c] = nullptr;
      total.rows += r.rows;
      total.heavy += r.heavy;
    }
    if (timer) timer->mark("queries");
    // the rows are released on `s` once it has waited for the copies
    static thread_local cudaEvent_t ev_copied = nullptr;
    if (!ev_copied) RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_copied, cudaEventDisableTiming));
    RTDL_CUDA_CHECK(cudaEventRecord(ev_copied, copy));
    RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ev_copied, 0));
    release();
  } catch (...) {
    sync_quietly(copy);
    sync_quietly(s);
    release();
    throw;
  }
  return total;
}

// ---- captured summary graphs ------------------------------------------------
namespace {

constexpr unsigned int kGraphStatusOverflow = 1u;  // traversal stack overflow (the plain call raises it)
constexpr unsigned int kGraphStatusGeneric = 2u;   // heavy queries left for the generic path
constexpr unsigned int kBatchGraphStatusRows = 4u;  // a batch graph's rows exceed the caller's row buffer

__global__ void k_graph_status(const unsigned int* small, const unsigned int* pass_count, uint32_t requests,
                               unsigned int* status) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < requests; r += gridDim.x * blockDim.x)
    status[r] = ((small[8 * (size_t)r + 1] & 1u) ? kGraphStatusOverflow : 0u) |
                (pass_count[(size_t)r * kRefinePasses + kRefinePasses - 1] ? kGraphStatusGeneric : 0u);
}


}  // namespace

struct SummaryGraph {
  Scene* sc = nullptr;
  const PreparedQueries* pq = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t R = 0, nq = 0, kcap = 0;  // requests, queries, row capacity per query
  std::vector<double> radius;
  std::vector<uint32_t> kmax;
  std::vector<void*> buffers;  // device, released at destroy
  DevBands* bands = nullptr;   // one per request
  unsigned long long* slab = nullptr;
  uint32_t* counts = nullptr;
  QueryInfo* qinfo = nullptr;
  uint8_t* flags = nullptr;
  uint32_t *heavy_list = nullptr, *heavy_m = nullptr, *heavy_t = nullptr;
  uint32_t *mid_list = nullptr, *big_list = nullptr, *fix_list = nullptr;
  unsigned int* small = nullptr;       // 8 counters per request (CollectParams::small)
  unsigned int* pass_count = nullptr;  // kRefinePasses per request: work left after each pass
  unsigned long long *offsets = nullptr, *poff = nullptr;
  void* scan_ws = nullptr;
  void* rows = nullptr;  // nq * kcap rows
  uint32_t* work[2] = {nullptr, nullptr};
  double *rad[2] = {nullptr, nullptr}, *lo[2] = {nullptr, nullptr}, *hi[2] = {nullptr, nullptr};
  uint32_t* full[2] = {nullptr, nullptr};
  double* frad[2] = {nullptr, nullptr};
  double* gen_rad = nullptr;
  uint32_t *cnt = nullptr, *gen_qin = nullptr, *gen_m = nullptr;
  SummaryPartial* partial = nullptr;
  uint32_t summary_blocks = 0;
  RtdlFixedRadiusRankedNeighborAggregate* agg = nullptr;  // one per request
  unsigned int* status = nullptr;                         // one per request
  RtdlFixedRadiusRankedNeighborAggregate* agg_host = nullptr;  // pinned
  unsigned int* status_host = nullptr;                          // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernels = 0;  // kernel nodes per replay
  uint64_t fallbacks = 0;
};

namespace {

void graph_check_requests(const Scene* sc, const double* radii, const uint32_t* kmax, uint32_t requests) {
  if (requests == 0) throw std::runtime_error("fixed_radius_neighbors_3d graph request_count must be positive");
  if (!radii || !kmax) throw std::runtime_error("radii and k_values must not be null");
  for (uint32_t r = 0; r < requests; ++r) {
    if (!(radii[r] >= 0.0)) throw std::runtime_error("fixed_radius_neighbors_3d radius must be non-negative");
    if (radii[r] > sc->max_radius + 1.0e-7)
      throw std::runtime_error("fixed_radius_neighbors_3d radius exceeds prepared max_radius");
    if (kmax[r] == 0) throw std::runtime_error("fixed_radius_neighbors_3d k_max must be positive");
    if (kmax[r] > 64)
      throw std::runtime_error("prepared ranked fixed_radius_neighbors_3d aggregate currently supports k_max <= 64");
  }
}

// One request's kernels, device-driven (no host reads, no allocation).
void graph_enqueue_request(SummaryGraph* g, uint32_t r, cudaStream_t s) {
  Scene* sc = g->sc;
  const PreparedQueries* pq = g->pq;
  const uint32_t nq = g->nq, np = nq;
  const double radius = g->radius[r];
  const uint32_t kmax = g->kmax[r];
  unsigned int* small = g->small + 8 * (size_t)r;
  unsigned int* pc = g->pass_count + (size_t)r * kRefinePasses;
  k_bands<<<1, 32, 0, s>>>(sc->stats, pq->qst, radius, 1, g->bands + r);
  RTDL_LAUNCHED(1);
  CollectParams C;
  C.S = sc->view();
  C.qpts = pq->qpts;
  C.qraw = static_cast<const double*>(pq->raw);
  C.qstride = sc->dim == 3 ? 4 : 3;
  C.qorder = pq->qorder;
  C.nq = np;
  C.kmax = kmax;
  C.bands = g->bands + r;
  C.warp_prob = nullptr;
  C.prob_kmax = nullptr;
  C.slab = g->slab;
  C.counts = g->counts;
  C.qinfo = g->qinfo;
  C.flags = g->flags;
  C.heavy_list = g->heavy_list;
  C.heavy_m = g->heavy_m;
  C.heavy_t = g->heavy_t;
  C.mid_list = g->mid_list;
  C.big_list = g->big_list;
  C.small = small;
  C.overflow_out = nullptr;
  C.stats = nullptr;
  launch_collect(C, np, nq, false, false, s);
  scan_counts_u64_ws(g->counts, pq->oorder, pq->identity, nq, g->offsets, g->scan_ws, s);
  // heavy queries: every refinement pass is launched; each reads its work count
  RefineDevice D;
  for (int b2 = 0; b2 < 2; ++b2) {
    D.work[b2] = g->work[b2];
    D.rad[b2] = g->rad[b2];
    D.lo[b2] = g->lo[b2];
    D.hi[b2] = g->hi[b2];
    D.frad[b2] = g->frad[b2];
    D.full[b2] = g->full[b2];
  }
  D.cnt = g->cnt;
  D.gen_qin = g->gen_qin;
  D.gen_m = g->gen_m;
  D.gen_rad = g->gen_rad;
  D.pass_count = pc;
  enqueue_refine_device(C, nullptr, nullptr, radius, nullptr, kmax, np, true, g->qinfo, g->flags, small, D, s);
  k_proc_offsets<<<grid_for(np, 256), 256, 0, s>>>(pq->qorder, pq->qrank, g->offsets, np, g->poff);
  RTDL_LAUNCHED(1);
  EmitParams E;
  E.S = sc->view();
  E.nq = np;
  E.slab = g->slab;
  E.qinfo = g->qinfo;
  E.poff = g->poff;
  E.sink.rows = g->rows;
  E.sink.capacity = (unsigned long long)nq * g->kcap;
  E.sink.ranked = 0;
  E.fix_list = g->fix_list;
  E.fix_count = small + 4;
  k_emit<<<emit_grid(np), kEmitThreads, 0, s>>>(E);
  k_emit_list<4, true><<<kStrideBlocks, kEmitListThreads, 0, s>>>(E, g->mid_list, 0, small + 2);
  k_emit_list<8, false><<<kStrideBlocks, kEmitListThreads, 0, s>>>(E, g->big_list, 0, small + 3);
  k_emit_fixup<<<kSmCount * 4, kFixupThreads, 0, s>>>(E);
  k_summarize<<<g->summary_blocks, kSummaryThreads, 0, s>>>(static_cast<const RtdlFixedRadiusNeighborRow*>(g->rows),
                                                            g->offsets, pq->oorder, pq->identity, pq->qpts, nq,
                                                            nullptr, g->partial);
  k_summary_final<<<1, 1024, 0, s>>>(g->partial, g->summary_blocks, nq, g->agg + r);
  RTDL_LAUNCHED(6);
}

void graph_release(SummaryGraph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  g->exec = nullptr;
  g->graph = nullptr;
}

void graph_capture(SummaryGraph* g) {
  graph_release(g);
  cudaStream_t s = g->stream;
  const unsigned long long before = launches_counted();
  RTDL_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->small, 0, sizeof(unsigned int) * 8 * (size_t)g->R, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->pass_count, 0, sizeof(unsigned int) * kRefinePasses * (size_t)g->R, s));
    for (uint32_t r = 0; r < g->R; ++r) graph_enqueue_request(g, r, s);
    k_graph_status<<<div_up(g->R, 256), 256, 0, s>>>(g->small, g->pass_count, g->R, g->status);
    RTDL_LAUNCHED(1);
  } catch (...) {
    cudaGraph_t partial = nullptr;
    cudaStreamEndCapture(s, &partial);
    if (partial) cudaGraphDestroy(partial);
    cudaGetLastError();
    count_launches(-(int)(launches_counted() - before));
    throw;
  }
  // captured kernels are counted when a replay launches them
  count_launches(-(int)(launches_counted() - before));
  RTDL_CUDA_CHECK(cudaStreamEndCapture(s, &g->graph));
  RTDL_CUDA_CHECK(cudaGraphInstantiate(&g->exec, g->graph, 0));
  size_t n = 0;
  RTDL_CUDA_CHECK(cudaGraphGetNodes(g->graph, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  RTDL_CUDA_CHECK(cudaGraphGetNodes(g->graph, nodes.data(), &n));
  g->kernels = 0;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    RTDL_CUDA_CHECK(cudaGraphNodeGetType(nodes[i], &t));
    if (t == cudaGraphNodeTypeKernel) ++g->kernels;
  }
}

void graph_set_requests(SummaryGraph* g, const double* radii, const uint32_t* kmax, uint32_t requests) {
  g->radius.assign(radii, radii + requests);
  g->kmax.assign(kmax, kmax + requests);
}

// Row buffer for the largest k_max of the requests (grown by an update, never shrunk).
void graph_size_rows(SummaryGraph* g) {
  uint32_t k = 1;
  for (uint32_t v : g->kmax) k = v > k ? v : k;
  if (g->rows && k <= g->kcap) return;
  dev_free(g->rows, g->stream);
  g->rows = nullptr;
  g->kcap = 0;
  g->rows = dev_alloc(sizeof(RtdlFixedRadiusNeighborRow) * (size_t)g->nq * k, g->stream);
  g->kcap = k;
}

}  // namespace

SummaryGraph* summary_graph_create(Scene* sc, const PreparedQueries* pq, const double* radii, const uint32_t* kmax,
                                   uint32_t requests) {
  if (!sc) throw std::runtime_error("prepared OptiX fixed-radius-neighbor 3D handle must not be null");
  if (!pq) throw std::runtime_error("prepared fixed-radius query handle must not be null");
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  if (pq->dim != sc->dim) throw std::runtime_error("prepared queries and scene differ in dimension");
  graph_check_requests(sc, radii, kmax, requests);
  if (pq->n == 0 || sc->n == 0)
    throw std::runtime_error("fixed_radius_neighbors_3d graph requires non-empty prepared search and query handles");
  SummaryGraph* g = new SummaryGraph();
  g->sc = sc;
  g->pq = pq;
  g->R = requests;
  g->nq = pq->n;
  graph_set_requests(g, radii, kmax, requests);
  try {
    RTDL_CUDA_CHECK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    cudaStream_t s = g->stream;
    // the scene and the prepared queries were built on their own streams
    RTDL_CUDA_CHECK(cudaStreamSynchronize(sc->stream));
    RTDL_CUDA_CHECK(cudaStreamSynchronize(pq->stream));
    unsigned int bad[2] = {0, 0};
    RTDL_CUDA_CHECK(cudaMemcpy(&bad[0], &sc->stats->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    RTDL_CUDA_CHECK(cudaMemcpy(&bad[1], &pq->qst->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    throw_if_bad(bad[0] | bad[1]);
    auto alloc = [&](size_t bytes) {
      void* p = dev_alloc(bytes ? bytes : 1, s);
      g->buffers.push_back(p);
      return p;
    };
    const size_t n = g->nq, R = g->R;
    g->bands = static_cast<DevBands*>(alloc(sizeof(DevBands) * R));
    g->slab = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * slab_base(g->nq)));
    g->counts = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->qinfo = static_cast<QueryInfo*>(alloc(sizeof(QueryInfo) * n));
    g->flags = static_cast<uint8_t*>(alloc(n));
    g->heavy_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->heavy_m = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->heavy_t = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->mid_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->big_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->fix_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->small = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * 8 * R));
    g->pass_count = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * kRefinePasses * R));
    g->offsets = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * (n + 1)));
    g->poff = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * n));
    g->scan_ws = alloc(scan_workspace_bytes(g->nq));
    graph_size_rows(g);
    for (int b = 0; b < 2; ++b) {
      g->work[b] = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
      g->rad[b] = static_cast<double*>(alloc(sizeof(double) * n));
      g->lo[b] = static_cast<double*>(alloc(sizeof(double) * n));
      g->hi[b] = static_cast<double*>(alloc(sizeof(double) * n));
      g->full[b] = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
      g->frad[b] = static_cast<double*>(alloc(sizeof(double) * n));
    }
    g->cnt = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->gen_qin = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->gen_m = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->gen_rad = static_cast<double*>(alloc(sizeof(double) * n));
    g->summary_blocks = div_up((uint64_t)n * 32, kSummaryThreads);
    g->partial = static_cast<SummaryPartial*>(alloc(sizeof(SummaryPartial) * g->summary_blocks));
    g->agg = static_cast<RtdlFixedRadiusRankedNeighborAggregate*>(
        alloc(sizeof(RtdlFixedRadiusRankedNeighborAggregate) * R));
    g->status = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * R));
    RTDL_CUDA_CHECK(cudaMallocHost(&g->agg_host, sizeof(RtdlFixedRadiusRankedNeighborAggregate) * R));
    RTDL_CUDA_CHECK(cudaMallocHost(&g->status_host, sizeof(unsigned int) * R));
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // allocations ready before capture
    graph_capture(g);
  } catch (...) {
    summary_graph_destroy(g);
    throw;
  }
  return g;
}

void summary_graph_update(SummaryGraph* g, const double* radii, const uint32_t* kmax, uint32_t requests) {
  if (!g) throw std::runtime_error("prepared fixed_radius_neighbors_3d graph handle must not be null");
  if (requests != g->R)
    throw std::runtime_error("fixed_radius_neighbors_3d graph request update requires unchanged request_count");
  graph_check_requests(g->sc, radii, kmax, requests);
  RTDL_CUDA_CHECK(cudaStreamSynchronize(g->stream));  // no replay in flight while the graph is replaced
  graph_set_requests(g, radii, kmax, requests);
  graph_size_rows(g);
  RTDL_CUDA_CHECK(cudaStreamSynchronize(g->stream));
  graph_capture(g);
}

void summary_graph_launch(SummaryGraph* g) {
  if (!g || !g->exec) throw std::runtime_error("prepared fixed_radius_neighbors_3d graph handle must not be null");
  RTDL_CUDA_CHECK(cudaGraphLaunch(g->exec, g->stream));
  count_launches(g->kernels);
}

void summary_graph_replay(SummaryGraph* g, RtdlFixedRadiusRankedNeighborAggregate* out) {
  if (!out) throw std::runtime_error("aggregates_out must not be null");
  summary_graph_launch(g);
  cudaStream_t s = g->stream;
  RTDL_CUDA_CHECK(cudaMemcpyAsync(g->agg_host, g->agg, sizeof(RtdlFixedRadiusRankedNeighborAggregate) * g->R,
                                  cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(g->status_host, g->status, sizeof(unsigned int) * g->R, cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  for (uint32_t r = 0; r < g->R; ++r) {
    if (g->status_host[r] & kGraphStatusOverflow) throw std::runtime_error("BVH traversal stack overflow");
    if (g->status_host[r] & kGraphStatusGeneric) {
      // the plain call, with its generic path for the queries refinement left
      run_ranked_summaries(g->sc, nullptr, g->nq, g->radius[r], g->kmax[r], nullptr, &out[r], s, nullptr, g->pq);
      ++g->fallbacks;
    } else {
      out[r] = g->agg_host[r];
    }
  }
}

const RtdlFixedRadiusRankedNeighborAggregate* summary_graph_device_aggregates(const SummaryGraph* g) { return g->agg; }
const unsigned int* summary_graph_device_status(const SummaryGraph* g) { return g->status; }
cudaStream_t summary_graph_stream(const SummaryGraph* g) { return g->stream; }
uint32_t summary_graph_requests(const SummaryGraph* g) { return g->R; }
uint64_t summary_graph_fallbacks(const SummaryGraph* g) { return g->fallbacks; }

void summary_graph_destroy(SummaryGraph* g) {
  if (!g) return;
  if (g->stream) cudaStreamSynchronize(g->stream);
  graph_release(g);
  for (void* p : g->buffers) dev_free(p, g->stream);
  dev_free(g->rows, g->stream);
  if (g->stream) {
    sync_quietly(g->stream);
    note_cleanup_error(cudaStreamDestroy(g->stream), "cudaStreamDestroy");
  }
  if (g->agg_host) cudaFreeHost(g->agg_host);
  if (g->status_host) cudaFreeHost(g->status_host);
  delete g;
}

namespace {
__global__ void k_identity_flag(const PointStats* qst, unsigned int* identity) {
  if (threadIdx.x == 0) *identity = qst->ids_unsorted ? 0u : 1u;
}
}  // namespace

PreparedQueries* prepare_query_set(const void* records_dev, uint32_t n, int dim, cudaStream_t s) {
  PreparedQueries* pq = new PreparedQueries();
  pq->dim = dim;
  pq->n = n;
  pq->stream = s;
  RTDL_CUDA_CHECK(cudaGetDevice(&pq->device));
  const size_t n1 = n ? n : 1;
  try {
    pq->raw = const_cast<void*>(records_dev);
    pq->qst = static_cast<PointStats*>(dev_alloc(sizeof(PointStats), s));
    pq->qpts = static_cast<float4*>(dev_alloc(sizeof(float4) * n1, s));
    pq->qorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n1, s));
    pq->oorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n1, s));
    pq->qrank = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n1, s));
    pq->identity = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int), s));
    reset_stats(pq->qst, s);
    prep_points(records_dev, n, dim, pq->qpts, pq->qst, s);
    k_identity_flag<<<1, 32, 0, s>>>(pq->qst, pq->identity);
    RTDL_LAUNCHED(1);
    uint32_t* codes = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n1, s));
    morton_codes(pq->qpts, n, dim, pq->qst, codes, s);  // the set's own box: the order only groups neighbours
    iota_u32(pq->qorder, n, s);
    radix_sort_pairs(codes, pq->qorder, n, 0, dim == 3 ? 30 : 32, nullptr, &pq->qst->bad, s);
    k_extract_ids<<<grid_for(n, 256), 256, 0, s>>>(pq->qpts, n, codes);
    RTDL_LAUNCHED(1);
    iota_u32(pq->oorder, n, s);
    radix_sort_pairs(codes, pq->oorder, n, 0, 32, pq->identity, &pq->qst->bad, s);
    k_invert<<<grid_for(n, 256), 256, 0, s>>>(pq->oorder, n, pq->identity, pq->qrank);
    RTDL_LAUNCHED(1);
    dev_free(codes, s);
  } catch (...) {
    pq->raw = nullptr;
    destroy_query_set(pq);
    throw;
  }
  return pq;
}

void destroy_query_set(PreparedQueries* pq) {
  if (!pq) return;
  cudaStream_t s = pq->stream;
  dev_free(pq->raw, s);
  dev_free(pq->qst, s);
  dev_free(pq->qpts, s);
  dev_free(pq->qorder, s);
  dev_free(pq->oorder, s);
  dev_free(pq->qrank, s);
  dev_free(pq->identity, s);
  delete pq;
}

QueryResult run_query_batch(Scene* sc, const void* queries_dev, const BatchSpec& bs, void* rows_dev,
                            size_t rows_capacity, void** rows_alloc, uint8_t* overflow_dev, cudaStream_t s,
                            PhaseTimer* timer) {
  if (rows_alloc) *rows_alloc = nullptr;
  if (sc->problems != 0 && sc->problems != bs.problems)
    throw std::runtime_error("query batch and scene batch differ in problem count");
  if (bs.qoff[0] != 0) throw std::runtime_error("query offsets must start at 0");
  for (uint32_t p = 0; p < bs.problems; ++p) {
    if (bs.qoff[p + 1] < bs.qoff[p]) throw std::runtime_error("query offsets must be non-decreasing");
    if (!(bs.radius[p] >= 0.0)) throw std::runtime_error("radius must be non-negative");
    if (bs.kmax[p] < 1 || bs.kmax[p] > 64) throw std::runtime_error("a problem batch takes k_max in [1, 64]");
  }
  const unsigned long long nq = bs.qoff[bs.problems];
  if (nq > 0xFFFFFFFFull) throw std::runtime_error("query_count exceeds uint32 limit");
  if (nq == 0 || sc->n == 0) {
    for (uint32_t p = 0; p <= bs.problems; ++p) bs.row_offsets[p] = 0;
    return QueryResult{};
  }
  return run_radius_query(sc, queries_dev, (uint32_t)nq, kFrn, 0.0, 0, rows_dev, rows_capacity, rows_alloc,
                          overflow_dev, s, timer, &bs);
}

// The list kernels take their per-lane lists in dynamic shared memory
// (block_threads x list length x 8 B, at most kMaxList x 256 x 8 = 128 KiB).
// The limit a launch may ask for is a per-function attribute of each device:
// it is raised once per device to that largest size, never per launch, so
// concurrent calls with different k cannot lower it under one another.
void ensure_pass1_shared_memory() {
  static std::mutex m;
  static std::vector<bool> done;
  int dev = 0;
  RTDL_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(m);
  if ((int)done.size() <= dev) done.resize(dev + 1, false);
  if (done[dev]) return;
  const int most = kMaxList * 256 * 8;
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true, true, kWalkRope>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true, false, kWalkRope>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true, true, kWalkNear>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true, false, kWalkNear>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
  done[dev] = true;
}

QueryResult run_query(Scene* sc, const void* queries_dev, uint32_t nq, int predicate, double radius, uint32_t limit,
                      void* rows_dev, size_t rows_capacity, void** rows_alloc, uint8_t* overflow_dev, cudaStream_t s,
                      PhaseTimer* timer) {
  QueryResult res;
  if (rows_alloc) *rows_alloc = nullptr;
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  const bool knn = predicate == kKnn;
  const int qstride = sc->dim == 3 ? 4 : 3;
  if (nq == 0) return res;
  if (sc->n == 0) {
    if (overflow_dev) RTDL_CUDA_CHECK(cudaMemsetAsync(overflow_dev, 0, nq, s));
    return res;
  }
  if (timer) timer->mark("start");
  if (!knn && limit <= (uint32_t)kMaxList)
    return run_radius_query(sc, queries_dev, nq, predicate, radius, limit, rows_dev, rows_capacity, rows_alloc,
                            overflow_dev, s, timer);
  QueryPrep qp = prepare_queries(sc, queries_dev, nq, !knn, radius, true, s);
  const bool all_heavy = knn && limit > (uint32_t)kMaxList;
  const int L = all_heavy ? 1 : (int)(limit < (uint32_t)kMaxList ? limit : (uint32_t)kMaxList);
  if (timer) timer->mark("query_prep");

  uint32_t* counts = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  uint8_t* flags = static_cast<uint8_t*>(dev_alloc(nq, s));
  uint32_t* temp = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (size_t)nq * L, s));
  uint32_t* heavy_list = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  uint32_t* heavy_m = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  unsigned int* small = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int) * 4, s));  // heavy count, error
  unsigned long long* offsets = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (nq + 1), s));
  RTDL_CUDA_CHECK(cudaMemsetAsync(small, 0, sizeof(unsigned int) * 4, s));
  GenericOut g;
  auto cleanup = [&]() {
    g.release(s);
    dev_free(counts, s);
    dev_free(flags, s);
    dev_free(temp, s);
    dev_free(heavy_list, s);
    dev_free(heavy_m, s);
    dev_free(small, s);
    dev_free(offsets, s);
    free_prep(qp, s);
  };
  try {
    if (all_heavy) {
      k_mark_all_heavy<<<grid_for(nq, 256), 256, 0, s>>>(qp.qorder, nq, sc->n, limit, counts, flags, temp,
                                                         heavy_list, heavy_m);
      RTDL_LAUNCHED(1);
      RTDL_CUDA_CHECK(cudaMemcpyAsync(small, &nq, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // nq lives on this host stack frame
    } else {
      Pass1Params P;
      P.S = sc->view();
      P.qpts = qp.qpts;
      P.qraw = static_cast<const double*>(queries_dev);
      P.qstride = qstride;
      P.qorder = qp.qorder;
      P.nq = nq;
      P.kmax = limit;
      P.L = L;
      P.bands = qp.bands;
      P.temp = temp;
      P.counts = counts;
      P.flags = flags;
      P.heavy_list = heavy_list;
      P.heavy_m = heavy_m;
      P.heavy_count = small;
      P.error = small + 1;
      const int threads = tuning().block_threads;
      const size_t shm = (size_t)threads * L * 8;
      const unsigned int blocks = div_up(nq, threads);
      const bool stats = stats_enabled();
      P.stats = nullptr;
      P.qcodes = qp.qcodes;
      P.scodes = sc->codes;
      if (stats) {
        P.stats = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * kStatCount, s));
        RTDL_CUDA_CHECK(cudaMemsetAsync(P.stats, 0, sizeof(unsigned long long) * kStatCount, s));
      }
      ensure_pass1_shared_memory();
      auto launch = [&](auto kernel) { kernel<<<blocks, threads, shm, s>>>(P); };
      const int walk = tuning().traversal == 1 ? kWalkLane : L >= kNearFirstMinList ? kWalkNear : kWalkRope;
      if (knn) {
        if (walk == kWalkNear) stats ? launch(k_pass1<true, true, kWalkNear>) : launch(k_pass1<true, false, kWalkNear>);
        else if (walk == kWalkRope) stats ? launch(k_pass1<true, true, kWalkRope>) : launch(k_pass1<true, false, kWalkRope>);
        else stats ? launch(k_pass1<true, true>) : launch(k_pass1<true, false>);
      } else {
        if (stats) launch(k_pass1<false, true>);
        else launch(k_pass1<false, false>);
      }
      RTDL_LAUNCHED(1);
      if (stats) {
        RTDL_CUDA_CHECK(cudaMemcpyAsync(last_stats().data(), P.stats, sizeof(unsigned long long) * kStatCount,
                                        cudaMemcpyDeviceToHost, s));
        dev_free(P.stats, s);
      }
    }
    if (timer) timer->mark("traverse");
    scan_counts_u64(counts, qp.oorder, &qp.bands->ids_sorted, nq, offsets, s);
    if (timer) timer->mark("scan");

    Readback* rb = pinned_readback();
    SmallReads reads(rb);
    reads.add(&rb->rows, offsets + nq, sizeof(unsigned long long));
    reads.add(&rb->heavy, small, sizeof(unsigned int) * 2);
    reads.add(&rb->scene_bad, &sc->stats->bad, sizeof(unsigned int));
    reads.add(&rb->query_bad, &qp.qst->bad, sizeof(unsigned int));
    reads.launch(s);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    const Readback r = *rb;
    check_readback(r);
    res.rows = r.rows;
    res.heavy = r.heavy;
    if (r.heavy > 0) {
      g = run_generic_path(sc, qp, queries_dev, qstride, r.heavy, heavy_list, heavy_m, limit, knn, small + 1, s);
      if (timer) timer->mark("generic_path");
    }
    if (rows_alloc != nullptr) {
      const size_t row_size = predicate == kFrn ? 16 : 24;
      rows_dev = res.rows ? dev_alloc(row_size * res.rows, s) : nullptr;
      rows_capacity = res.rows;
      *rows_alloc = rows_dev;
    }
    if (res.rows > 0 || overflow_dev != nullptr) {
      ExpandParams E;
      E.S = sc->view();
      E.qpts = qp.qpts;
      E.qraw = static_cast<const double*>(queries_dev);
      E.qstride = qstride;
      E.oorder = qp.oorder;
      E.bands = qp.bands;
      E.nq = nq;
      E.L = L;
      E.counts = counts;
      E.flags = flags;
      E.temp = temp;
      E.heavy_out = g.heavy_out;
      E.heavy_out_off = g.heavy_out_off;
      E.offsets = offsets;
      E.rows = rows_dev;
      E.capacity = rows_dev ? rows_capacity : 0;
      E.ranked = predicate == kFrn ? 0 : 1;
      E.overflow_out = overflow_dev;
      E.error = small + 1;
      E.work_list = nullptr;
      E.qrank = nullptr;
      // lists of at most L rows unless some query took the generic path
      const int group = (r.heavy > 0 || L > 16) ? 32 : L > 8 ? 16 : L > 4 ? 8 : L > 2 ? 4 : L > 1 ? 2 : 1;
      const unsigned int blocks = grid_for((uint64_t)nq * group, kExpandThreads);
      switch (group) {
        case 1: k_expand<1><<<blocks, kExpandThreads, 0, s>>>(E); break;
        case 2: k_expand<2><<<blocks, kExpandThreads, 0, s>>>(E); break;
        case 4: k_expand<4><<<blocks, kExpandThreads, 0, s>>>(E); break;
        case 8: k_expand<8><<<blocks, kExpandThreads, 0, s>>>(E); break;
        case 16: k_expand<16><<<blocks, kExpandThreads, 0, s>>>(E); break;
        default: k_expand<32><<<blocks, kExpandThreads, 0, s>>>(E); break;
      }
      RTDL_LAUNCHED(1);
    }
    if (timer) timer->mark("emit");
    RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->error, small + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    if (rb->error & 8u) throw std::runtime_error("LBVH traversal stack overflow");
    if (rb->error & 6u) throw std::runtime_error("generic neighbor path produced an inconsistent candidate count");
  } catch (...) {
    sync_quietly(s);
    cleanup();
    throw;
  }
  cleanup();
  return res;
}

HausdorffResult run_directed_hausdorff(Scene* sc, const void* queries_dev, uint32_t nq, double* nearest_dist_dev,
                                       uint32_t* nearest_id_dev, cudaStream_t s, PhaseTimer* timer) {
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  if (nq == 0 || sc->n == 0) throw std::runtime_error("Hausdorff distance requires non-empty point sets");
  const int qstride = sc->dim == 3 ? 4 : 3;
  if (timer) timer->mark("start");
  QueryPrep qp = prepare_queries(sc, queries_dev, nq, false, 0.0, false, s);
  if (timer) timer->mark("query_prep");
  uint32_t* counts = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  uint8_t* flags = static_cast<uint8_t*>(dev_alloc(nq, s));
  uint32_t* temp = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  unsigned int* small = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int) * 4, s));
  RTDL_CUDA_CHECK(cudaMemsetAsync(small, 0, sizeof(unsigned int) * 4, s));
  Pass1Params P;
  P.S = sc->view();
  P.qpts = qp.qpts;
  P.qraw = static_cast<const double*>(queries_dev);
  P.qstride = qstride;
  P.qorder = qp.qorder;
  P.nq = nq;
  P.kmax = 1;
  P.L = 1;
  P.bands = qp.bands;
  P.temp = temp;
  P.counts = counts;
  P.flags = flags;
  P.heavy_list = nullptr;
  P.heavy_m = nullptr;
  P.heavy_count = small;
  P.error = small + 1;
  const int threads = tuning().block_threads;
  P.stats = nullptr;
  P.qcodes = qp.qcodes;
  P.scodes = sc->codes;
  if (tuning().traversal != 1)
    k_pass1<true, false, kWalkRope><<<div_up(nq, threads), threads, (size_t)threads * 8, s>>>(P);
  else
    k_pass1<true, false><<<div_up(nq, threads), threads, (size_t)threads * 8, s>>>(P);
  RTDL_LAUNCHED(1);
  if (timer) timer->mark("traverse");
  const unsigned int blocks = grid_for(nq, 256) < 2 * kSmCount ? grid_for(nq, 256) : 2 * kSmCount;
  Witness* partial = static_cast<Witness*>(dev_alloc(sizeof(Witness) * blocks, s));
  Witness* best = static_cast<Witness*>(dev_alloc(sizeof(Witness), s));
  k_nearest_reduce<<<blocks, 256, 0, s>>>(sc->view(), qp.qpts, static_cast<const double*>(queries_dev), qstride, nq,
                                          temp, nearest_dist_dev, nearest_id_dev, partial);
  k_witness_final<<<1, 32, 0, s>>>(partial, (int)blocks, best);
  RTDL_LAUNCHED(2);
  // one read of the witness (into the record's row-range words) and the error words
  Readback* rb = pinned_readback();
  static_assert(sizeof(Witness) <= sizeof(rb->chunk_rows), "readback record too small for the witness");
  SmallReads reads(rb);
  reads.add(rb->chunk_rows, best, sizeof(Witness));
  reads.add(&rb->scene_bad, &sc->stats->bad, sizeof(unsigned int));
  reads.add(&rb->query_bad, &qp.qst->bad, sizeof(unsigned int));
  reads.add(&rb->error, small + 1, sizeof(unsigned int));
  reads.launch(s);
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  Witness w;
  memcpy(&w, rb->chunk_rows, sizeof(Witness));
  const unsigned int bad[3] = {rb->scene_bad, rb->query_bad, rb->error};
  if (timer) timer->mark("reduce");
  dev_free(counts, s);
  dev_free(flags, s);
  dev_free(temp, s);
  dev_free(small, s);
  dev_free(partial, s);
  dev_free(best, s);
  free_prep(qp, s);
  throw_if_bad(bad[0] | bad[1]);
  if (bad[2] & 8u) throw std::runtime_error("LBVH traversal stack overflow");
  HausdorffResult out;
  unsigned long long db = w.dist;
  memcpy(&out.distance, &db, sizeof(double));
  out.source_id = w.qid;
  out.target_id = w.nid;
  return out;
}


// ---- allocation-free directed Hausdorff ------------------------------------
// Some callers cannot allocate device memory while they run this query: an
// application that hands the whole device heap to its own allocator, code
// running between the capture points of a larger CUDA graph it does not own,
// or a real-time loop where an allocation could stall.  For them
// rtdl_b200_scene_directed_hausdorff_noalloc takes every scratch buffer of
// the nearest pass and of the max-witness reduction from this file-scope
// device array instead of the stream-ordered allocator.  Every GPU that loads
// the library holds the array until the process exits.
namespace {

constexpr uint32_t kNoAllocMaxQueries = 1u << 18;  // 262,144 queries per call
constexpr unsigned int kNoAllocReduceBlocks = 2 * kSmCount;

constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

struct NoAllocLayout {  // byte offsets into the scratch array, 256-B aligned
  static constexpr size_t kStats = 0;
  static constexpr size_t kBands = align256(kStats + sizeof(PointStats));
  static constexpr size_t kSmall = align256(kBands + sizeof(DevBands));
  static constexpr size_t kBest = align256(kSmall + 4 * sizeof(unsigned int));
  static constexpr size_t kPartial = align256(kBest + sizeof(Witness));
  static constexpr size_t kQpts = align256(kPartial + kNoAllocReduceBlocks * sizeof(Witness));
  static constexpr size_t kOrder = align256(kQpts + (size_t)kNoAllocMaxQueries * sizeof(float4));
  static constexpr size_t kTemp = align256(kOrder + (size_t)kNoAllocMaxQueries * sizeof(uint32_t));
  static constexpr size_t kCounts = align256(kTemp + (size_t)kNoAllocMaxQueries * sizeof(uint32_t));
  static constexpr size_t kFlags = align256(kCounts + (size_t)kNoAllocMaxQueries * sizeof(uint32_t));
  static constexpr size_t kCodes = align256(kFlags + (size_t)kNoAllocMaxQueries);
  static constexpr size_t kTotal = align256(kCodes + (size_t)kNoAllocMaxQueries * sizeof(uint32_t));
};

// 9.75 MiB: scratch for up to kNoAllocMaxQueries queries.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NoAllocLayout::kTotal];

// Converts the reduced witness into the public record and folds in the
// input checks, so the call never needs a host round trip.
__global__ void k_noalloc_finish(const Witness* best, const PointStats* scene_stats, const PointStats* query_stats,
                                 RtdlB200Witness* out) {
  if (threadIdx.x != 0) return;
  RtdlB200Witness w;
  unsigned long long db = best->dist;
  w.distance = __longlong_as_double((long long)db);
  w.source_id = best->qid;
  w.target_id = best->nid;
  const unsigned int bad = scene_stats->bad | query_stats->bad;
  w.status = (bad & kBadSortWait) ? 3u : bad ? 1u : 0u;
  w.reserved = 0u;
  *out = w;
}

unsigned char* noalloc_scratch_for_current_device() {
  static std::mutex m;
  static std::vector<unsigned char*> ptrs;
  int dev = 0;
  RTDL_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(m);
  if ((int)ptrs.size() <= dev) ptrs.resize(dev + 1, nullptr);
  if (ptrs[dev] == nullptr) {
    // The symbol name is a host-side stand-in; the device address comes from
    // the runtime, per device, with that device current.
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                               cudaGetErrorString(e));
    ptrs[dev] = static_cast<unsigned char*>(p);
  }
  return ptrs[dev];
}

}  // namespace

void run_directed_hausdorff_noalloc(Scene* sc, const void* queries_dev, uint32_t nq, double* nearest_dist_dev,
                                    uint32_t* nearest_id_dev, RtdlB200Witness* witness_dev, cudaStream_t s) {
  if (sc->problems) throw std::runtime_error("a problem batch is queried with the batch entry points");
  if (nq == 0 || sc->n == 0) throw std::runtime_error("Hausdorff distance requires non-empty point sets");
  if (nq > kNoAllocMaxQueries)
    throw std::runtime_error("rtdl_b200_scene_directed_hausdorff_noalloc: query_count exceeds the limit of 262144 "
                             "queries set by its fixed scratch array");
  unsigned char* base = noalloc_scratch_for_current_device();
  PointStats* qst = reinterpret_cast<PointStats*>(base + NoAllocLayout::kStats);
  DevBands* bands = reinterpret_cast<DevBands*>(base + NoAllocLayout::kBands);
  unsigned int* small = reinterpret_cast<unsigned int*>(base + NoAllocLayout::kSmall);
  Witness* best = reinterpret_cast<Witness*>(base + NoAllocLayout::kBest);
  Witness* partial = reinterpret_cast<Witness*>(base + NoAllocLayout::kPartial);
  float4* qpts = reinterpret_cast<float4*>(base + NoAllocLayout::kQpts);
  uint32_t* qorder = reinterpret_cast<uint32_t*>(base + NoAllocLayout::kOrder);
  uint32_t* temp = reinterpret_cast<uint32_t*>(base + NoAllocLayout::kTemp);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + NoAllocLayout::kCounts);
  uint8_t* flags = reinterpret_cast<uint8_t*>(base + NoAllocLayout::kFlags);
  uint32_t* codes = reinterpret_cast<uint32_t*>(base + NoAllocLayout::kCodes);
  // The array keeps the previous call's contents: reset what must start at zero.
  reset_stats(qst, s);
  RTDL_CUDA_CHECK(cudaMemsetAsync(small, 0, 4 * sizeof(unsigned int), s));
  prep_points(queries_dev, nq, sc->dim, qpts, qst, s);
  k_bands<<<1, 32, 0, s>>>(sc->stats, qst, 0.0, 0, bands);
  RTDL_LAUNCHED(1);
  iota_u32(qorder, nq, s);  // input order: no sort, hence no sort scratch
  morton_codes(qpts, nq, sc->dim, sc->stats, codes, s);  // seeds the nearest search (input order)
  Pass1Params P;
  P.S = sc->view();
  P.qpts = qpts;
  P.qraw = static_cast<const double*>(queries_dev);
  P.qstride = sc->dim == 3 ? 4 : 3;
  P.qorder = qorder;
  P.nq = nq;
  P.kmax = 1;
  P.L = 1;
  P.bands = bands;
  P.temp = temp;
  P.counts = counts;
  P.flags = flags;
  P.heavy_list = nullptr;
  P.heavy_m = nullptr;
  P.heavy_count = small;
  P.error = small + 1;
  P.stats = nullptr;
  P.qcodes = codes;
  P.scodes = sc->codes;
  const int threads = tuning().block_threads;
  k_pass1<true, false><<<div_up(nq, threads), threads, (size_t)threads * 8, s>>>(P);
  RTDL_LAUNCHED(1);
  const unsigned int blocks = grid_for(nq, 256) < kNoAllocReduceBlocks ? grid_for(nq, 256) : kNoAllocReduceBlocks;
  k_nearest_reduce<<<blocks, 256, 0, s>>>(sc->view(), qpts, static_cast<const double*>(queries_dev), P.qstride, nq,
                                          temp, nearest_dist_dev, nearest_id_dev, partial);
  k_witness_final<<<1, 32, 0, s>>>(partial, (int)blocks, best);
  k_noalloc_finish<<<1, 32, 0, s>>>(best, sc->stats, qst, witness_dev);
  RTDL_LAUNCHED(3);
}


// ---- captured graphs over prepared problem batches --------------------------
// Many uneven fixed-radius problems, already built into problem batches
// (build_scene_batch: one LBVH per batch, each problem one subtree), answered
// by one CUDA graph replay with no host read-back inside.  Per batch the graph
// holds ONE persistent collect launch -- a grid that fills the GPU once, whose
// warps take 32-query packets (one problem each) from a device work queue
// until the batch's packets are gone, so small and large problems share the
// SMs -- then the scan (rows of this batch start where the previous batch's
// end), the device-driven radius refinement, and the emit kernels striding
// over device list lengths.  Batches run one after another in the graph and
// share one set of scratch buffers sized for the largest.  A batch whose heavy
// queries the refinement passes do not resolve is flagged in its status word
// and recomputed by the plain batch call at replay, so rows always equal it.
namespace {

__global__ void k_add_row_base(unsigned long long* offsets, uint32_t n, const unsigned long long* base,
                               unsigned long long* next_base) {
  const unsigned long long b = *base;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
    const unsigned long long v = offsets[i] + b;
    offsets[i] = v;
    if (i == n) *next_base = v;
  }
}

__global__ void k_empty_batch_rows(const unsigned long long* base, uint32_t problems, unsigned long long* prob_rows,
                                   unsigned long long* next_base) {
  const unsigned long long b = *base;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p <= problems; p += gridDim.x * blockDim.x) prob_rows[p] = b;
  if (blockIdx.x == 0 && threadIdx.x == 0) *next_base = b;
}

// Persistent collect over one batch: 32-query packets from a work queue.
template <int MIN_BLOCKS, int LEAF>
__global__ void __launch_bounds__(256, MIN_BLOCKS) k_collect_persistent(CollectParams P, unsigned int* queue) {
  const uint32_t packets = (P.nq + 31u) / 32u;
  const uint32_t lane = threadIdx.x & 31u;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(queue, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= packets) return;
    collect_packet_body<false, false, true, LEAF>(P, item * 32u + lane);
  }
}

constexpr int kPersistentMinBlocks = 5;

__global__ void k_batch_graph_status(const unsigned int* small, const unsigned int* pass_count, uint32_t batches,
                                     const unsigned long long* total, unsigned long long capacity,
                                     unsigned int* status) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < batches; b += gridDim.x * blockDim.x)
    status[b] = ((small[8 * (size_t)b + 1] & 1u) ? kGraphStatusOverflow : 0u) |
                (pass_count[(size_t)b * kRefinePasses + kRefinePasses - 1] ? kGraphStatusGeneric : 0u) |
                (*total > capacity ? kBatchGraphStatusRows : 0u);
}

}  // namespace

struct BatchGraphPart {  // one prepared problem batch
  Scene* sc = nullptr;                        // borrowed
  const void* queries = nullptr;              // the caller's records of this batch's problems
  uint32_t p0 = 0, problems = 0;              // global problem range
  uint32_t nq = 0;
  std::vector<unsigned long long> qoff;       // problems + 1, local
  std::vector<double> radius;
  std::vector<uint32_t> kmax;
  QueryPrep qp;
  uint32_t* qrank = nullptr;
  unsigned long long* offsets = nullptr;      // nq + 1, global row offsets once the base is added
};

struct BatchGraph {
  std::vector<BatchGraphPart> parts;
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t problems = 0;
  void* rows = nullptr;                       // the caller's
  unsigned long long capacity = 0;
  std::vector<void*> buffers;
  // scratch shared by the batches (sized for the largest)
  unsigned long long* slab = nullptr;
  uint32_t* counts = nullptr;
  QueryInfo* qinfo = nullptr;
  uint8_t* flags = nullptr;
  uint32_t *heavy_list = nullptr, *heavy_m = nullptr, *heavy_t = nullptr;
  uint32_t *mid_list = nullptr, *big_list = nullptr, *fix_list = nullptr;
  unsigned long long* poff = nullptr;
  void* scan_ws = nullptr;
  RefineDevice D{};
  // per batch
  unsigned int* small = nullptr;        // 8 counters per batch
  unsigned int* pass_count = nullptr;   // kRefinePasses per batch
  unsigned int* queue = nullptr;        // work-queue counter per batch
  unsigned long long* base = nullptr;   // batches + 1: first row of each batch, then the total
  unsigned long long* prob_rows = nullptr;  // problems + 1: first row of each problem, then the total
  unsigned int* status = nullptr;
  unsigned int* status_host = nullptr;      // pinned
  unsigned long long* rows_host = nullptr;  // pinned, problems + 1
  unsigned int persistent_grid = 0;
  bool hybrid = true;  // leaf buckets tested lane- or point-major per bucket (the tuning at creation)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernels = 0;
  uint64_t fallbacks = 0;
};

namespace {

void batch_graph_enqueue(BatchGraph* g, uint32_t i, cudaStream_t s) {
  BatchGraphPart& b = g->parts[i];
  unsigned int* small = g->small + 8 * (size_t)i;
  if (b.nq == 0) {  // no queries in this batch: its problems get no rows
    k_empty_batch_rows<<<div_up(b.problems + 1, 256), 256, 0, s>>>(g->base + i, b.problems, g->prob_rows + b.p0,
                                                                  g->base + i + 1);
    RTDL_LAUNCHED(1);
    return;
  }
  uint32_t kmax = 1;
  for (uint32_t k : b.kmax) kmax = k > kmax ? k : kmax;
  CollectParams C;
  C.S = b.qp.view;
  C.qpts = b.qp.qpts;
  C.qraw = static_cast<const double*>(b.queries);
  C.qstride = b.sc->dim == 3 ? 4 : 3;
  C.qorder = b.qp.qorder;
  C.nq = b.qp.nproc;
  C.kmax = kmax;
  C.bands = b.qp.bands;
  C.warp_prob = b.qp.warp_prob;
  C.prob_kmax = b.qp.prob_kmax;
  C.slab = g->slab;
  C.counts = g->counts;
  C.qinfo = g->qinfo;
  C.flags = g->flags;
  C.heavy_list = g->heavy_list;
  C.heavy_m = g->heavy_m;
  C.heavy_t = g->heavy_t;
  C.mid_list = g->mid_list;
  C.big_list = g->big_list;
  C.small = small;
  C.overflow_out = nullptr;
  C.stats = nullptr;
  const uint32_t np = b.qp.nproc;
  if (g->hybrid)
    k_collect_persistent<kPersistentMinBlocks, kLeafHybrid><<<g->persistent_grid, 256, 0, s>>>(C, g->queue + i);
  else
    k_collect_persistent<kPersistentMinBlocks, kLeafLaneMajor><<<g->persistent_grid, 256, 0, s>>>(C, g->queue + i);
  RTDL_LAUNCHED(1);
  scan_counts_u64_ws(g->counts, b.qp.oorder, b.qp.order_identity, b.nq, b.offsets, g->scan_ws, s);
  k_add_row_base<<<grid_for(b.nq + 1, 256), 256, 0, s>>>(b.offsets, b.nq, g->base + i, g->base + i + 1);
  k_problem_rows<<<div_up(b.problems + 1, 256), 256, 0, s>>>(b.offsets, b.qp.qoff, b.problems, g->prob_rows + b.p0);
  RTDL_LAUNCHED(2);
  RefineDevice D = g->D;
  D.pass_count = g->pass_count + (size_t)i * kRefinePasses;
  enqueue_refine_device(C, b.qp.qprob, b.qp.prob_radius, 0.0, b.qp.prob_kmax, kmax, np, false, g->qinfo, g->flags,
                        small, D, s);
  k_proc_offsets<<<grid_for(np, 256), 256, 0, s>>>(b.qp.qorder, b.qrank, b.offsets, np, g->poff);
  RTDL_LAUNCHED(1);
  EmitParams E;
  E.S = b.sc->view();
  E.nq = np;
  E.slab = g->slab;
  E.qinfo = g->qinfo;
  E.poff = g->poff;
  E.sink.rows = g->rows;
  E.sink.capacity = g->rows ? g->capacity : 0;
  E.sink.ranked = 0;
  E.fix_list = g->fix_list;
  E.fix_count = small + 4;
  k_emit<<<emit_grid(np), kEmitThreads, 0, s>>>(E);
  k_emit_list<4, true><<<kStrideBlocks, kEmitListThreads, 0, s>>>(E, g->mid_list, 0, small + 2);
  k_emit_list<8, false><<<kStrideBlocks, kEmitListThreads, 0, s>>>(E, g->big_list, 0, small + 3);
  k_emit_fixup<<<kSmCount * 4, kFixupThreads, 0, s>>>(E);
  RTDL_LAUNCHED(4);
}

void batch_graph_release(BatchGraph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  g->exec = nullptr;
  g->graph = nullptr;
}

void batch_graph_capture(BatchGraph* g) {
  batch_graph_release(g);
  cudaStream_t s = g->stream;
  const uint32_t B = (uint32_t)g->parts.size();
  const unsigned long long before = launches_counted();
  RTDL_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->small, 0, sizeof(unsigned int) * 8 * (size_t)B, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->pass_count, 0, sizeof(unsigned int) * kRefinePasses * (size_t)B, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->queue, 0, sizeof(unsigned int) * B, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->base, 0, sizeof(unsigned long long), s));
    for (uint32_t i = 0; i < B; ++i) batch_graph_enqueue(g, i, s);
    k_batch_graph_status<<<div_up(B, 256), 256, 0, s>>>(g->small, g->pass_count, B, g->base + B, g->capacity,
                                                        g->status);
    RTDL_LAUNCHED(1);
  } catch (...) {
    cudaGraph_t partial = nullptr;
    cudaStreamEndCapture(s, &partial);
    if (partial) cudaGraphDestroy(partial);
    cudaGetLastError();
    count_launches(-(int)(launches_counted() - before));
    throw;
  }
  count_launches(-(int)(launches_counted() - before));  // counted when a replay launches them
  RTDL_CUDA_CHECK(cudaStreamEndCapture(s, &g->graph));
  RTDL_CUDA_CHECK(cudaGraphInstantiate(&g->exec, g->graph, 0));
  size_t n = 0;
  RTDL_CUDA_CHECK(cudaGraphGetNodes(g->graph, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  RTDL_CUDA_CHECK(cudaGraphGetNodes(g->graph, nodes.data(), &n));
  g->kernels = 0;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    RTDL_CUDA_CHECK(cudaGraphNodeGetType(nodes[i], &t));
    if (t == cudaGraphNodeTypeKernel) ++g->kernels;
  }
}

}  // namespace

BatchGraph* batch_graph_create(Scene* const* batches, uint32_t batch_count, const void* queries_dev,
                               const unsigned long long* query_offsets, const double* radius, const uint32_t* kmax,
                               void* rows_dev, unsigned long long rows_capacity) {
  if (batch_count == 0) throw std::runtime_error("a batch graph needs at least one problem batch");
  if (!batches || !query_offsets || !radius || !kmax)
    throw std::runtime_error("batches, query_offsets, radius and k_max must not be null");
  for (uint32_t i = 0; i < batch_count; ++i) {
    if (!batches[i] || batches[i]->problems == 0)
      throw std::runtime_error("batch graph inputs must be problem batch handles");
    if (batches[i]->dim != batches[0]->dim) throw std::runtime_error("problem batches of a graph must share a dimension");
  }
  BatchGraph* g = new BatchGraph();
  try {
    RTDL_CUDA_CHECK(cudaGetDevice(&g->device));
    RTDL_CUDA_CHECK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    cudaStream_t s = g->stream;
    g->rows = rows_dev;
    g->capacity = rows_dev ? rows_capacity : 0;
    uint32_t p0 = 0, most_np = 0, most_nq = 0;
    const size_t rec = batches[0]->dim == 2 ? sizeof(RtdlPoint) : sizeof(RtdlPoint3D);
    g->parts.reserve(batch_count);
    for (uint32_t i = 0; i < batch_count; ++i) {
      Scene* sc = batches[i];
      RTDL_CUDA_CHECK(cudaStreamSynchronize(sc->stream));  // built on its own stream
      g->parts.emplace_back();
      BatchGraphPart& b = g->parts.back();
      b.sc = sc;
      b.p0 = p0;
      b.problems = sc->problems;
      const unsigned long long q0 = query_offsets[p0], q1 = query_offsets[p0 + sc->problems];
      if (q1 < q0 || q1 - q0 > 0xFFFFFFFFull - 32) throw std::runtime_error("query offsets must be non-decreasing");
      b.nq = (uint32_t)(q1 - q0);
      if (b.nq > 0 && !queries_dev) throw std::runtime_error("query_points_dev must not be null when queries exist");
      b.queries = static_cast<const char*>(queries_dev) + q0 * rec;
      b.qoff.resize(sc->problems + 1);
      for (uint32_t p = 0; p <= sc->problems; ++p) b.qoff[p] = query_offsets[p0 + p] - q0;
      b.radius.assign(radius + p0, radius + p0 + sc->problems);
      b.kmax.assign(kmax + p0, kmax + p0 + sc->problems);
      for (uint32_t p = 0; p < sc->problems; ++p) {
        if (b.qoff[p + 1] < b.qoff[p]) throw std::runtime_error("query offsets must be non-decreasing");
        if (!(b.radius[p] >= 0.0)) throw std::runtime_error("radius must be non-negative");
        if (b.kmax[p] < 1 || b.kmax[p] > 64) throw std::runtime_error("a problem batch takes k_max in [1, 64]");
      }
      if (b.nq > 0) {
        BatchSpec bs;
        bs.problems = sc->problems;
        bs.qoff = b.qoff.data();
        bs.radius = b.radius.data();
        bs.kmax = b.kmax.data();
        b.qp = prepare_queries_batch(sc, b.queries, b.nq, bs, s);
        b.qrank = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * b.nq, s));
        k_invert<<<grid_for(b.nq, 256), 256, 0, s>>>(b.qp.oorder, b.nq, b.qp.order_identity, b.qrank);
        RTDL_LAUNCHED(1);
      }
      b.offsets = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * ((size_t)b.nq + 1), s));
      RTDL_CUDA_CHECK(cudaMemsetAsync(b.offsets, 0, sizeof(unsigned long long) * ((size_t)b.nq + 1), s));
      most_np = b.qp.nproc > most_np ? b.qp.nproc : most_np;
      most_nq = b.nq > most_nq ? b.nq : most_nq;
      p0 += sc->problems;
    }
    g->problems = p0;
    const size_t n = most_np ? most_np : 1, nqm = most_nq ? most_nq : 1, B = batch_count;
    auto alloc = [&](size_t bytes) {
      void* p = dev_alloc(bytes ? bytes : 1, s);
      g->buffers.push_back(p);
      return p;
    };
    g->slab = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * slab_base((uint32_t)n)));
    g->counts = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->qinfo = static_cast<QueryInfo*>(alloc(sizeof(QueryInfo) * n));
    g->flags = static_cast<uint8_t*>(alloc(nqm));
    g->heavy_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->heavy_m = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->heavy_t = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->mid_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->big_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->fix_list = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
    g->poff = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * n));
    g->scan_ws = alloc(scan_workspace_bytes((uint32_t)nqm));
    for (int k = 0; k < 2; ++k) {
      g->D.work[k] = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
      g->D.rad[k] = static_cast<double*>(alloc(sizeof(double) * n));
      g->D.lo[k] = static_cast<double*>(alloc(sizeof(double) * n));
      g->D.hi[k] = static_cast<double*>(alloc(sizeof(double) * n));
      g->D.full[k] = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * n));
      g->D.frad[k] = static_cast<double*>(alloc(sizeof(double) * n));
    }
    g->D.cnt = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->D.gen_qin = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->D.gen_m = static_cast<uint32_t*>(alloc(sizeof(uint32_t) * nqm));
    g->D.gen_rad = static_cast<double*>(alloc(sizeof(double) * nqm));
    g->small = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * 8 * B));
    g->pass_count = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * kRefinePasses * B));
    g->queue = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * B));
    g->base = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * (B + 1)));
    g->prob_rows = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long) * ((size_t)g->problems + 1)));
    g->status = static_cast<unsigned int*>(alloc(sizeof(unsigned int) * B));
    RTDL_CUDA_CHECK(cudaMemsetAsync(g->prob_rows, 0, sizeof(unsigned long long) * ((size_t)g->problems + 1), s));
    RTDL_CUDA_CHECK(cudaMallocHost(&g->status_host, sizeof(unsigned int) * B));
    RTDL_CUDA_CHECK(cudaMallocHost(&g->rows_host, sizeof(unsigned long long) * ((size_t)g->problems + 1)));
    g->hybrid = tuning().traversal == 4;
    int per_sm = 0;
    if (g->hybrid)
      RTDL_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, k_collect_persistent<kPersistentMinBlocks, kLeafHybrid>, 256, 0));
    else
      RTDL_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, k_collect_persistent<kPersistentMinBlocks, kLeafLaneMajor>, 256, 0));
    int sms = kSmCount;
    RTDL_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    g->persistent_grid = (unsigned int)(sms * (per_sm > 0 ? per_sm : 1));
    // bad coordinates or a failed sort wait in a batch or its queries fail creation
    Readback* rb = pinned_readback();
    for (auto& b : g->parts) {
      RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->scene_bad, &b.sc->stats->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                      s));
      rb->query_bad = 0;
      if (b.qp.qst)
        RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->query_bad, &b.qp.qst->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                        s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      throw_if_bad(rb->query_bad | rb->scene_bad);
    }
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // everything allocated and prepared before capture
    batch_graph_capture(g);
  } catch (...) {
    batch_graph_destroy(g);
    throw;
  }
  return g;
}

void batch_graph_launch(BatchGraph* g, cudaStream_t s) {
  count_launches(g->kernels);
  if (s && s != g->stream) {
    cudaEvent_t e;
    RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    RTDL_CUDA_CHECK(cudaEventRecord(e, s));
    RTDL_CUDA_CHECK(cudaStreamWaitEvent(g->stream, e, 0));
    RTDL_CUDA_CHECK(cudaGraphLaunch(g->exec, g->stream));
    RTDL_CUDA_CHECK(cudaEventRecord(e, g->stream));
    RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, e, 0));
    note_cleanup_error(cudaEventDestroy(e), "cudaEventDestroy");
  } else {
    RTDL_CUDA_CHECK(cudaGraphLaunch(g->exec, g->stream));
  }
}

void batch_graph_replay(BatchGraph* g, unsigned long long* row_offsets_out, unsigned int* status_out) {
  batch_graph_launch(g, nullptr);
  cudaStream_t s = g->stream;
  const uint32_t B = (uint32_t)g->parts.size();
  RTDL_CUDA_CHECK(cudaMemcpyAsync(g->status_host, g->status, sizeof(unsigned int) * B, cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(g->rows_host, g->prob_rows, sizeof(unsigned long long) * ((size_t)g->problems + 1),
                                  cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  unsigned int all = 0;
  for (uint32_t i = 0; i < B; ++i) {
    const unsigned int st = g->status_host[i];
    all |= st;
    if (st & kGraphStatusOverflow) throw std::runtime_error("LBVH traversal stack overflow");
    if ((st & kGraphStatusGeneric) && g->rows && !(st & kBatchGraphStatusRows)) {
      // heavy queries the refinement did not resolve: this batch's rows by the plain batch call
      BatchGraphPart& b = g->parts[i];
      const unsigned long long first = g->rows_host[b.p0];
      std::vector<unsigned long long> local(b.problems + 1);
      BatchSpec bs;
      bs.problems = b.problems;
      bs.qoff = b.qoff.data();
      bs.radius = b.radius.data();
      bs.kmax = b.kmax.data();
      bs.row_offsets = local.data();
      run_query_batch(b.sc, b.queries, bs, static_cast<char*>(g->rows) + first * sizeof(RtdlFixedRadiusNeighborRow),
                      g->capacity - first, nullptr, nullptr, s, nullptr);
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      ++g->fallbacks;
    }
  }
  if (status_out) *status_out = all;
  if (row_offsets_out)
    std::memcpy(row_offsets_out, g->rows_host, sizeof(unsigned long long) * ((size_t)g->problems + 1));
}

uint32_t batch_graph_problems(const BatchGraph* g) { return g->problems; }
int batch_graph_kernels(const BatchGraph* g) { return g->kernels; }
uint64_t batch_graph_fallbacks(const BatchGraph* g) { return g->fallbacks; }

void batch_graph_destroy(BatchGraph* g) {
  if (!g) return;
  if (g->stream) sync_quietly(g->stream);
  batch_graph_release(g);
  cudaStream_t s = g->stream;
  for (auto& b : g->parts) {
    if (b.nq > 0) free_prep(b.qp, s);
    dev_free(b.qrank, s);
    dev_free(b.offsets, s);
  }
  for (void* p : g->buffers) dev_free(p, s);
  if (g->status_host) note_cleanup_error(cudaFreeHost(g->status_host), "cudaFreeHost");
  if (g->rows_host) note_cleanup_error(cudaFreeHost(g->rows_host), "cudaFreeHost");
  if (s) {
    sync_quietly(s);
    note_cleanup_error(cudaStreamDestroy(s), "cudaStreamDestroy");
  }
  delete g;
}

}  // namespace rtdl_b200
