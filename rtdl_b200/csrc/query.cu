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
__global__ void k_bands(const PointStats* scene, const PointStats* queries, double radius, int has_radius,
                        DevBands* out) {
  if (threadIdx.x != 0) return;
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
  *out = b;
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

// Exact comparison of two candidates by the reference's sort key.
__device__ __noinline__ bool exact_before(const Ctx& c, uint32_t ia, uint32_t ib) {
  const double da = __dsqrt_rn(exact_d2(c, ia)), db = __dsqrt_rn(exact_d2(c, ib));
  if (da != db) return da < db;
  const uint32_t na = __float_as_uint(__ldg(&c.pts[ia].w)), nb = __float_as_uint(__ldg(&c.pts[ib].w));
  if (na != nb) return na < nb;
  return __ldg(&c.perm[ia]) < __ldg(&c.perm[ib]);
}

// True when candidate a orders strictly before candidate b.  FP32 keys decide
// whenever they are further apart than the error band; otherwise FP64 does.
__device__ __forceinline__ bool before(const Ctx& c, float ka, uint32_t ia, float kb, uint32_t ib) {
  const float d = kb - ka;
  const float t = key_tol(c, fmaxf(ka, kb));
  if (d > t) return true;
  if (-d > t) return false;
  return exact_before(c, ia, ib);
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
};

// One thread per query, queries in Morton order so a warp walks neighbouring
// subtrees.  KNN == false: radius-limited (fixed_radius_neighbors and
// bounded_knn_rows); KNN == true: k nearest.
template <bool KNN>
__global__ void __launch_bounds__(256) k_pass1(Pass1Params P) {
  extern __shared__ uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int L = P.L;
  uint32_t* lkey = smem + (size_t)warp * 64 * L;
  uint32_t* lidx = lkey + 32 * L;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.nq) return;
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
    }
    lkey[pos * 32 + lane] = __float_as_uint(key);
    lidx[pos * 32 + lane] = idx;
    if (len == L) {
      klast = __uint_as_float(lkey[(L - 1) * 32 + lane]);
      ilast = lidx[(L - 1) * 32 + lane];
    }
  };

  auto visit_leaf = [&](int first, int cnt) {
    for (int i = first; i < first + cnt; ++i) {
      const float4 p = __ldg(&S.pts[i]);
      const float dx = p.x - c.qx, dy = p.y - c.qy, dz = p.z - c.qz;
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      if (!KNN) {
        if (d2 > B.hi2) continue;
        if (prune && !before(c, d2, (uint32_t)i, klast, ilast)) continue;
        if (d2 >= B.lo2 && exact_d2(c, (uint32_t)i) > B.r2) continue;
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

  auto box_ok = [&](float kb) -> bool {
    if (!KNN && kb > B.box_hi2) return false;
    const bool full = KNN ? (len == L) : prune;
    if (full && box_beyond(c, kb, klast)) return false;
    return true;
  };

  if (S.n > 0) {
    if (S.root_cnt > 0) {
      visit_leaf(S.root_ref, S.root_cnt);
    } else {
      int2 stack[kStackDepth];
      int sp = 0;
      int cur = S.root_ref;
      while (true) {
        const float4* nd = S.nodes + 4 * (size_t)cur;
        const float4 a = __ldg(nd), b = __ldg(nd + 1), e = __ldg(nd + 2), f = __ldg(nd + 3);
        float k0 = box_d2(c.qx, c.qy, c.qz, a, b), k1 = box_d2(c.qx, c.qy, c.qz, e, f);
        int r0 = __float_as_int(a.w), n0 = __float_as_int(b.w);
        int r1 = __float_as_int(e.w), n1 = __float_as_int(f.w);
        if (k1 < k0) {
          const float tk = k0; k0 = k1; k1 = tk;
          const int tr = r0; r0 = r1; r1 = tr;
          const int tn = n0; n0 = n1; n1 = tn;
        }
        int next = -1;
        if (box_ok(k0)) {
          if (n0) visit_leaf(r0, n0);
          else next = r0;
        }
        if (box_ok(k1)) {
          if (n1) {
            visit_leaf(r1, n1);
          } else if (next < 0) {
            next = r1;
          } else {
            if (sp >= kStackDepth) {
              atomicOr(P.error, 1u);
              break;
            }
            stack[sp++] = make_int2(r1, __float_as_int(k1));
          }
        }
        if (next < 0) {
          while (sp > 0) {
            const int2 en = stack[--sp];
            if (box_ok(__int_as_float(en.y))) {
              next = en.x;
              break;
            }
          }
          if (next < 0) break;
        }
        cur = next;
      }
    }
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

__device__ __forceinline__ bool heavy_greater(const HeavyEntry& a, const HeavyEntry& b, const uint32_t* perm) {
  if (a.key != b.key) return a.key > b.key;
  if (a.nid != b.nid) return a.nid > b.nid;
  if (a.sidx == kNone || b.sidx == kNone) return a.sidx == kNone && b.sidx != kNone;
  return perm[a.sidx] > perm[b.sidx];
}

__global__ void __launch_bounds__(kHeavyThreads)
    k_heavy_sort(const unsigned long long* seg_off, const uint32_t* seg_size, HeavyEntry* scratch,
                 const uint32_t* perm) {
  HeavyEntry* e = scratch + seg_off[blockIdx.x];
  const uint32_t P2 = seg_size[blockIdx.x];
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
};

// A warp per query in output order writes its rows with the exact FP64 distance.
__global__ void __launch_bounds__(kExpandThreads) k_expand(ExpandParams P) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const bool ids_sorted = P.bands->ids_sorted != 0;
  const bool scene_inexact = *P.S.inexact != 0;
  for (uint64_t j = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < P.nq; j += warps) {
    const uint32_t qin = ids_sorted ? (uint32_t)j : P.oorder[j];
    const uint32_t cnt = P.counts[qin];
    const uint8_t fl = P.flags[qin];
    if (P.overflow_out != nullptr && lane == 0) P.overflow_out[qin] = fl & 1;
    if (cnt == 0 || P.rows == nullptr) continue;
    const unsigned long long base = P.offsets[j];
    const uint32_t qid = __float_as_uint(P.qpts[qin].w);
    const double* r = P.qraw + (size_t)qin * P.qstride;
    const double ex = r[1], ey = r[2], ez = P.qstride == 4 ? r[3] : 0.0;
    const uint32_t* src = (fl & 2) ? P.heavy_out + P.heavy_out_off[P.temp[(size_t)qin * P.L]]
                                   : P.temp + (size_t)qin * P.L;
    for (uint32_t s = lane; s < cnt; s += 32) {
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

struct Readback {
  unsigned long long rows;
  unsigned int heavy;
  unsigned int error;
  unsigned int scene_bad;
  unsigned int query_bad;
  unsigned int pad[2];
};

Readback* pinned_readback() {
  thread_local Readback* rb = nullptr;
  if (rb == nullptr) RTDL_CUDA_CHECK(cudaMallocHost(&rb, sizeof(Readback)));
  return rb;
}

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
  DevBands* bands = nullptr;
  uint32_t* qorder = nullptr;
  uint32_t* oorder = nullptr;
};

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
  uint32_t* qcodes = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  morton_codes(qp.qpts, nq, sc->dim, sc->stats, qcodes, s);
  iota_u32(qp.qorder, nq, s);
  radix_sort_pairs(qcodes, qp.qorder, nq, 0, sc->dim == 3 ? 30 : 32, nullptr, s);
  if (want_output_order) {
    qp.oorder = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
    k_extract_ids<<<grid_for(nq, 256), 256, 0, s>>>(qp.qpts, nq, qcodes);
    RTDL_LAUNCHED(1);
    iota_u32(qp.oorder, nq, s);
    radix_sort_pairs(qcodes, qp.oorder, nq, 0, 32, &qp.bands->ids_sorted, s);
  }
  dev_free(qcodes, s);
  return qp;
}

void free_prep(QueryPrep& qp, cudaStream_t s) {
  dev_free(qp.qst, s);
  dev_free(qp.qpts, s);
  dev_free(qp.bands, s);
  dev_free(qp.qorder, s);
  dev_free(qp.oorder, s);
}

}  // namespace

QueryResult run_query(Scene* sc, const void* queries_dev, uint32_t nq, int predicate, double radius, uint32_t limit,
                      void* rows_dev, size_t rows_capacity, void** rows_alloc, uint8_t* overflow_dev, cudaStream_t s,
                      PhaseTimer* timer) {
  QueryResult res;
  if (rows_alloc) *rows_alloc = nullptr;
  const bool knn = predicate == kKnn;
  const int qstride = sc->dim == 3 ? 4 : 3;
  if (nq == 0) return res;
  if (sc->n == 0) {
    if (overflow_dev) RTDL_CUDA_CHECK(cudaMemsetAsync(overflow_dev, 0, nq, s));
    return res;
  }
  if (timer) timer->mark("start");
  QueryPrep qp = prepare_queries(sc, queries_dev, nq, !knn, radius, true, s);
  if (timer) timer->mark("query_prep");

  const bool all_heavy = knn && limit > (uint32_t)kMaxList;
  const int L = all_heavy ? 1 : (int)(limit < (uint32_t)kMaxList ? limit : (uint32_t)kMaxList);
  uint32_t* counts = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  uint8_t* flags = static_cast<uint8_t*>(dev_alloc(nq, s));
  uint32_t* temp = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (size_t)nq * L, s));
  uint32_t* heavy_list = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  uint32_t* heavy_m = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * nq, s));
  unsigned int* small = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int) * 4, s));  // heavy count, error
  unsigned long long* offsets = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (nq + 1), s));
  RTDL_CUDA_CHECK(cudaMemsetAsync(small, 0, sizeof(unsigned int) * 4, s));

  if (all_heavy) {
    k_mark_all_heavy<<<grid_for(nq, 256), 256, 0, s>>>(qp.qorder, nq, sc->n, limit, counts, flags, temp, heavy_list,
                                                       heavy_m);
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
    if (knn) {
      RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
      k_pass1<true><<<blocks, threads, shm, s>>>(P);
    } else {
      RTDL_CUDA_CHECK(cudaFuncSetAttribute(k_pass1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
      k_pass1<false><<<blocks, threads, shm, s>>>(P);
    }
    RTDL_LAUNCHED(1);
  }
  if (timer) timer->mark("traverse");
  scan_counts_u64(counts, qp.oorder, &qp.bands->ids_sorted, nq, offsets, s);
  if (timer) timer->mark("scan");

  Readback* rb = pinned_readback();
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->rows, offsets + nq, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->heavy, small, sizeof(unsigned int) * 2, cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->scene_bad, &sc->stats->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->query_bad, &qp.qst->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  const Readback r = *rb;
  auto cleanup = [&]() {
    dev_free(counts, s);
    dev_free(flags, s);
    dev_free(temp, s);
    dev_free(heavy_list, s);
    dev_free(heavy_m, s);
    dev_free(small, s);
    dev_free(offsets, s);
    free_prep(qp, s);
  };
  if (r.scene_bad || r.query_bad) {
    cleanup();
    throw std::runtime_error("point coordinates must be finite with magnitude <= 1e18");
  }
  if (r.error & 1u) {
    cleanup();
    throw std::runtime_error("BVH traversal stack overflow");
  }
  res.rows = r.rows;
  res.heavy = r.heavy;

  uint32_t* heavy_out = nullptr;
  unsigned long long* heavy_out_off = nullptr;
  if (r.heavy > 0) {
    const uint32_t H = r.heavy;
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
    if (seg_total > kScratchLimit) {
      cleanup();
      throw std::runtime_error(
          "b200 backend: the generic path for limits above 64 needs more than 4 GiB of sort scratch; "
          "reduce k/k_max or split the query set");
    }
    unsigned long long* d_seg_off = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * H, s));
    uint32_t* d_seg_size = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * H, s));
    heavy_out_off = static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * H, s));
    uint32_t* d_out_cnt = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * H, s));
    HeavyEntry* scratch = static_cast<HeavyEntry*>(dev_alloc(sizeof(HeavyEntry) * seg_total, s));
    heavy_out = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (out_total ? out_total : 1), s));
    RTDL_CUDA_CHECK(cudaMemcpyAsync(d_seg_off, seg_off.data(), sizeof(unsigned long long) * H, cudaMemcpyHostToDevice, s));
    RTDL_CUDA_CHECK(cudaMemcpyAsync(d_seg_size, seg_size.data(), sizeof(uint32_t) * H, cudaMemcpyHostToDevice, s));
    RTDL_CUDA_CHECK(cudaMemcpyAsync(heavy_out_off, out_off.data(), sizeof(unsigned long long) * H, cudaMemcpyHostToDevice, s));
    RTDL_CUDA_CHECK(cudaMemcpyAsync(d_out_cnt, out_cnt.data(), sizeof(uint32_t) * H, cudaMemcpyHostToDevice, s));
    k_heavy_gather<<<H, kHeavyThreads, 0, s>>>(sc->view(), qp.qpts, static_cast<const double*>(queries_dev), qstride,
                                               heavy_list, d_seg_off, d_seg_size, knn ? 1 : 0, qp.bands, scratch,
                                               small + 1);
    k_heavy_sort<<<H, kHeavyThreads, 0, s>>>(d_seg_off, d_seg_size, scratch, sc->perm);
    k_heavy_emit<<<H, kHeavyThreads, 0, s>>>(d_seg_off, heavy_out_off, d_out_cnt, scratch, heavy_out);
    RTDL_LAUNCHED(3);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // the host vectors above are read by the copies
    dev_free(d_seg_off, s);
    dev_free(d_seg_size, s);
    dev_free(d_out_cnt, s);
    dev_free(scratch, s);
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
    E.heavy_out = heavy_out;
    E.heavy_out_off = heavy_out_off;
    E.offsets = offsets;
    E.rows = rows_dev;
    E.capacity = rows_capacity;
    E.ranked = predicate == kFrn ? 0 : 1;
    E.overflow_out = overflow_dev;
    E.error = small + 1;
    const unsigned int blocks = grid_for((uint64_t)nq * 32, kExpandThreads);
    k_expand<<<blocks, kExpandThreads, 0, s>>>(E);
    RTDL_LAUNCHED(1);
  }
  if (timer) timer->mark("emit");
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&rb->error, small + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  const unsigned int late_error = rb->error;
  dev_free(heavy_out, s);
  dev_free(heavy_out_off, s);
  cleanup();
  if (late_error & 6u) throw std::runtime_error("generic neighbor path produced an inconsistent candidate count");
  return res;
}

HausdorffResult run_directed_hausdorff(Scene* sc, const void* queries_dev, uint32_t nq, double* nearest_dist_dev,
                                       uint32_t* nearest_id_dev, cudaStream_t s, PhaseTimer* timer) {
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
  k_pass1<true><<<div_up(nq, threads), threads, (size_t)threads * 8, s>>>(P);
  RTDL_LAUNCHED(1);
  if (timer) timer->mark("traverse");
  const unsigned int blocks = grid_for(nq, 256) < 2 * kSmCount ? grid_for(nq, 256) : 2 * kSmCount;
  Witness* partial = static_cast<Witness*>(dev_alloc(sizeof(Witness) * blocks, s));
  Witness* best = static_cast<Witness*>(dev_alloc(sizeof(Witness), s));
  k_nearest_reduce<<<blocks, 256, 0, s>>>(sc->view(), qp.qpts, static_cast<const double*>(queries_dev), qstride, nq,
                                          temp, nearest_dist_dev, nearest_id_dev, partial);
  k_witness_final<<<1, 32, 0, s>>>(partial, (int)blocks, best);
  RTDL_LAUNCHED(2);
  Readback* rb = pinned_readback();
  Witness* hw = reinterpret_cast<Witness*>(rb);
  static_assert(sizeof(Witness) <= sizeof(Readback), "readback buffer too small");
  RTDL_CUDA_CHECK(cudaMemcpyAsync(hw, best, sizeof(Witness), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  const Witness w = *hw;
  if (timer) timer->mark("reduce");
  unsigned int bad[2] = {0, 0};
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&bad[0], &sc->stats->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaMemcpyAsync(&bad[1], &qp.qst->bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  dev_free(counts, s);
  dev_free(flags, s);
  dev_free(temp, s);
  dev_free(small, s);
  dev_free(partial, s);
  dev_free(best, s);
  free_prep(qp, s);
  if (bad[0] || bad[1]) throw std::runtime_error("point coordinates must be finite with magnitude <= 1e18");
  HausdorffResult out;
  unsigned long long db = w.dist;
  memcpy(&out.distance, &db, sizeof(double));
  out.source_id = w.qid;
  out.target_id = w.nid;
  return out;
}

}  // namespace rtdl_b200
