// lbvh.cu -- on-device LBVH over the search points.
//
// Build steps, all on one stream with no host round trip:
//   1. prep:    AoS FP64 records (RtdlPoint / RtdlPoint3D) -> float4 {x, y, z, id}
//               plus set statistics (box, largest |coordinate|, FP32
//               exactness, finiteness, id order);
//   2. morton:  30-bit (3D, 10 bits per axis) or 32-bit (2D, 16 bits per
//               axis) codes relative to the set's box;
//   3. sort:    stable radix sort of (code, input index) pairs (sort_scan.cu);
//   4. gather:  points into code order (coalesced float4 stores); exact FP64
//               coordinates alongside when the set is not FP32-exact;
//   5. karras:  one thread per internal node finds its key range and split
//               (Karras 2012, "Maximizing Parallelism in the Construction of
//               BVHs, Octrees, and k-d Trees"; equal codes are split on the
//               index, so duplicates are handled);
//   6. collapse: the tree the traversal sees keeps an internal node only
//               while it covers more than leaf_size points; smaller subtrees
//               (and single points hanging off large nodes) become leaf
//               buckets;
//   7. refit:   bottom-up boxes of the collapsed tree, one thread per bucket,
//               an atomic arrival counter per node lets the second child to
//               arrive continue;
//   8. compact: the collapsed tree is written in depth-first pre-order as
//               32-B records {box, leaf reference or "internal", rope}: the
//               left child of an internal node is the next record, and the
//               rope is the record that follows the node's subtree.  A walk
//               is then stackless and reads nearly consecutive memory.  A
//               node's pre-order index is 2 L + depth - r, with L the leaf
//               buckets left of it, depth its depth and r the right turns on
//               its root path; its rope is the right child of the internal
//               node whose split equals the node's last point.
#include <cuda/atomic>

#include "internal.cuh"

namespace rtdl_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kLeafFlag = 0x40000000;  // child is a single point (Karras leaf)

inline unsigned int grid_for(uint64_t n, int threads = kThreads) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  const uint64_t cap = (uint64_t)kSmCount * 16;
  return (unsigned int)(b < cap ? b : cap);
}

constexpr int kPrepThreads = 256;

// k_prep's grid: enough blocks to fill the SMs a few times over, few enough
// that the per-block atomics stay cheap.
inline unsigned int prep_grid(uint64_t n) {
  uint64_t b = (n + kPrepThreads - 1) / kPrepThreads;
  if (b < 1) b = 1;
  const uint64_t cap = (uint64_t)kSmCount * 4;
  return (unsigned int)(b < cap ? b : cap);
}

template <int DIM>
__global__ void __launch_bounds__(kPrepThreads) k_prep(const double* __restrict__ raw, uint32_t n, float4* __restrict__ out,
                       PointStats* __restrict__ st) {
  constexpr int kStride = DIM == 3 ? 4 : 3;  // record size in doubles (id occupies the first slot)
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  double max_abs = 0.0;
  unsigned int inexact = 0, bad = 0, unsorted = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double* r = raw + i * kStride;
    const uint32_t id = *reinterpret_cast<const uint32_t*>(r);
    double c[3] = {r[1], r[2], DIM == 3 ? r[3] : 0.0};
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double v = c[a];
      const double av = fabs(v);
      if (!(av <= kMaxCoordinate)) bad = 1;  // also catches NaN
      f[a] = __double2float_rn(v);
      if ((double)f[a] != v) inexact = 1;
      lo[a] = fminf(lo[a], f[a]);
      hi[a] = fmaxf(hi[a], f[a]);
      max_abs = fmax(max_abs, av);
    }
    if (i > 0) {
      const uint32_t prev = *reinterpret_cast<const uint32_t*>(raw + (i - 1) * kStride);
      if (id < prev) unsorted = 1;
    }
    out[i] = make_float4(f[0], f[1], f[2], __uint_as_float(id));
  }
  // warp reduction, then a block reduction through shared memory, then one set
  // of atomics per block (same-address atomics from every warp would
  // serialise in L2)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    max_abs = fmax(max_abs, __shfl_xor_sync(0xffffffffu, max_abs, o));
    inexact |= __shfl_xor_sync(0xffffffffu, inexact, o);
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    unsorted |= __shfl_xor_sync(0xffffffffu, unsorted, o);
  }
  __shared__ float s_lo[3][kPrepThreads / 32], s_hi[3][kPrepThreads / 32];
  __shared__ double s_abs[kPrepThreads / 32];
  __shared__ unsigned int s_flags[kPrepThreads / 32];
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      s_lo[a][warp] = lo[a];
      s_hi[a][warp] = hi[a];
    }
    s_abs[warp] = max_abs;
    s_flags[warp] = inexact | (bad << 1) | (unsorted << 2);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int fl = 0;
    for (int w = 0; w < nwarps; ++w) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(lo[a], s_lo[a][w]);
        hi[a] = fmaxf(hi[a], s_hi[a][w]);
      }
      max_abs = fmax(max_abs, s_abs[w]);
      fl |= s_flags[w];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (lo[a] <= hi[a]) {
        atomicMin(&st->lo[a], float_to_ordered(lo[a]));
        atomicMax(&st->hi[a], float_to_ordered(hi[a]));
      }
    }
    atomicMax(&st->max_abs_bits, (unsigned long long)__double_as_longlong(max_abs));
    if (fl & 1u) atomicOr(&st->inexact, 1u);
    if (fl & 2u) atomicOr(&st->bad, kBadCoordinates);
    if (fl & 4u) atomicOr(&st->ids_unsorted, 1u);
  }
}

__global__ void k_reset_stats(PointStats* st) {
  if (threadIdx.x == 0) {
    for (int a = 0; a < 3; ++a) {
      st->lo[a] = 0xFFFFFFFFu;
      st->hi[a] = 0u;
    }
    st->max_abs_bits = 0ull;
    st->inexact = 0u;
    st->bad = 0u;
    st->ids_unsorted = 0u;
    st->pad = 0u;
  }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {  // 10 bits -> every third bit
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__device__ __forceinline__ uint32_t spread16(uint32_t v) {  // 16 bits -> every other bit
  v &= 0xFFFFu;
  v = (v | (v << 8)) & 0x00FF00FFu;
  v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

__global__ void k_morton(const float4* __restrict__ pts, uint32_t n, int dim, const PointStats* __restrict__ box,
                         uint32_t* __restrict__ codes) {
  float lo[3], scale[3];
  const float cells = dim == 3 ? 1023.0f : 65535.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const unsigned int ol = box->lo[a], oh = box->hi[a];
    const bool empty = ol == 0xFFFFFFFFu;
    const float l = empty ? 0.f : ordered_to_float(ol);
    const float h = empty ? 0.f : ordered_to_float(oh);
    lo[a] = l;
    const float ext = h - l;
    scale[a] = (ext > 0.f && isfinite(ext)) ? cells / ext : 0.f;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float4 p = pts[i];
    const float c[3] = {p.x, p.y, p.z};
    uint32_t q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float t = (c[a] - lo[a]) * scale[a];
      t = fminf(fmaxf(t, 0.f), cells);
      q[a] = (uint32_t)t;
    }
    codes[i] = dim == 3 ? (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2])
                        : (spread16(q[0]) << 1) | spread16(q[1]);
  }
}

template <int DIM>
__global__ void k_gather(const float4* __restrict__ in, const double* __restrict__ raw, const uint32_t* __restrict__ perm,
                         uint32_t n, float4* __restrict__ out, double* __restrict__ out64,
                         const PointStats* __restrict__ st) {
  constexpr int kStride = DIM == 3 ? 4 : 3;
  const bool want64 = st->inexact != 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t src = perm[i];
    out[i] = in[src];
    if (want64) {
      const double* r = raw + (uint64_t)src * kStride;
      out64[3 * i + 0] = r[1];
      out64[3 * i + 1] = r[2];
      out64[3 * i + 2] = DIM == 3 ? r[3] : 0.0;
    }
  }
}

// Common-prefix length of the (code, index) keys of sorted positions i and j;
// -1 outside [0, n).
__device__ __forceinline__ int prefix_len(const uint32_t* __restrict__ codes, int64_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

__global__ void k_karras(const uint32_t* __restrict__ codes, uint32_t n, int* __restrict__ child_l,
                         int* __restrict__ child_r, int* __restrict__ first, int* __restrict__ last,
                         int* __restrict__ parent_int, int* __restrict__ parent_leaf,
                         int* __restrict__ right_of_split) {
  const int64_t nn = n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn - 1; i += (int64_t)gridDim.x * blockDim.x) {
    const int d = (prefix_len(codes, nn, i, i + 1) - prefix_len(codes, nn, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = prefix_len(codes, nn, i, i - d);
    int64_t lmax = 2;
    while (prefix_len(codes, nn, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (prefix_len(codes, nn, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = prefix_len(codes, nn, i, j);
    int64_t s = 0;
    int64_t t = l;
    do {
      t = (t + 1) >> 1;
      if (prefix_len(codes, nn, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
    const int64_t lo = i < j ? i : j;
    const int64_t hi = i < j ? j : i;
    int cl, cr;
    const int up_l = (int)i << 1, up_r = ((int)i << 1) | 1;
    if (lo == gamma) {
      cl = (int)gamma | kLeafFlag;
      parent_leaf[gamma] = up_l;
    } else {
      cl = (int)gamma;
      parent_int[gamma] = up_l;
    }
    if (hi == gamma + 1) {
      cr = (int)(gamma + 1) | kLeafFlag;
      parent_leaf[gamma + 1] = up_r;
    } else {
      cr = (int)(gamma + 1);
      parent_int[gamma + 1] = up_r;
    }
    child_l[i] = cl;
    child_r[i] = cr;
    first[i] = (int)lo;
    last[i] = (int)hi;
    // node index of the right child: internal nodes keep their index, point
    // leaves follow the n - 1 internal nodes
    right_of_split[gamma] = (cr & kLeafFlag) ? (int)(nn - 1) + (cr & ~kLeafFlag) : cr;
  }
}

// Karras entities: internal node k for e < n - 1, point e - (n - 1) otherwise.
struct Ent {
  const int* child_l;
  const int* child_r;
  const int* first;
  const int* last;
  const int* parent_int;
  const int* parent_leaf;
  uint32_t n;
  __device__ __forceinline__ bool is_point(int e) const { return e >= (int)n - 1; }
  __device__ __forceinline__ int lo(int e) const { return is_point(e) ? e - ((int)n - 1) : first[e]; }
  __device__ __forceinline__ int hi(int e) const { return is_point(e) ? e - ((int)n - 1) : last[e]; }
  // parent link: (parent index << 1) | 1 when e is its parent's right child;
  // -1 at the root
  __device__ __forceinline__ int link(int e) const {
    return is_point(e) ? parent_leaf[e - ((int)n - 1)] : parent_int[e];
  }
  __device__ __forceinline__ int parent(int e) const {
    const int v = link(e);
    return v < 0 ? -1 : v >> 1;
  }
  __device__ __forceinline__ int child_code(int e) const {  // as stored in child_l / child_r
    return is_point(e) ? ((e - ((int)n - 1)) | kLeafFlag) : e;
  }
};

__device__ __forceinline__ uint32_t problem_of(uint32_t code, int code_bits) {
  return code_bits >= 32 ? 0u : code >> code_bits;
}

// True when entity e's points belong to more than one problem of a batch
// (codes == nullptr: a single problem).
__device__ __forceinline__ bool spans_problems(const Ent& E, int e, const uint32_t* codes, int code_bits) {
  return codes != nullptr && problem_of(codes[E.lo(e)], code_bits) != problem_of(codes[E.hi(e)], code_bits);
}

// Marks the nodes of the collapsed tree (flag bit 0) and its leaf buckets
// (bit 1); a bucket sets leaf_start at its first point and records itself in
// bucket_at there.  In a problem batch a
// node whose points span problems is never a bucket, so each problem keeps a
// subtree of its own.
__global__ void k_mark_collapsed(Ent E, int leaf_size, const uint32_t* codes, int code_bits,
                                 uint8_t* __restrict__ flags, uint32_t* __restrict__ leaf_start,
                                 int* __restrict__ bucket_at) {
  const int total = 2 * (int)E.n - 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int par = e == 0 ? -1 : E.parent(e);
    const bool in = e == 0 || (par >= 0 && (E.hi(par) - E.lo(par) + 1 > leaf_size ||
                                            spans_problems(E, par, codes, code_bits)));
    uint8_t f = 0;
    if (in) {
      f = 1;
      if (E.is_point(e) || (E.hi(e) - E.lo(e) + 1 <= leaf_size && !spans_problems(E, e, codes, code_bits))) {
        f |= 2;
        leaf_start[E.lo(e)] = 1u;
        bucket_at[E.lo(e)] = e;
      }
    }
    flags[e] = f;
  }
}

// Narrows the bucket counts to 32 bits and lists the buckets' entities in
// point order (bucket b = the b-th bucket from the left).
__global__ void k_bucket_list(const uint64_t* __restrict__ leaves_before, const uint32_t* __restrict__ leaf_start,
                              const int* __restrict__ bucket_at, uint32_t n, uint32_t* __restrict__ leaves_before32,
                              int* __restrict__ buckets) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = leaves_before[i];
    leaves_before32[i] = (uint32_t)b;
    if (i < n && leaf_start[i]) buckets[b] = bucket_at[i];
  }
}

// Boxes of the collapsed tree, bottom-up from its leaf buckets: one thread
// per bucket takes the min / max over the bucket's points (a contiguous run
// of at most 32 sorted points), then walks towards the root; at each internal
// node an acquire-release arrival counter lets the second child to arrive
// continue (the first stops).  The walking thread carries its subtree's box
// in registers and reads only the sibling's box.  Min and max are exact, so
// the boxes equal a refit from the single points.  Only internal nodes of the
// collapsed tree get a box; a single-point bucket's box is its point.
__global__ void __launch_bounds__(kThreads) k_refit_buckets(Ent E, const int* __restrict__ buckets,
                                                           const uint32_t* __restrict__ bucket_count,
                                                           const float4* __restrict__ pts,
                                                           unsigned int* __restrict__ arrivals, float4* boxes) {
  const uint32_t m = *bucket_count;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < m; b += (uint64_t)gridDim.x * blockDim.x) {
    const int e = buckets[b];
    const int a = E.lo(e), z = E.hi(e);
    const float4 p0 = pts[a];
    float4 lo = make_float4(p0.x, p0.y, p0.z, 0.f), hi = lo;
#pragma unroll 4
    for (int j = a + 1; j <= z; ++j) {
      const float4 p = pts[j];
      lo = make_float4(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z), 0.f);
      hi = make_float4(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z), 0.f);
    }
    if (!E.is_point(e)) {
      __stcg(&boxes[2 * e], lo);
      __stcg(&boxes[2 * e + 1], hi);
    }
    int v = E.link(e);
    while (v >= 0) {
      const int p = v >> 1;
      // the node's links are loaded before the arrival so their latency
      // overlaps the atomic's; only the sibling's box waits for it
      const int sib = (v & 1) ? E.child_l[p] : E.child_r[p];
      const int up = E.parent_int[p];
      cuda::atomic_ref<unsigned int, cuda::thread_scope_device> arrived(arrivals[p]);
      if (arrived.fetch_add(1u, cuda::memory_order_acq_rel) == 0u) break;  // the sibling is not finished yet
      float4 sl, sh;
      if (sib & kLeafFlag) {
        sl = pts[sib & ~kLeafFlag];
        sh = sl;
      } else {
        sl = __ldcg(&boxes[2 * sib]);
        sh = __ldcg(&boxes[2 * sib + 1]);
      }
      lo = make_float4(fminf(lo.x, sl.x), fminf(lo.y, sl.y), fminf(lo.z, sl.z), 0.f);
      hi = make_float4(fmaxf(hi.x, sh.x), fmaxf(hi.y, sh.y), fmaxf(hi.z, sh.z), 0.f);
      __stcg(&boxes[2 * p], lo);
      __stcg(&boxes[2 * p + 1], hi);
      v = up;
    }
  }
}

// Writes each collapsed-tree node at its pre-order index; the rope field holds
// the Karras entity of the rope until k_translate_ropes maps it.
__global__ void k_compact(Ent E, const uint8_t* __restrict__ flags, const uint32_t* __restrict__ leaves_before,
                          const float4* __restrict__ pts, const float4* __restrict__ boxes,
                          const int* __restrict__ right_of_split, int* __restrict__ ent2pre,
                          float4* __restrict__ nodes) {
  const int total = 2 * (int)E.n - 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const uint8_t f = flags[e];
    if (!(f & 1)) continue;
    int depth = 0, right = 0;
    for (int x = e; x != 0;) {
      const int v = E.link(x);
      ++depth;
      right += v & 1;
      x = v >> 1;
    }
    const int a = E.lo(e), b = E.hi(e);
    const int pre = 2 * (int)leaves_before[a] + depth - right;
    ent2pre[e] = pre;
    float4 lo, hi;
    if (E.is_point(e)) {
      lo = pts[a];
      hi = lo;
    } else {
      lo = boxes[2 * e];
      hi = boxes[2 * e + 1];
    }
    const int ref = (f & 2) ? leaf_ref(a, b - a + 1) : kInternalNode;
    const int rope_ent = b == (int)E.n - 1 ? kRopeEnd : right_of_split[b];
    nodes[2 * pre] = make_float4(lo.x, lo.y, lo.z, __int_as_float(ref));
    nodes[2 * pre + 1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(rope_ent));
  }
}

__global__ void k_translate_ropes(const uint32_t* __restrict__ leaves_total, const int* __restrict__ ent2pre,
                                  float4* __restrict__ nodes) {
  const int m = 2 * (int)(*leaves_total) - 1;  // nodes of the collapsed tree
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int r = __float_as_int(nodes[2 * i + 1].w);
    nodes[2 * i + 1].w = __int_as_float(r == kRopeEnd ? kRopeEnd : ent2pre[r]);
  }
}

// Problem batch: the subtree root of each problem is the collapsed-tree node
// whose points lie in one problem while its parent's span several (or the
// root itself).
__global__ void k_batch_roots(Ent E, const uint8_t* __restrict__ flags, const uint32_t* __restrict__ codes,
                              int code_bits, const int* __restrict__ ent2pre, int* __restrict__ prob_root) {
  const int total = 2 * (int)E.n - 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    if (!(flags[e] & 1) || spans_problems(E, e, codes, code_bits)) continue;
    if (e != 0 && !spans_problems(E, E.parent(e), codes, code_bits)) continue;
    prob_root[problem_of(codes[E.lo(e)], code_bits)] = ent2pre[e];
  }
}

__global__ void k_batch_single_root(const uint32_t* __restrict__ codes, int code_bits, int* __restrict__ prob_root) {
  prob_root[problem_of(codes[0], code_bits)] = 0;
}

// Problem id of every point: one block per problem fills its range.
__global__ void k_batch_ids(const unsigned long long* __restrict__ offsets, uint32_t* __restrict__ pid) {
  const uint32_t p = blockIdx.x;
  const unsigned long long a = offsets[p], b = offsets[p + 1];
  for (unsigned long long i = a + threadIdx.x; i < b; i += blockDim.x) pid[i] = p;
}

// Per-problem boxes: a warp whose points share one problem reduces first and
// issues one set of atomics; mixed warps fall back to per-lane atomics.
__global__ void k_batch_boxes(const float4* __restrict__ pts, const uint32_t* __restrict__ pid, uint32_t n,
                              PointStats* __restrict__ st) {
  const int lane = threadIdx.x & 31;
  for (uint64_t i0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull; i0 < n;
       i0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = i0 + lane;
    const bool valid = i < n;
    const uint32_t p = valid ? pid[i] : 0xFFFFFFFFu;
    const float4 q = valid ? pts[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    float lo[3] = {valid ? q.x : INFINITY, valid ? q.y : INFINITY, valid ? q.z : INFINITY};
    float hi[3] = {valid ? q.x : -INFINITY, valid ? q.y : -INFINITY, valid ? q.z : -INFINITY};
    const uint32_t p0 = __shfl_sync(0xffffffffu, p, 0);
    if (__all_sync(0xffffffffu, p == p0 || !valid)) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
          hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
      }
      if (lane == 0 && p0 != 0xFFFFFFFFu) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          atomicMin(&st[p0].lo[a], float_to_ordered(lo[a]));
          atomicMax(&st[p0].hi[a], float_to_ordered(hi[a]));
        }
      }
    } else if (valid) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        atomicMin(&st[p].lo[a], float_to_ordered(lo[a]));
        atomicMax(&st[p].hi[a], float_to_ordered(hi[a]));
      }
    }
  }
}

__global__ void k_reset_stats_n(PointStats* st, uint32_t m) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      st[i].lo[a] = 0xFFFFFFFFu;
      st[i].hi[a] = 0u;
    }
    st[i].max_abs_bits = 0ull;
    st[i].inexact = 0u;
    st[i].bad = 0u;
    st[i].ids_unsorted = 0u;
    st[i].pad = 0u;
  }
}

// Composite sort keys (problem << code_bits) | Morton code of the point in its
// problem's box, code_bits / dim bits per axis.
__global__ void k_batch_codes(const float4* __restrict__ pts, const uint32_t* __restrict__ pid, uint32_t n, int dim,
                              const PointStats* __restrict__ st, int stats_stride, int code_bits,
                              uint32_t* __restrict__ codes) {
  const int bpa = code_bits / dim;
  const float cells = (float)((1u << bpa) - 1u);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = pid[i];
    const PointStats& box = st[(size_t)p * stats_stride];
    const float4 q = pts[i];
    const float c[3] = {q.x, q.y, q.z};
    uint32_t m[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const unsigned int ol = box.lo[a], oh = box.hi[a];
      const float l = ol == 0xFFFFFFFFu ? 0.f : ordered_to_float(ol);
      const float h = ol == 0xFFFFFFFFu ? 0.f : ordered_to_float(oh);
      const float ext = h - l;
      const float scale = (ext > 0.f && isfinite(ext)) ? cells / ext : 0.f;
      float t = (c[a] - l) * scale;
      t = fminf(fmaxf(t, 0.f), cells);
      m[a] = (uint32_t)t;
    }
    const uint32_t mort = dim == 3 ? (spread10(m[0]) << 2) | (spread10(m[1]) << 1) | spread10(m[2])
                                   : (spread16(m[0]) << 1) | spread16(m[1]);
    codes[i] = (code_bits < 32 ? (p << code_bits) : 0u) | mort;
  }
}

// A one-point scene: a single leaf bucket.
__global__ void k_single_point(const float4* __restrict__ pts, float4* __restrict__ nodes) {
  const float4 p = pts[0];
  nodes[0] = make_float4(p.x, p.y, p.z, __int_as_float(leaf_ref(0, 1)));
  nodes[1] = make_float4(p.x, p.y, p.z, __int_as_float(kRopeEnd));
}

}  // namespace

void reset_stats(PointStats* stats, cudaStream_t s) {
  k_reset_stats<<<1, 32, 0, s>>>(stats);
  RTDL_LAUNCHED(1);
}

void prep_points(const void* points_dev, uint32_t n, int dim, float4* out, PointStats* stats, cudaStream_t s) {
  if (n == 0) return;
  const double* raw = static_cast<const double*>(points_dev);
  if (dim == 3)
    k_prep<3><<<prep_grid(n), kPrepThreads, 0, s>>>(raw, n, out, stats);
  else
    k_prep<2><<<prep_grid(n), kPrepThreads, 0, s>>>(raw, n, out, stats);
  RTDL_LAUNCHED(1);
}

void morton_codes(const float4* pts, uint32_t n, int dim, const PointStats* box_stats, uint32_t* codes, cudaStream_t s) {
  if (n == 0) return;
  k_morton<<<grid_for(n), kThreads, 0, s>>>(pts, n, dim, box_stats, codes);
  RTDL_LAUNCHED(1);
}

int batch_problem_bits(uint32_t problems) {
  int b = 0;
  while (b < 32 && (1ull << b) < (unsigned long long)problems) ++b;
  return b;
}

int batch_code_bits(uint32_t problems, int dim) {
  int bits = 32 - batch_problem_bits(problems);
  if (bits > (dim == 3 ? 30 : 32)) bits = dim == 3 ? 30 : 32;
  return bits - bits % dim;
}

void batch_problem_ids(const unsigned long long* offsets_dev, uint32_t problems, uint32_t n, uint32_t* pid,
                       cudaStream_t s) {
  if (n == 0 || problems == 0) return;
  k_batch_ids<<<problems, 256, 0, s>>>(offsets_dev, pid);
  RTDL_LAUNCHED(1);
}

void batch_boxes(const float4* pts, const uint32_t* pid, uint32_t n, PointStats* prob_stats, uint32_t problems,
                 cudaStream_t s) {
  k_reset_stats_n<<<div_up(problems, 256), 256, 0, s>>>(prob_stats, problems);
  RTDL_LAUNCHED(1);
  if (n == 0) return;
  k_batch_boxes<<<grid_for(n), kThreads, 0, s>>>(pts, pid, n, prob_stats);
  RTDL_LAUNCHED(1);
}

void batch_codes(const float4* pts, const uint32_t* pid, uint32_t n, int dim, const PointStats* prob_stats,
                 int stats_stride, int code_bits, uint32_t* codes, cudaStream_t s) {
  if (n == 0) return;
  k_batch_codes<<<grid_for(n), kThreads, 0, s>>>(pts, pid, n, dim, prob_stats, stats_stride, code_bits, codes);
  RTDL_LAUNCHED(1);
}

namespace {

Scene* build_scene_impl(const void* points_dev, uint32_t n, int dim, cudaStream_t s, int leaf_size,
                        const unsigned long long* offsets, uint32_t problems) {
  if (dim != 2 && dim != 3) throw std::runtime_error("dimension must be 2 or 3");
  if (n > (uint32_t)kMaxScenePoints)
    throw std::runtime_error("search_count exceeds the scene limit of 67,108,864 points");
  if (leaf_size < 1) leaf_size = 1;
  if (leaf_size > 32) leaf_size = 32;
  const bool batch = offsets != nullptr;
  Scene* sc = new Scene();
  sc->dim = dim;
  sc->n = n;
  sc->stream = s;
  sc->leaf_size = leaf_size;
  RTDL_CUDA_CHECK(cudaGetDevice(&sc->device));
  sc->stats = static_cast<PointStats*>(dev_alloc(sizeof(PointStats), s));
  reset_stats(sc->stats, s);
  if (batch) {
    sc->problems = problems;
    sc->code_bits = batch_code_bits(problems, dim);
    sc->prob_offsets.assign(offsets, offsets + problems + 1);
    sc->prob_stats = static_cast<PointStats*>(dev_alloc(sizeof(PointStats) * problems, s));
    sc->prob_root = static_cast<int*>(dev_alloc(sizeof(int) * problems, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(sc->prob_root, 0xFF, sizeof(int) * problems, s));  // kRopeEnd: no points
  }
  if (n == 0) {
    if (batch) batch_boxes(nullptr, nullptr, 0, sc->prob_stats, problems, s);
    return sc;
  }
  const double* raw = static_cast<const double*>(points_dev);
  float4* pts_in = static_cast<float4*>(dev_alloc(sizeof(float4) * n, s));
  prep_points(points_dev, n, dim, pts_in, sc->stats, s);
  uint32_t* codes = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n, s));
  if (batch) {
    unsigned long long* d_off =
        static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * (problems + 1), s));
    RTDL_CUDA_CHECK(cudaMemcpyAsync(d_off, sc->prob_offsets.data(), sizeof(unsigned long long) * (problems + 1),
                                    cudaMemcpyHostToDevice, s));
    uint32_t* pid = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n, s));
    batch_problem_ids(d_off, problems, n, pid, s);
    batch_boxes(pts_in, pid, n, sc->prob_stats, problems, s);
    batch_codes(pts_in, pid, n, dim, sc->prob_stats, 1, sc->code_bits, codes, s);
    dev_free(pid, s);
    dev_free(d_off, s);
  } else {
    morton_codes(pts_in, n, dim, sc->stats, codes, s);
  }
  sc->perm = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n, s));
  iota_u32(sc->perm, n, s);
  radix_sort_pairs(codes, sc->perm, n, 0, batch ? 32 : (dim == 3 ? 30 : 32), nullptr, &sc->stats->bad, s);
  sc->pts = static_cast<float4*>(dev_alloc(sizeof(float4) * n, s));
  sc->pts64 = static_cast<double*>(dev_alloc(sizeof(double) * 3 * (size_t)n, s));
  if (dim == 3)
    k_gather<3><<<grid_for(n), kThreads, 0, s>>>(pts_in, raw, sc->perm, n, sc->pts, sc->pts64, sc->stats);
  else
    k_gather<2><<<grid_for(n), kThreads, 0, s>>>(pts_in, raw, sc->perm, n, sc->pts, sc->pts64, sc->stats);
  RTDL_LAUNCHED(1);
  dev_free(pts_in, s);
  if (n >= 2) {
    const uint32_t ni = n - 1;
    int* child_l = static_cast<int*>(dev_alloc(sizeof(int) * ni, s));
    int* child_r = static_cast<int*>(dev_alloc(sizeof(int) * ni, s));
    int* first = static_cast<int*>(dev_alloc(sizeof(int) * ni, s));
    int* last = static_cast<int*>(dev_alloc(sizeof(int) * ni, s));
    int* parent_int = static_cast<int*>(dev_alloc(sizeof(int) * ni, s));
    int* parent_leaf = static_cast<int*>(dev_alloc(sizeof(int) * n, s));
    int* right_of_split = static_cast<int*>(dev_alloc(sizeof(int) * ni, s));
    unsigned int* arrivals = static_cast<unsigned int*>(dev_alloc(sizeof(unsigned int) * ni, s));
    float4* boxes = static_cast<float4*>(dev_alloc(sizeof(float4) * 2 * (size_t)ni, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(arrivals, 0, sizeof(unsigned int) * ni, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(parent_int, 0xFF, sizeof(int) * ni, s));  // root keeps -1
    k_karras<<<grid_for(ni), kThreads, 0, s>>>(codes, n, child_l, child_r, first, last, parent_int, parent_leaf,
                                              right_of_split);
    RTDL_LAUNCHED(1);
    Ent E{child_l, child_r, first, last, parent_int, parent_leaf, n};
    const uint64_t ents = 2ull * n - 1;
    uint8_t* flags = static_cast<uint8_t*>(dev_alloc(ents, s));
    uint32_t* leaf_start = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n, s));
    int* bucket_at = static_cast<int*>(dev_alloc(sizeof(int) * n, s));
    int* buckets = static_cast<int*>(dev_alloc(sizeof(int) * n, s));
    uint64_t* leaves_before = static_cast<uint64_t*>(dev_alloc(sizeof(uint64_t) * (n + 1), s));
    uint32_t* leaves_before32 = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * (n + 1), s));
    int* ent2pre = static_cast<int*>(dev_alloc(sizeof(int) * ents, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(leaf_start, 0, sizeof(uint32_t) * n, s));
    RTDL_CUDA_CHECK(cudaMemsetAsync(ent2pre, 0xFF, sizeof(int) * ents, s));  // kRopeEnd for entities off the tree
    k_mark_collapsed<<<grid_for(ents), kThreads, 0, s>>>(E, leaf_size, batch ? codes : nullptr, sc->code_bits,
                                                         flags, leaf_start, bucket_at);
    RTDL_LAUNCHED(1);
    scan_counts_u64(leaf_start, nullptr, nullptr, n, reinterpret_cast<unsigned long long*>(leaves_before), s);
    k_bucket_list<<<grid_for(n + 1), kThreads, 0, s>>>(leaves_before, leaf_start, bucket_at, n, leaves_before32,
                                                       buckets);
    k_refit_buckets<<<grid_for(div_up(n, 4)), kThreads, 0, s>>>(E, buckets, leaves_before32 + n, sc->pts, arrivals,
                                                               boxes);
    sc->nodes = static_cast<float4*>(dev_alloc(sizeof(float4) * 2 * ents, s));
    k_compact<<<grid_for(ents), kThreads, 0, s>>>(E, flags, leaves_before32, sc->pts, boxes, right_of_split, ent2pre,
                                                  sc->nodes);
    k_translate_ropes<<<grid_for(ents), kThreads, 0, s>>>(leaves_before32 + n, ent2pre, sc->nodes);
    RTDL_LAUNCHED(4);
    if (batch) {
      k_batch_roots<<<grid_for(ents), kThreads, 0, s>>>(E, flags, codes, sc->code_bits, ent2pre, sc->prob_root);
      RTDL_LAUNCHED(1);
    }
    dev_free(child_l, s);
    dev_free(child_r, s);
    dev_free(first, s);
    dev_free(last, s);
    dev_free(parent_int, s);
    dev_free(parent_leaf, s);
    dev_free(arrivals, s);
    dev_free(boxes, s);
    dev_free(right_of_split, s);
    dev_free(flags, s);
    dev_free(leaf_start, s);
    dev_free(bucket_at, s);
    dev_free(buckets, s);
    dev_free(leaves_before, s);
    dev_free(leaves_before32, s);
    dev_free(ent2pre, s);
  } else if (n == 1) {
    sc->nodes = static_cast<float4*>(dev_alloc(sizeof(float4) * 2, s));
    k_single_point<<<1, 1, 0, s>>>(sc->pts, sc->nodes);
    RTDL_LAUNCHED(1);
    if (batch) {
      k_batch_single_root<<<1, 1, 0, s>>>(codes, sc->code_bits, sc->prob_root);
      RTDL_LAUNCHED(1);
    }
  }
  sc->codes = codes;  // kept: nearest searches seed from a window around the query's code
  return sc;
}

}  // namespace

Scene* build_scene(const void* points_dev, uint32_t n, int dim, cudaStream_t s, int leaf_size) {
  return build_scene_impl(points_dev, n, dim, s, leaf_size, nullptr, 0);
}

Scene* build_scene_batch(const void* points_dev, const unsigned long long* offsets, uint32_t problems, int dim,
                         cudaStream_t s, int leaf_size) {
  if (problems == 0) throw std::runtime_error("a problem batch needs at least one problem");
  for (uint32_t p = 0; p < problems; ++p)
    if (offsets[p + 1] < offsets[p]) throw std::runtime_error("problem offsets must be non-decreasing");
  if (offsets[0] != 0) throw std::runtime_error("problem offsets must start at 0");
  if (offsets[problems] > (unsigned long long)kMaxScenePoints)
    throw std::runtime_error("a problem batch holds at most 67,108,864 search points");
  if (batch_problem_bits(problems) > 26)
    throw std::runtime_error("a problem batch holds at most 67,108,864 problems");
  return build_scene_impl(points_dev, (uint32_t)offsets[problems], dim, s, leaf_size, offsets, problems);
}

void destroy_scene(Scene* sc) {
  if (!sc) return;
  cudaStream_t s = sc->stream;
  dev_free(sc->pts, s);
  dev_free(sc->perm, s);
  dev_free(sc->pts64, s);
  dev_free(sc->nodes, s);
  dev_free(sc->codes, s);
  dev_free(sc->stats, s);
  dev_free(sc->prob_stats, s);
  dev_free(sc->prob_root, s);
  if (sc->own_stream && s) {
    sync_quietly(s);
    note_cleanup_error(cudaStreamDestroy(s), "cudaStreamDestroy");
  }
  delete sc;
}

}  // namespace rtdl_b200
