// sort_scan.cu -- device prefix scans and a stable LSD radix sort, written for
// this library (no CUB): the LBVH build sorts Morton codes with it, the query
// path sorts queries into Morton order and into query-id order, and row
// offsets come from the scan.
//
// Scan: reduce-then-scan over 2,048-element tiles (256 threads x 8 items), a
// single-block pass over the tile sums, then a downsweep.  Deterministic and
// free of inter-block waits.
// Radix sort: 8-bit digits.  One kernel counts the digits of every pass in a
// single read of the keys; then one scatter kernel per pass.  A scatter block
// takes the next tile index from a counter, counts its tile's digits, and
// finds each digit's offset among the earlier tiles by decoupled look-back
// (Merrill and Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", 2016): per (tile, digit) a status word holds either the tile's
// own count or the inclusive count over tiles 0..tile, and a block walks back
// over the earlier tiles' words until it meets an inclusive one.  Tile indices
// are handed out in the order blocks start, so every tile a block waits on
// belongs to a block that is already running; each wait is still bounded and
// reports through an error word when it runs out.  Inside a tile each warp
// owns a contiguous run: the warp counts its digits (a key's peers from eight
// ballots on the digit's bits, one shared-memory add per digit group; 1% faster
// at 4M keys than __match_any_sync), a block-wide scan over (digit, warp)
// turns the counts into bases, and the warp then places its keys in order, so
// the sort stays stable.
#include <cuda/atomic>

#include "internal.cuh"

namespace rtdl_b200 {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

__device__ __forceinline__ uint32_t load_count(const uint32_t* counts, const uint32_t* order,
                                               const unsigned int* identity_flag, uint32_t i) {
  if (order == nullptr || (identity_flag != nullptr && *identity_flag)) return counts[i];
  return counts[order[i]];
}

// Block-wide exclusive scan of one value per thread (blockDim == kScanThreads).
template <typename T>
__device__ T block_exclusive_scan(T v, T* total) {
  __shared__ T warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < kScanThreads / 32 ? warp_sums[lane] : T(0);
    T wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = wi - w;
    if (lane == kScanThreads / 32 - 1) warp_sums[0] = warp_sums[0];  // keep ordering explicit
    if (lane == kScanThreads / 32 - 1) *total = wi;
  }
  __syncthreads();
  T r = warp_sums[warp] + inc - v;
  __syncthreads();
  return r;
}

template <typename Out>
__global__ void k_scan_reduce(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag,
                              uint32_t n, Out* block_sums) {
  __shared__ Out total;
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  Out s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    uint64_t idx = base + i;
    if (idx < n) s += (Out)load_count(counts, order, identity_flag, (uint32_t)idx);
  }
  block_exclusive_scan<Out>(s, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// One block of 1,024 threads scans the tile sums in place (exclusive) and
// writes the grand total to *grand_total.
template <typename Out>
__global__ void k_scan_tile_sums(Out* sums, uint32_t num, Out* grand_total) {
  __shared__ Out warp_sums[32];
  __shared__ Out carry_s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (uint32_t chunk = 0; chunk < num; chunk += blockDim.x) {
    uint32_t i = chunk + threadIdx.x;
    Out v = i < num ? sums[i] : Out(0);
    Out inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      Out y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      Out w = warp_sums[lane];
      Out wi = w;
      for (int o = 1; o < 32; o <<= 1) {
        Out y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += y;
      }
      warp_sums[lane] = wi - w;
    }
    __syncthreads();
    Out carry = carry_s;
    Out excl = carry + warp_sums[warp] + inc - v;
    if (i < num) sums[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry_s = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *grand_total = carry_s;
}

template <typename Out>
__global__ void k_scan_down(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag,
                            uint32_t n, const Out* block_prefix, Out* out) {
  __shared__ Out total;
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  Out s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    uint64_t idx = base + i;
    v[i] = idx < n ? load_count(counts, order, identity_flag, (uint32_t)idx) : 0u;
    s += (Out)v[i];
  }
  Out run = block_exclusive_scan<Out>(s, &total) + block_prefix[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    uint64_t idx = base + i;
    if (idx < n) out[idx] = run;
    run += (Out)v[i];
  }
}

template <typename Out>
void scan_impl(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag, uint32_t n,
               Out* out, Out* workspace, cudaStream_t s) {
  uint32_t tiles = div_up(n, kScanTile);
  if (tiles == 0) tiles = 1;
  Out* sums = workspace ? workspace : static_cast<Out*>(dev_alloc(sizeof(Out) * tiles, s));
  k_scan_reduce<Out><<<tiles, kScanThreads, 0, s>>>(counts, order, identity_flag, n, sums);
  k_scan_tile_sums<Out><<<1, 1024, 0, s>>>(sums, tiles, out + n);
  k_scan_down<Out><<<tiles, kScanThreads, 0, s>>>(counts, order, identity_flag, n, sums, out);
  RTDL_LAUNCHED(3);
  if (!workspace) dev_free(sums, s);
}

constexpr uint32_t kLookLocal = 1u << 30;       // status word: the tile's own count of the digit
constexpr uint32_t kLookInclusive = 2u << 30;   // status word: the count over tiles 0..this one
constexpr uint32_t kLookValue = (1u << 30) - 1u;
constexpr int kLookSpinLimit = 1 << 22;         // polls of one status word before the wait gives up
constexpr int kMaxPasses = 4;

// Lanes of the warp holding the same 8-bit digit (valid lanes only), from
// eight ballots on the digit's bits.
__device__ __forceinline__ unsigned int digit_peers(uint32_t d, bool valid) {
  unsigned int peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool bit = (d >> b) & 1u;
    const unsigned int bb = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? bb : ~bb;
  }
  return peers;
}

// Digit counts of every pass (counts[pass * 256 + digit]) in one read of the
// keys; each warp keeps its own shared histograms.
__global__ void __launch_bounds__(kSortThreads) k_radix_hist_all(const uint32_t* __restrict__ keys, uint32_t n,
                                                                int begin_bit, int passes, uint32_t* counts,
                                                                const unsigned int* skip) {
  if (skip != nullptr && *skip) return;
  __shared__ unsigned int h[kSortWarps][kMaxPasses][256];
  const int t = threadIdx.x, warp = t >> 5;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w)
#pragma unroll
    for (int p = 0; p < kMaxPasses; ++p) h[w][p][t] = 0;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + t; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&h[warp][p][(k >> (begin_bit + 8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int p = 0; p < passes; ++p) {
    unsigned int c = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) c += h[w][p][t];
    if (c) atomicAdd(&counts[p * 256 + t], c);
  }
}

__global__ void __launch_bounds__(kSortThreads)
    k_radix_onesweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                     uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n, int shift,
                     const uint32_t* __restrict__ digit_counts, uint32_t* status, unsigned int* tile_counter,
                     unsigned int* wait_error, const unsigned int* skip) {
  if (skip != nullptr && *skip) return;
  __shared__ unsigned int wcnt[kSortWarps][256];  // a warp's digit counts, then its tile-local digit bases
  __shared__ unsigned int dbase[256];             // tile-local start of each digit
  __shared__ unsigned int gbase[256];             // global start of each digit for this tile
  __shared__ unsigned int total, tile_s;
  __shared__ uint32_t skeys[kSortTile], svals[kSortTile];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const unsigned int lt_mask = (1u << lane) - 1u;
  if (t == 0) tile_s = atomicAdd(tile_counter, 1u);
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) wcnt[w][t] = 0;
  __syncthreads();
  const uint32_t tile = tile_s;
  // the warp's run of the tile: kSortItems rounds of 32 consecutive keys
  const uint64_t tile0 = (uint64_t)tile * kSortTile;
  const uint64_t base = tile0 + (uint64_t)warp * (kSortItems * 32);
  uint32_t key[kSortItems];
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const uint64_t idx = base + (uint64_t)i * 32 + lane;
    const bool valid = idx < n;
    key[i] = valid ? keys_in[idx] : 0u;
    const uint32_t d = (key[i] >> shift) & 255u;
    const unsigned int peers = digit_peers(d, valid);
    if (valid && (peers & lt_mask) == 0) wcnt[warp][d] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // thread t owns digit t: offsets of the warps within the digit and the
  // tile's count of the digit
  unsigned int r = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const unsigned int c = wcnt[w][t];
    wcnt[w][t] = r;
    r += c;
  }
  // publish the count, then look back over the earlier tiles for the digit's
  // offset among them
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> mine(status[(uint64_t)tile * 256 + t]);
  uint32_t before = 0;
  if (tile == 0) {
    mine.store(kLookInclusive | r, cuda::memory_order_relaxed);
  } else {
    mine.store(kLookLocal | r, cuda::memory_order_relaxed);
    int64_t j = (int64_t)tile - 1;
    int spins = 0;
    while (j >= 0) {
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> w(status[(uint64_t)j * 256 + t]);
      const uint32_t v = w.load(cuda::memory_order_relaxed);
      if (v & kLookInclusive) {
        before += v & kLookValue;
        break;
      }
      if (v & kLookLocal) {
        before += v & kLookValue;
        --j;
        continue;
      }
      if (++spins > kLookSpinLimit) {
        atomicOr(wait_error, kBadSortWait);
        break;
      }
      __nanosleep(64);
    }
    mine.store(kLookInclusive | ((before + r) & kLookValue), cuda::memory_order_relaxed);
  }
  const unsigned int db = block_exclusive_scan<unsigned int>(r, &total);
  const unsigned int dstart = block_exclusive_scan<unsigned int>(digit_counts[t], &total);
  dbase[t] = db;
  gbase[t] = dstart + before;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) wcnt[w][t] += db;
  __syncthreads();
  // place the keys in the tile's digit order in shared memory (stable)
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const uint64_t idx = base + (uint64_t)i * 32 + lane;
    const bool valid = idx < n;
    const uint32_t d = (key[i] >> shift) & 255u;
    const unsigned int peers = digit_peers(d, valid);
    if (valid) {
      const unsigned int pos = wcnt[warp][d] + __popc(peers & lt_mask);
      skeys[pos] = key[i];
      svals[pos] = vals_in[idx];
    }
    __syncwarp();
    if (valid && (peers & lt_mask) == 0) wcnt[warp][d] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // write out: consecutive threads take consecutive keys of a digit's run,
  // so the global stores are contiguous; a position beyond n (possible only
  // after a wait ran out) is not written
  const unsigned int tile_n = (unsigned int)(n - tile0 < (uint64_t)kSortTile ? n - tile0 : (uint64_t)kSortTile);
  for (unsigned int j = t; j < tile_n; j += kSortThreads) {
    const uint32_t k = skeys[j];
    const uint32_t d = (k >> shift) & 255u;
    const unsigned int pos = gbase[d] + (j - dbase[d]);
    if (pos < n) {
      keys_out[pos] = k;
      vals_out[pos] = svals[j];
    }
  }
}

__global__ void k_iota(uint32_t* out, uint32_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

}  // namespace

void scan_counts_u64(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag, uint32_t n,
                     unsigned long long* out, cudaStream_t s) {
  scan_impl<unsigned long long>(counts, order, identity_flag, n, out, nullptr, s);
}

size_t scan_workspace_bytes(uint32_t n) {
  const uint32_t tiles = div_up(n, kScanTile);
  return sizeof(unsigned long long) * (tiles ? tiles : 1);
}

void scan_counts_u64_ws(const uint32_t* counts, const uint32_t* order, const unsigned int* identity_flag, uint32_t n,
                        unsigned long long* out, void* workspace, cudaStream_t s) {
  scan_impl<unsigned long long>(counts, order, identity_flag, n, out, static_cast<unsigned long long*>(workspace), s);
}

void iota_u32(uint32_t* out, uint32_t n, cudaStream_t s) {
  if (n == 0) return;
  unsigned int blocks = div_up(n, 256);
  if (blocks > 8 * kSmCount * 4) blocks = 8 * kSmCount * 4;
  k_iota<<<blocks, 256, 0, s>>>(out, n);
  RTDL_LAUNCHED(1);
}

void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, int begin_bit, int end_bit,
                      const unsigned int* skip_flag, unsigned int* wait_error, cudaStream_t s) {
  if (n <= 1 || end_bit <= begin_bit) return;
  if (n > kLookValue) throw std::runtime_error("radix sort input too large");
  if (begin_bit < 0 || end_bit > 32) throw std::runtime_error("radix sort bit range must lie in [0, 32)");
  int passes = (end_bit - begin_bit + 7) / 8;
  if (passes & 1) ++passes;  // even pass count leaves the result in the caller's buffers
  int real = 0;              // passes that sort (the rest only copy)
  while (real < passes && begin_bit + 8 * real < 32) ++real;
  const uint32_t tiles = div_up(n, kSortTile);
  uint32_t* keys_alt = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n, s));
  uint32_t* vals_alt = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * n, s));
  // per sorting pass: 256 digit counts, a tile counter and tiles x 256 status words
  const size_t per_pass = 256 + 1 + (size_t)tiles * 256;
  const size_t work_words = per_pass * (size_t)real;
  uint32_t* work = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * work_words, s));
  RTDL_CUDA_CHECK(cudaMemsetAsync(work, 0, sizeof(uint32_t) * work_words, s));
  uint32_t* counts = work;                                    // real x 256
  unsigned int* tile_counters = work + 256 * (size_t)real;    // real
  uint32_t* status = work + 257 * (size_t)real;               // real x tiles x 256
  unsigned int hist_blocks = div_up(n, kSortThreads * 8);
  if (hist_blocks > (unsigned int)kSmCount * 2) hist_blocks = kSmCount * 2;
  k_radix_hist_all<<<hist_blocks, kSortThreads, 0, s>>>(keys, n, begin_bit, real, counts, skip_flag);
  RTDL_LAUNCHED(1);
  uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
  for (int p = 0; p < passes; ++p) {
    const int shift = begin_bit + 8 * p;
    if (p < real) {
      k_radix_onesweep<<<tiles, kSortThreads, 0, s>>>(ki, vi, ko, vo, n, shift, counts + 256 * p, status +
                                                      (size_t)p * tiles * 256, tile_counters + p, wait_error,
                                                      skip_flag);
      RTDL_LAUNCHED(1);
    } else {
      // A padding pass beyond the key width: a plain copy keeps the ping-pong even.
      RTDL_CUDA_CHECK(cudaMemcpyAsync(ko, ki, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
      RTDL_CUDA_CHECK(cudaMemcpyAsync(vo, vi, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    RTDL_CUDA_CHECK(cudaGetLastError());
    uint32_t* tk = ki; ki = ko; ko = tk;
    uint32_t* tv = vi; vi = vo; vo = tv;
  }
  dev_free(keys_alt, s);
  dev_free(vals_alt, s);
  dev_free(work, s);
}

}  // namespace rtdl_b200
