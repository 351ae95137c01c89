// api.cu -- the C ABI of librtdl_b200.so (declared in include/rtdl_b200.h).
//
// Every entry point follows the reference's native-call convention
// (rubaolee/rtdl src/native/optix/rtdl_optix_core.cpp:58-66): exceptions are
// caught at the boundary and turned into status 1 plus a message.
// Device memory comes from the stream-ordered allocator with the release
// threshold raised, so repeated calls reuse pooled memory without OS calls.
// Rows handed to the caller live in pinned host buffers from a small pool, so
// the device-to-host copy runs at full PCIe rate; rtdl_b200_free_rows returns
// them to the pool.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "internal.cuh"

namespace rtdl_b200 {

namespace {
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long launches_counted() { return g_launches.load(std::memory_order_relaxed); }

void check_launch(int n, const char* file, int line) {
  count_launches(n);
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return;
  const char* base = std::strrchr(file, '/');
  throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " at kernel launch (" +
                           (base ? base + 1 : file) + ":" + std::to_string(line) + ")");
}

namespace {
thread_local std::string g_cleanup_error;

std::mutex& tuning_mutex() {
  static std::mutex m;
  return m;
}
Tuning& tuning_global() {
  static Tuning t;
  return t;
}
Tuning tuning_copy() {
  std::lock_guard<std::mutex> g(tuning_mutex());
  return tuning_global();
}
thread_local Tuning g_tuning_snapshot;
thread_local int g_tuning_depth = 0;
}  // namespace

void note_cleanup_error(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();  // consumed here: a later launch check must not report it
  if (g_cleanup_error.empty())
    g_cleanup_error = std::string("CUDA error: ") + cudaGetErrorString(e) + " at " + what;
}

TuningScope::TuningScope() : outer(g_tuning_depth == 0) {
  if (outer) g_tuning_snapshot = tuning_copy();
  ++g_tuning_depth;
}
TuningScope::~TuningScope() { --g_tuning_depth; }

const Tuning& tuning() {
  if (g_tuning_depth == 0) g_tuning_snapshot = tuning_copy();  // outside an entry point: the current setting
  return g_tuning_snapshot;
}

void set_tuning(const Tuning& t) {
  std::lock_guard<std::mutex> g(tuning_mutex());
  tuning_global() = t;
}

void ensure_pool_configured(int device) {
  static std::mutex m;
  static std::vector<bool> done;
  std::lock_guard<std::mutex> g(m);
  if ((int)done.size() <= device) done.resize(device + 1, false);
  if (done[device]) return;
  cudaMemPool_t pool;
  RTDL_CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = UINT64_MAX;
  RTDL_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  done[device] = true;
}

void* dev_alloc(size_t bytes, cudaStream_t s) {
  if (bytes == 0) bytes = 16;
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error("device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  return p;
}

void dev_free(void* p, cudaStream_t s) {
  if (p) note_cleanup_error(cudaFreeAsync(p, s), "cudaFreeAsync");
}


namespace {

thread_local std::vector<std::pair<const char*, double>> g_last_timings;

}  // namespace

PhaseTimer::PhaseTimer(cudaStream_t s) : stream(s) {}
PhaseTimer::~PhaseTimer() {
  for (auto& m : marks) note_cleanup_error(cudaEventDestroy(m.second), "cudaEventDestroy");
}
void PhaseTimer::mark(const char* name) {
  cudaEvent_t e;
  RTDL_CUDA_CHECK(cudaEventCreate(&e));
  RTDL_CUDA_CHECK(cudaEventRecord(e, stream));
  marks.emplace_back(name, e);
}
void PhaseTimer::publish() {
  g_last_timings.clear();
  double total = 0.0;
  for (size_t i = 1; i < marks.size(); ++i) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, marks[i - 1].second, marks[i].second) != cudaSuccess) {
      cudaGetLastError();
      ms = 0.f;
    }
    g_last_timings.emplace_back(marks[i].first, (double)ms);
    total += ms;
  }
  g_last_timings.emplace_back("total", total);
}

namespace {

// Pinned host buffers for returned rows.
class PinnedPool {
 public:
  void* get(size_t bytes) {
    if (bytes == 0) bytes = 16;
    {
      std::lock_guard<std::mutex> g(m_);
      auto it = free_.lower_bound(bytes);
      if (it != free_.end() && it->first <= 2 * bytes + (4u << 20)) {
        void* p = it->second;
        cached_ -= it->first;
        live_[p] = it->first;
        free_.erase(it);
        return p;
      }
    }
    const size_t rounded = (bytes + (2u << 20) - 1) & ~((size_t)(2u << 20) - 1);
    void* p = nullptr;
    if (cudaMallocHost(&p, rounded) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    std::lock_guard<std::mutex> g(m_);
    live_[p] = rounded;
    return p;
  }
  bool put(void* p) {
    std::lock_guard<std::mutex> g(m_);
    auto it = live_.find(p);
    if (it == live_.end()) return false;
    const size_t sz = it->second;
    live_.erase(it);
    if (cached_ + sz > limit()) {
      note_cleanup_error(cudaFreeHost(p), "cudaFreeHost");
    } else {
      free_.emplace(sz, p);
      cached_ += sz;
    }
    return true;
  }

 private:
  static size_t limit() {
    static size_t lim = [] {
      const char* env = std::getenv("RTDL_B200_PINNED_POOL_MB");
      return (size_t)(env ? std::atoll(env) : 8192) << 20;
    }();
    return lim;
  }
  std::mutex m_;
  std::multimap<size_t, void*> free_;
  std::unordered_map<void*, size_t> live_;
  size_t cached_ = 0;
};

PinnedPool& pinned_pool() {
  static PinnedPool* p = new PinnedPool();  // never destroyed: outlives static teardown order
  return *p;
}

cudaStream_t library_stream() {
  static std::mutex m;
  static std::map<int, cudaStream_t> streams;
  int dev = 0;
  RTDL_CUDA_CHECK(cudaGetDevice(&dev));
  ensure_pool_configured(dev);
  std::lock_guard<std::mutex> g(m);
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  RTDL_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[dev] = s;
  return s;
}

void set_error(const char* msg, char* error_out, size_t error_size) {
  if (!error_out || error_size == 0) return;
  std::strncpy(error_out, msg, error_size - 1);
  error_out[error_size - 1] = '\0';
}

// Every entry point runs through here: the thread's last runtime error is
// cleared first (an error left by earlier, unrelated runtime calls on this
// thread is not this call's), the call runs with one tuning snapshot, and a
// cleanup error that nothing else reported fails the call.
template <typename Fn>
int guarded(Fn&& fn, char* error_out, size_t error_size) {
  TuningScope scope;
  try {
    if (error_out && error_size) error_out[0] = '\0';
    if (scope.outer) {
      cudaGetLastError();
      g_cleanup_error.clear();
    }
    fn();
    if (scope.outer && !g_cleanup_error.empty()) {
      set_error(g_cleanup_error.c_str(), error_out, error_size);
      g_cleanup_error.clear();
      return 1;
    }
    return 0;
  } catch (const std::exception& ex) {
    set_error(ex.what(), error_out, error_size);
    if (scope.outer) g_cleanup_error.clear();
    return 1;
  } catch (...) {
    set_error("unknown native error", error_out, error_size);
    if (scope.outer) g_cleanup_error.clear();
    return 1;
  }
}


size_t record_size(int dim) { return dim == 3 ? sizeof(RtdlPoint3D) : sizeof(RtdlPoint); }

void* upload(const void* host, size_t bytes, cudaStream_t s) {
  void* d = dev_alloc(bytes, s);
  RTDL_CUDA_CHECK(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, s));
  return d;
}

// Downloads `bytes` of device rows into a caller-owned host buffer.
void* download_rows(const void* d_rows, size_t bytes, cudaStream_t s) {
  void* host = pinned_pool().get(bytes);
  bool pinned = host != nullptr;
  if (!pinned) {
    host = std::malloc(bytes ? bytes : 1);
    if (!host) throw std::runtime_error("host allocation of rows failed");
  }
  if (bytes) {
    cudaError_t e = cudaMemcpyAsync(host, d_rows, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      if (pinned) pinned_pool().put(host);
      else std::free(host);
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " while downloading rows");
    }
  }
  return host;
}

void validate_common(double radius, size_t limit, size_t nq, size_t ns, bool has_radius, const char* what,
                     const char* limit_name) {
  if (has_radius && !(radius >= 0.0))
    throw std::runtime_error(std::string(what) + " radius must be non-negative");
  if (limit == 0) throw std::runtime_error(std::string(what) + " " + limit_name + " must be positive");
  if (nq > (size_t)UINT32_MAX) throw std::runtime_error(std::string(what) + " query_count exceeds uint32 limit");
  if (ns > (size_t)UINT32_MAX) throw std::runtime_error(std::string(what) + " search_count exceeds uint32 limit");
  if (limit > (size_t)UINT32_MAX)
    throw std::runtime_error(std::string(what) + " " + limit_name + " exceeds uint32 limit");
}

// Host buffer for rows copied range by range: pinned from the pool, else malloc'd.
void* rows_host_buffer(size_t bytes, bool* pinned) {
  void* host = pinned_pool().get(bytes);
  *pinned = host != nullptr;
  if (!host) {
    host = std::malloc(bytes ? bytes : 1);
    if (!host) throw std::runtime_error("host allocation of rows failed");
  }
  return host;
}

// Query sets of two kRangeQueries or more are answered in ranges of their
// input order (run_build_and_query_chunked, at most kMaxQueryRanges ranges of
// at least kRangeQueries queries), so the copy of the rows to the host, which
// bounds the call, starts after the first range's query.  Each range costs
// a query's fixed overhead (about 0.5 ms): at 1,048,576 clustered queries
// (30 M rows) a call took 11.5 ms in one piece, 10.6 ms in 4 ranges,
// 12.6 ms in 8 and 19.7 ms in 16.
constexpr size_t kRangeQueries = 1u << 17;
constexpr int kMaxQueryRanges = 4;

// The ranged form of run_rows_call: one host buffer with room for every
// query's limit rows (pinned, from the pool) takes each range's rows.
void run_rows_call_ranged(const void* q, size_t nq, const void* sp, size_t ns, int dim, int predicate, double radius,
                          size_t limit, int ranges, void** rows_out, size_t* row_count_out) {
  cudaStream_t s = library_stream(), copy = aux_stream(0);
  PhaseTimer timer(s);
  timer.mark("begin");
  const size_t rec = record_size(dim);
  const size_t row_size = predicate == kFrn ? sizeof(RtdlFixedRadiusNeighborRow) : sizeof(RtdlKnnNeighborRow);
  void* d_search = upload(sp, rec * ns, s);
  timer.mark("upload");
  Scene* sc = nullptr;
  bool pinned = false;
  void* host = nullptr;
  try {
    host = rows_host_buffer(row_size * nq * limit, &pinned);
    BuildQueryInputs in{d_search, (uint32_t)ns, nullptr, q, (uint32_t)nq, dim};
    QueryResult r = run_build_and_query_chunked(in, predicate, radius, (uint32_t)limit, s, copy, &timer, &sc, host,
                                                (unsigned long long)nq * limit, ranges);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));  // s has waited for the copies
    timer.mark("download");
    timer.publish();
    *rows_out = host;
    *row_count_out = (size_t)r.rows;
  } catch (...) {
    sync_quietly(copy);
    if (host && !(pinned && pinned_pool().put(host))) std::free(host);
    destroy_scene(sc);
    dev_free(d_search, s);
    sync_quietly(s);
    throw;
  }
  destroy_scene(sc);
  dev_free(d_search, s);
}

// Plain per-call launch: upload, build, query, download.  Fixed-radius rows
// are copied to the host range by range while later ranges are still being
// emitted (the copy stream is this thread's second stream, idle by then).
void run_rows_call(const void* q, size_t nq, const void* sp, size_t ns, int dim, int predicate, double radius,
                   size_t limit, void** rows_out, size_t* row_count_out) {
  const int ranges = (int)std::min<size_t>(kMaxQueryRanges, nq / kRangeQueries);
  if (predicate != kKnn && limit <= (size_t)kMaxList && ranges >= 2)
    return run_rows_call_ranged(q, nq, sp, ns, dim, predicate, radius, limit, ranges, rows_out, row_count_out);
  cudaStream_t s = library_stream();
  PhaseTimer timer(s);
  timer.mark("begin");
  const size_t rec = record_size(dim);
  void* d_search = upload(sp, rec * ns, s);
  timer.mark("upload");
  Scene* sc = nullptr;
  void* d_query = nullptr;
  void* d_rows = nullptr;
  RowDownload dl;
  dl.alloc = rows_host_buffer;
  dl.copy = aux_stream();
  auto release_host = [&]() {
    if (dl.host && !(dl.pinned && pinned_pool().put(dl.host))) std::free(dl.host);
    dl.host = nullptr;
  };
  try {
    BuildQueryInputs in{d_search, (uint32_t)ns, nullptr, q, (uint32_t)nq, dim};
    QueryResult r = run_build_and_query(in, predicate, radius, (uint32_t)limit, nullptr, 0, &d_rows, nullptr, s,
                                        aux_stream(), &timer, &sc, &d_query, &dl);
    const size_t row_size = predicate == kFrn ? sizeof(RtdlFixedRadiusNeighborRow) : sizeof(RtdlKnnNeighborRow);
    void* host;
    if (dl.host) {  // the copies were queued while the rows were emitted
      static thread_local cudaEvent_t ev_copied = nullptr;
      if (!ev_copied) RTDL_CUDA_CHECK(cudaEventCreateWithFlags(&ev_copied, cudaEventDisableTiming));
      RTDL_CUDA_CHECK(cudaEventRecord(ev_copied, dl.copy));
      RTDL_CUDA_CHECK(cudaStreamWaitEvent(s, ev_copied, 0));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      host = dl.host;
      dl.host = nullptr;
    } else {
      host = download_rows(d_rows, row_size * r.rows, s);
    }
    timer.mark("download");
    timer.publish();
    *rows_out = host;
    *row_count_out = (size_t)r.rows;
  } catch (...) {
    sync_quietly(aux_stream());
    release_host();
    dev_free(d_rows, s);
    destroy_scene(sc);
    dev_free(d_search, s);
    dev_free(d_query, s);
    sync_quietly(s);
    throw;
  }
  dev_free(d_rows, s);
  destroy_scene(sc);
  dev_free(d_search, s);
  dev_free(d_query, s);
}

struct PreparedHandle {
  Scene* scene;
  int dim;
};

}  // namespace

int scene_leaf_size() {
  if (tuning().leaf_size > 0) return tuning().leaf_size;
  return 32;
}

cudaStream_t aux_stream(int which) {
  static thread_local std::map<std::pair<int, int>, cudaStream_t> streams;
  int dev = 0;
  RTDL_CUDA_CHECK(cudaGetDevice(&dev));
  auto it = streams.find({dev, which});
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  RTDL_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[{dev, which}] = s;
  return s;
}
}  // namespace rtdl_b200

using namespace rtdl_b200;

extern "C" {

int rtdl_b200_get_version(int* major, int* minor, int* patch) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  if (patch) *patch = 0;
  return 0;
}

int rtdl_b200_set_device(int device) {
  return cudaSetDevice(device) == cudaSuccess ? 0 : 1;
}

int rtdl_b200_set_tuning(int leaf_size, int block_threads, int traversal) {
  if (leaf_size < 0 || leaf_size > 32) return 1;
  if (block_threads != 64 && block_threads != 128 && block_threads != 256) return 1;
  if (traversal < 0 || traversal > 4) return 1;
  Tuning t;
  t.leaf_size = leaf_size;
  t.block_threads = block_threads;
  t.traversal = traversal;
  set_tuning(t);
  return 0;
}

int rtdl_b200_get_last_phase_timings(const char** names_out, double* values_ms_out, int capacity) {
  const int n = (int)g_last_timings.size();
  for (int i = 0; i < n && i < capacity; ++i) {
    if (names_out) names_out[i] = g_last_timings[i].first;
    if (values_ms_out) values_ms_out[i] = g_last_timings[i].second;
  }
  return n;
}

int rtdl_b200_get_last_query_stats(unsigned long long* values_out, int capacity) {
  const auto& v = last_stats();
  for (int i = 0; i < (int)v.size() && i < capacity; ++i) values_out[i] = v[i];
  return (int)v.size();
}

int rtdl_b200_get_launch_count(unsigned long long* count_out) {
  if (!count_out) return 1;
  *count_out = g_launches.load(std::memory_order_relaxed);
  return 0;
}

void rtdl_b200_free_rows(void* rows) {
  if (!rows) return;
  if (!pinned_pool().put(rows)) std::free(rows);
}

int rtdl_b200_run_fixed_radius_neighbors(const RtdlPoint* query_points, size_t query_count,
                                         const RtdlPoint* search_points, size_t search_count, double radius,
                                         size_t k_max, RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
                                         char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(radius, k_max, query_count, search_count, true, "fixed_radius_neighbors", "k_max");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    run_rows_call(query_points, query_count, search_points, search_count, 2, kFrn, radius, k_max,
                  reinterpret_cast<void**>(rows_out), row_count_out);
  }, error_out, error_size);
}

int rtdl_b200_run_fixed_radius_neighbors_3d(const RtdlPoint3D* query_points, size_t query_count,
                                            const RtdlPoint3D* search_points, size_t search_count, double radius,
                                            size_t k_max, RtdlFixedRadiusNeighborRow** rows_out,
                                            size_t* row_count_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(radius, k_max, query_count, search_count, true, "fixed_radius_neighbors", "k_max");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    run_rows_call(query_points, query_count, search_points, search_count, 3, kFrn, radius, k_max,
                  reinterpret_cast<void**>(rows_out), row_count_out);
  }, error_out, error_size);
}

int rtdl_b200_run_fixed_radius_neighbors_device(const void* query_points_dev, size_t query_count,
                                                const void* search_points_dev, size_t search_count, int dimension,
                                                double radius, size_t k_max, void* rows_dev, size_t rows_capacity,
                                                size_t* row_count_out, uint8_t* overflow_dev, void* stream,
                                                char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!row_count_out) throw std::runtime_error("row_count_out must not be null");
    if (dimension != 2 && dimension != 3) throw std::runtime_error("dimension must be 2 or 3");
    validate_common(radius, k_max, query_count, search_count, true, "fixed_radius_neighbors", "k_max");
    *row_count_out = 0;
    if (query_count == 0) return;
    if (!query_points_dev) throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    if (!search_points_dev && search_count)
      throw std::runtime_error("search_points pointer must not be null when search_count is nonzero");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : library_stream();
    int dev = 0;
    RTDL_CUDA_CHECK(cudaGetDevice(&dev));
    ensure_pool_configured(dev);
    if (search_count == 0) {
      if (overflow_dev) RTDL_CUDA_CHECK(cudaMemsetAsync(overflow_dev, 0, query_count, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      return;
    }
    PhaseTimer timer(s);
    timer.mark("begin");
    Scene* sc = nullptr;
    void* owned = nullptr;
    try {
      BuildQueryInputs in{search_points_dev, (uint32_t)search_count, query_points_dev, nullptr, (uint32_t)query_count,
                          dimension};
      QueryResult r = run_build_and_query(in, kFrn, radius, (uint32_t)k_max, rows_dev, rows_capacity, nullptr,
                                          overflow_dev, s, aux_stream(), &timer, &sc, &owned);
      destroy_scene(sc);
      sc = nullptr;
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      timer.publish();
      *row_count_out = (size_t)r.rows;
    } catch (...) {
      sync_quietly(aux_stream());
      destroy_scene(sc);
      sync_quietly(s);
      throw;
    }
  }, error_out, error_size);
}

int rtdl_b200_run_bounded_knn_rows(const RtdlPoint* query_points, size_t query_count, const RtdlPoint* search_points,
                                   size_t search_count, double radius, size_t k_max, RtdlKnnNeighborRow** rows_out,
                                   size_t* row_count_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(radius, k_max, query_count, search_count, true, "bounded_knn_rows", "k_max");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    run_rows_call(query_points, query_count, search_points, search_count, 2, kBounded, radius, k_max,
                  reinterpret_cast<void**>(rows_out), row_count_out);
  }, error_out, error_size);
}

int rtdl_b200_run_bounded_knn_rows_3d(const RtdlPoint3D* query_points, size_t query_count,
                                      const RtdlPoint3D* search_points, size_t search_count, double radius,
                                      size_t k_max, RtdlKnnNeighborRow** rows_out, size_t* row_count_out,
                                      char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(radius, k_max, query_count, search_count, true, "bounded_knn_rows", "k_max");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    run_rows_call(query_points, query_count, search_points, search_count, 3, kBounded, radius, k_max,
                  reinterpret_cast<void**>(rows_out), row_count_out);
  }, error_out, error_size);
}

int rtdl_b200_run_k_closest_hits(const RtdlPoint* query_points, size_t query_count, const RtdlPoint* search_points,
                                 size_t search_count, size_t k, RtdlKnnNeighborRow** rows_out, size_t* row_count_out,
                                 char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(0.0, k, query_count, search_count, false, "knn_rows", "k");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    run_rows_call(query_points, query_count, search_points, search_count, 2, kKnn, 0.0, k,
                  reinterpret_cast<void**>(rows_out), row_count_out);
  }, error_out, error_size);
}

int rtdl_b200_run_k_closest_hits_3d(const RtdlPoint3D* query_points, size_t query_count,
                                    const RtdlPoint3D* search_points, size_t search_count, size_t k,
                                    RtdlKnnNeighborRow** rows_out, size_t* row_count_out, char* error_out,
                                    size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(0.0, k, query_count, search_count, false, "knn_rows", "k");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    run_rows_call(query_points, query_count, search_points, search_count, 3, kKnn, 0.0, k,
                  reinterpret_cast<void**>(rows_out), row_count_out);
  }, error_out, error_size);
}

namespace rtdl_b200 {
namespace {
int scene_create_impl(const void* points, size_t count, int dimension, int points_on_device, void* stream,
                      void** scene_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!scene_out) throw std::runtime_error("scene_out must not be null");
    *scene_out = nullptr;
    if (dimension != 2 && dimension != 3) throw std::runtime_error("dimension must be 2 or 3");
    if (!points && count != 0) throw std::runtime_error("points pointer must not be null when count is nonzero");
    if (count > (size_t)UINT32_MAX) throw std::runtime_error("search_count exceeds uint32 limit");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : library_stream();
    int dev = 0;
    RTDL_CUDA_CHECK(cudaGetDevice(&dev));
    ensure_pool_configured(dev);
    const void* d_points = points;
    void* owned = nullptr;
    if (!points_on_device && count) {
      owned = upload(points, record_size(dimension) * count, s);
      d_points = owned;
    }
    Scene* sc = nullptr;
    try {
      sc = build_scene(d_points, (uint32_t)count, dimension, s, scene_leaf_size());
      unsigned int bad = 0;
      RTDL_CUDA_CHECK(cudaMemcpyAsync(&bad, &sc->stats->bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      throw_if_bad(bad);
    } catch (...) {
      destroy_scene(sc);
      dev_free(owned, s);
      sync_quietly(s);
      throw;
    }
    dev_free(owned, s);
    *scene_out = sc;
  }, error_out, error_size);
}
}  // namespace
}  // namespace rtdl_b200

int rtdl_b200_scene_create(const void* points, size_t count, int dimension, int points_on_device, void* stream,
                           void** scene_out, char* error_out, size_t error_size) {
  return scene_create_impl(points, count, dimension, points_on_device, stream, scene_out, error_out,
                           error_size);
}

void rtdl_b200_scene_destroy(void* scene) {
  Scene* sc = static_cast<Scene*>(scene);
  if (!sc) return;
  cudaStream_t s = sc->stream;
  destroy_scene(sc);
  if (s) cudaStreamSynchronize(s);
}

int rtdl_b200_scene_query(void* scene, const void* query_points, size_t query_count, int predicate, double radius,
                          size_t limit, void** rows_out, size_t* row_count_out, uint8_t* overflow_out,
                          char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    if (predicate < 0 || predicate > 2) throw std::runtime_error("predicate must be 0, 1 or 2");
    const char* what = predicate == kFrn ? "fixed_radius_neighbors" : predicate == kBounded ? "bounded_knn_rows" : "knn_rows";
    validate_common(radius, limit, query_count, sc->n, predicate != kKnn, what, predicate == kKnn ? "k" : "k_max");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0) return;
    if (!query_points) throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    timer.mark("begin");
    void* d_query = upload(query_points, record_size(sc->dim) * query_count, s);
    uint8_t* d_overflow = overflow_out ? static_cast<uint8_t*>(dev_alloc(query_count, s)) : nullptr;
    if (d_overflow) RTDL_CUDA_CHECK(cudaMemsetAsync(d_overflow, 0, query_count, s));
    timer.mark("upload");
    void* d_rows = nullptr;
    try {
      QueryResult r = run_query(sc, d_query, (uint32_t)query_count, predicate, radius, (uint32_t)limit, nullptr, 0,
                                &d_rows, d_overflow, s, &timer);
      const size_t row_size = predicate == kFrn ? sizeof(RtdlFixedRadiusNeighborRow) : sizeof(RtdlKnnNeighborRow);
      if (d_overflow) RTDL_CUDA_CHECK(cudaMemcpyAsync(overflow_out, d_overflow, query_count, cudaMemcpyDeviceToHost, s));
      void* host = download_rows(d_rows, row_size * r.rows, s);
      timer.mark("download");
      timer.publish();
      *rows_out = host;
      *row_count_out = (size_t)r.rows;
    } catch (...) {
      dev_free(d_rows, s);
      dev_free(d_query, s);
      dev_free(d_overflow, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_rows, s);
    dev_free(d_query, s);
    dev_free(d_overflow, s);
  }, error_out, error_size);
}

int rtdl_b200_scene_query_device(void* scene, const void* query_points_dev, size_t query_count, int predicate,
                                 double radius, size_t limit, void* rows_dev, size_t rows_capacity,
                                 size_t* row_count_out, uint8_t* overflow_dev, void* stream, char* error_out,
                                 size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (!row_count_out) throw std::runtime_error("row_count_out must not be null");
    if (predicate < 0 || predicate > 2) throw std::runtime_error("predicate must be 0, 1 or 2");
    const char* what = predicate == kFrn ? "fixed_radius_neighbors" : predicate == kBounded ? "bounded_knn_rows" : "knn_rows";
    validate_common(radius, limit, query_count, sc->n, predicate != kKnn, what, predicate == kKnn ? "k" : "k_max");
    *row_count_out = 0;
    if (query_count == 0) return;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    QueryResult r = run_query(sc, query_points_dev, (uint32_t)query_count, predicate, radius, (uint32_t)limit,
                              rows_dev, rows_capacity, nullptr, overflow_dev, s, &timer);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    timer.publish();
    *row_count_out = (size_t)r.rows;
  }, error_out, error_size);
}

int rtdl_b200_batch_create(const void* points, const unsigned long long* point_offsets, uint32_t problems,
                           int dimension, int points_on_device, void* stream, void** batch_out, char* error_out,
                           size_t error_size) {
  return guarded([&]() {
    if (!batch_out) throw std::runtime_error("batch_out must not be null");
    *batch_out = nullptr;
    if (dimension != 2 && dimension != 3) throw std::runtime_error("dimension must be 2 or 3");
    if (problems == 0) throw std::runtime_error("a problem batch needs at least one problem");
    if (!point_offsets) throw std::runtime_error("point_offsets must not be null");
    const unsigned long long count = point_offsets[problems];
    if (!points && count != 0) throw std::runtime_error("points pointer must not be null when count is nonzero");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : library_stream();
    int dev = 0;
    RTDL_CUDA_CHECK(cudaGetDevice(&dev));
    ensure_pool_configured(dev);
    const void* d_points = points;
    void* owned = nullptr;
    Scene* sc = nullptr;
    try {
      if (!points_on_device && count) {
        owned = upload(points, record_size(dimension) * count, s);
        d_points = owned;
      }
      sc = build_scene_batch(d_points, point_offsets, problems, dimension, s, scene_leaf_size());
      unsigned int bad = 0;
      RTDL_CUDA_CHECK(cudaMemcpyAsync(&bad, &sc->stats->bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      throw_if_bad(bad);
    } catch (...) {
      destroy_scene(sc);
      dev_free(owned, s);
      sync_quietly(s);
      throw;
    }
    dev_free(owned, s);
    *batch_out = sc;
  }, error_out, error_size);
}

void rtdl_b200_batch_destroy(void* batch) { rtdl_b200_scene_destroy(batch); }

int rtdl_b200_batch_fixed_radius_neighbors(void* batch, const void* query_points,
                                           const unsigned long long* query_offsets, const double* radius,
                                           const uint32_t* k_max, RtdlFixedRadiusNeighborRow** rows_out,
                                           unsigned long long* row_offsets_out, uint8_t* overflow_out,
                                           char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(batch);
    if (!sc || sc->problems == 0) throw std::runtime_error("batch must be a problem batch handle");
    if (!query_offsets || !radius || !k_max || !rows_out || !row_offsets_out)
      throw std::runtime_error("query_offsets, radius, k_max, rows_out and row_offsets_out must not be null");
    *rows_out = nullptr;
    const unsigned long long nq = query_offsets[sc->problems];
    if (!query_points && nq != 0) throw std::runtime_error("query_points pointer must not be null when queries exist");
    BatchSpec bs;
    bs.problems = sc->problems;
    bs.qoff = query_offsets;
    bs.radius = radius;
    bs.kmax = k_max;
    bs.row_offsets = row_offsets_out;
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    timer.mark("begin");
    void* d_query = nq ? upload(query_points, record_size(sc->dim) * nq, s) : nullptr;
    uint8_t* d_overflow = (overflow_out && nq) ? static_cast<uint8_t*>(dev_alloc(nq, s)) : nullptr;
    if (d_overflow) RTDL_CUDA_CHECK(cudaMemsetAsync(d_overflow, 0, nq, s));
    timer.mark("upload");
    void* d_rows = nullptr;
    try {
      QueryResult r = run_query_batch(sc, d_query, bs, nullptr, 0, &d_rows, d_overflow, s, &timer);
      if (d_overflow) RTDL_CUDA_CHECK(cudaMemcpyAsync(overflow_out, d_overflow, nq, cudaMemcpyDeviceToHost, s));
      void* host = download_rows(d_rows, sizeof(RtdlFixedRadiusNeighborRow) * r.rows, s);
      timer.mark("download");
      timer.publish();
      *rows_out = static_cast<RtdlFixedRadiusNeighborRow*>(host);
    } catch (...) {
      dev_free(d_rows, s);
      dev_free(d_query, s);
      dev_free(d_overflow, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_rows, s);
    dev_free(d_query, s);
    dev_free(d_overflow, s);
  }, error_out, error_size);
}

int rtdl_b200_batch_fixed_radius_neighbors_device(void* batch, const void* query_points_dev,
                                                  const unsigned long long* query_offsets, const double* radius,
                                                  const uint32_t* k_max, void* rows_dev, size_t rows_capacity,
                                                  unsigned long long* row_offsets_out, uint8_t* overflow_dev,
                                                  void* stream, char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(batch);
    if (!sc || sc->problems == 0) throw std::runtime_error("batch must be a problem batch handle");
    if (!query_offsets || !radius || !k_max || !row_offsets_out)
      throw std::runtime_error("query_offsets, radius, k_max and row_offsets_out must not be null");
    BatchSpec bs;
    bs.problems = sc->problems;
    bs.qoff = query_offsets;
    bs.radius = radius;
    bs.kmax = k_max;
    bs.row_offsets = row_offsets_out;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    run_query_batch(sc, query_points_dev, bs, rows_dev, rows_capacity, nullptr, overflow_dev, s, &timer);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    timer.publish();
  }, error_out, error_size);
}

int rtdl_b200_batch_graph_create(void* const* batches, uint32_t batch_count, const void* query_points_dev,
                                 const unsigned long long* query_offsets, const double* radius,
                                 const uint32_t* k_max, void* rows_dev, size_t rows_capacity, void** graph_out,
                                 char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!graph_out) throw std::runtime_error("graph_out must not be null");
    *graph_out = nullptr;
    if (!batches) throw std::runtime_error("batches must not be null");
    std::vector<Scene*> scenes(batch_count);
    for (uint32_t i = 0; i < batch_count; ++i) scenes[i] = static_cast<Scene*>(batches[i]);
    *graph_out = batch_graph_create(scenes.data(), batch_count, query_points_dev, query_offsets, radius, k_max,
                                    rows_dev, rows_capacity);
  }, error_out, error_size);
}

int rtdl_b200_batch_graph_replay(void* graph, unsigned long long* row_offsets_out, uint32_t* status_out,
                                 char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!graph) throw std::runtime_error("graph must not be null");
    unsigned int st = 0;
    batch_graph_replay(static_cast<BatchGraph*>(graph), row_offsets_out, &st);
    if (status_out) *status_out = st;
  }, error_out, error_size);
}

int rtdl_b200_batch_graph_launch(void* graph, void* stream, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!graph) throw std::runtime_error("graph must not be null");
    batch_graph_launch(static_cast<BatchGraph*>(graph), static_cast<cudaStream_t>(stream));
  }, error_out, error_size);
}

int rtdl_b200_batch_graph_info(void* graph, uint32_t* problems_out, int* kernel_nodes_out,
                               unsigned long long* fallbacks_out) {
  if (!graph) return 1;
  const BatchGraph* g = static_cast<const BatchGraph*>(graph);
  if (problems_out) *problems_out = batch_graph_problems(g);
  if (kernel_nodes_out) *kernel_nodes_out = batch_graph_kernels(g);
  if (fallbacks_out) *fallbacks_out = (unsigned long long)batch_graph_fallbacks(g);
  return 0;
}

void rtdl_b200_batch_graph_destroy(void* graph) { batch_graph_destroy(static_cast<BatchGraph*>(graph)); }

int rtdl_b200_scene_fixed_radius_neighbors_multi_device(void* scene, const void* query_points_dev,
                                                        const unsigned long long* query_offsets, uint32_t requests,
                                                        const double* radius, const uint32_t* k_max, void* rows_dev,
                                                        size_t rows_capacity, unsigned long long* row_offsets_out,
                                                        uint8_t* overflow_dev, void* stream, char* error_out,
                                                        size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (sc->problems != 0) throw std::runtime_error("a problem batch is queried with the batch entry points");
    if (requests == 0) throw std::runtime_error("requests must be positive");
    if (!query_offsets || !radius || !k_max || !row_offsets_out)
      throw std::runtime_error("query_offsets, radius, k_max and row_offsets_out must not be null");
    BatchSpec bs;
    bs.problems = requests;
    bs.qoff = query_offsets;
    bs.radius = radius;
    bs.kmax = k_max;
    bs.row_offsets = row_offsets_out;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    run_query_batch(sc, query_points_dev, bs, rows_dev, rows_capacity, nullptr, overflow_dev, s, &timer);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    timer.publish();
  }, error_out, error_size);
}

int rtdl_b200_scene_directed_hausdorff(void* scene, const void* query_points, size_t query_count,
                                       double* distance_out, uint32_t* source_id_out, uint32_t* target_id_out,
                                       double* nearest_distance_out, uint32_t* nearest_id_out, char* error_out,
                                       size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (query_count > (size_t)UINT32_MAX) throw std::runtime_error("query_count exceeds uint32 limit");
    if (query_count == 0 || sc->n == 0) throw std::runtime_error("Hausdorff distance requires non-empty point sets");
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    timer.mark("begin");
    void* d_query = upload(query_points, record_size(sc->dim) * query_count, s);
    double* d_nd = nearest_distance_out ? static_cast<double*>(dev_alloc(sizeof(double) * query_count, s)) : nullptr;
    uint32_t* d_ni = nearest_id_out ? static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * query_count, s)) : nullptr;
    timer.mark("upload");
    try {
      HausdorffResult h = run_directed_hausdorff(sc, d_query, (uint32_t)query_count, d_nd, d_ni, s, &timer);
      if (d_nd) RTDL_CUDA_CHECK(cudaMemcpyAsync(nearest_distance_out, d_nd, sizeof(double) * query_count, cudaMemcpyDeviceToHost, s));
      if (d_ni) RTDL_CUDA_CHECK(cudaMemcpyAsync(nearest_id_out, d_ni, sizeof(uint32_t) * query_count, cudaMemcpyDeviceToHost, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      timer.mark("download");
      timer.publish();
      if (distance_out) *distance_out = h.distance;
      if (source_id_out) *source_id_out = h.source_id;
      if (target_id_out) *target_id_out = h.target_id;
    } catch (...) {
      dev_free(d_query, s);
      dev_free(d_nd, s);
      dev_free(d_ni, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_query, s);
    dev_free(d_nd, s);
    dev_free(d_ni, s);
  }, error_out, error_size);
}

int rtdl_b200_scene_directed_hausdorff_device(void* scene, const void* query_points_dev, size_t query_count,
                                              double* nearest_distance_dev, uint32_t* nearest_id_dev,
                                              double* distance_out, uint32_t* source_id_out, uint32_t* target_id_out,
                                              void* stream, char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (query_count > (size_t)UINT32_MAX) throw std::runtime_error("query_count exceeds uint32 limit");
    if (query_count == 0 || sc->n == 0) throw std::runtime_error("Hausdorff distance requires non-empty point sets");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    HausdorffResult h = run_directed_hausdorff(sc, query_points_dev, (uint32_t)query_count, nearest_distance_dev,
                                               nearest_id_dev, s, &timer);
    timer.publish();
    if (distance_out) *distance_out = h.distance;
    if (source_id_out) *source_id_out = h.source_id;
    if (target_id_out) *target_id_out = h.target_id;
  }, error_out, error_size);
}

int rtdl_b200_scene_directed_hausdorff_noalloc(void* scene, const void* query_points_dev, size_t query_count,
                                               double* nearest_distance_dev, uint32_t* nearest_id_dev,
                                               RtdlB200Witness* witness_dev, void* stream, char* error_out,
                                               size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (!witness_dev) throw std::runtime_error("witness_dev must not be null");
    if (query_count > (size_t)UINT32_MAX) throw std::runtime_error("query_count exceeds uint32 limit");
    if (query_count != 0 && !query_points_dev) throw std::runtime_error("query_points_dev must not be null");
    run_directed_hausdorff_noalloc(sc, query_points_dev, (uint32_t)query_count, nearest_distance_dev, nearest_id_dev,
                                   witness_dev, static_cast<cudaStream_t>(stream));
  }, error_out, error_size);
}

int rtdl_b200_prepare_fixed_radius_neighbors_3d(const RtdlPoint3D* search_points, size_t search_count,
                                                double max_radius, void** prepared_out, char* error_out,
                                                size_t error_size) {
  return guarded([&]() {
    if (!prepared_out) throw std::runtime_error("prepared_out must not be null");
    if (!search_points && search_count != 0)
      throw std::runtime_error("search_points pointer must not be null when search_count is nonzero");
    if (!(max_radius > 0.0)) throw std::runtime_error("fixed_radius_neighbors_3d max_radius must be positive");
    if (search_count > (size_t)UINT32_MAX)
      throw std::runtime_error("fixed_radius_neighbors_3d search_count exceeds uint32 limit");
    *prepared_out = nullptr;
    void* scene = nullptr;
    char err[1024];
    if (scene_create_impl(search_points, search_count, 3, 0, nullptr, &scene, err, sizeof(err)) != 0)
      throw std::runtime_error(err);
    static_cast<Scene*>(scene)->max_radius = max_radius;
    *prepared_out = scene;
  }, error_out, error_size);
}

int rtdl_b200_run_prepared_fixed_radius_neighbors_3d(void* prepared, const RtdlPoint3D* query_points,
                                                     size_t query_count, double radius, size_t k_max,
                                                     RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
                                                     char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(prepared);
    if (!sc) throw std::runtime_error("prepared handle must not be null");
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    validate_common(radius, k_max, query_count, sc->n, true, "fixed_radius_neighbors_3d", "k_max");
    if (sc->dim != 3) throw std::runtime_error("prepared scene is not 3D");
    // same tolerance as the reference (rtdl_optix_workloads.cpp:15629-15631)
    if (radius > sc->max_radius + 1.0e-7)
      throw std::runtime_error("fixed_radius_neighbors_3d radius exceeds prepared max_radius");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || sc->n == 0) return;
    char err[1024];
    void* rows = nullptr;
    if (rtdl_b200_scene_query(sc, query_points, query_count, kFrn, radius, k_max, &rows, row_count_out, nullptr, err,
                              sizeof(err)) != 0)
      throw std::runtime_error(err);
    *rows_out = static_cast<RtdlFixedRadiusNeighborRow*>(rows);
  }, error_out, error_size);
}

void rtdl_b200_destroy_prepared_fixed_radius_neighbors_3d(void* prepared) { rtdl_b200_scene_destroy(prepared); }

namespace {
// Shared checks of the prepared ranked-summary calls (messages as
// rtdl_optix_workloads.cpp:15011-15022).
Scene* prepared_summary_scene(void* prepared, double radius, size_t query_count, size_t k_max) {
  Scene* sc = static_cast<Scene*>(prepared);
  if (!sc) throw std::runtime_error("prepared OptiX fixed-radius-neighbor 3D handle must not be null");
  if (sc->dim != 3) throw std::runtime_error("prepared scene is not 3D");
  if (radius < 0.0) throw std::runtime_error("fixed_radius_neighbors_3d radius must be non-negative");
  if (radius > sc->max_radius + 1.0e-7)
    throw std::runtime_error("fixed_radius_neighbors_3d radius exceeds prepared max_radius");
  if (query_count > (size_t)UINT32_MAX) throw std::runtime_error("fixed_radius_neighbors_3d query_count exceeds uint32 limit");
  if (k_max == 0) throw std::runtime_error("fixed_radius_neighbors_3d k_max must be positive");
  if (k_max > 64)
    throw std::runtime_error("prepared ranked fixed_radius_neighbors_3d aggregate currently supports k_max <= 64");
  return sc;
}
}  // namespace

int rtdl_b200_run_prepared_ranked_fixed_radius_neighbor_summaries_3d(
    void* prepared, const RtdlPoint3D* query_points, size_t query_count, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborSummary** rows_out, size_t* row_count_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    *rows_out = nullptr;
    *row_count_out = 0;
    Scene* sc = prepared_summary_scene(prepared, radius, query_count, k_max);
    if (query_count == 0 || sc->n == 0) return;
    if (!query_points) throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    timer.mark("begin");
    void* d_query = upload(query_points, sizeof(RtdlPoint3D) * query_count, s);
    RtdlFixedRadiusRankedNeighborSummary* d_sum = nullptr;
    try {
      d_sum = static_cast<RtdlFixedRadiusRankedNeighborSummary*>(
          dev_alloc(sizeof(RtdlFixedRadiusRankedNeighborSummary) * query_count, s));
      timer.mark("upload");
      RtdlFixedRadiusRankedNeighborAggregate agg;
      run_ranked_summaries(sc, d_query, (uint32_t)query_count, radius, (uint32_t)k_max, d_sum, &agg, s, &timer);
      void* host = download_rows(d_sum, sizeof(RtdlFixedRadiusRankedNeighborSummary) * query_count, s);
      timer.mark("download");
      timer.publish();
      *rows_out = static_cast<RtdlFixedRadiusRankedNeighborSummary*>(host);
      *row_count_out = query_count;
    } catch (...) {
      dev_free(d_sum, s);
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_sum, s);
    dev_free(d_query, s);
  }, error_out, error_size);
}

int rtdl_b200_aggregate_prepared_ranked_fixed_radius_neighbor_summaries_3d(
    void* prepared, const RtdlPoint3D* query_points, size_t query_count, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!aggregate_out) throw std::runtime_error("aggregate_out must not be null");
    *aggregate_out = RtdlFixedRadiusRankedNeighborAggregate{query_count, 0u, 0u, 0u, 0.0};
    Scene* sc = prepared_summary_scene(prepared, radius, query_count, k_max);
    if (query_count == 0 || sc->n == 0) return;
    if (!query_points) throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    timer.mark("begin");
    void* d_query = upload(query_points, sizeof(RtdlPoint3D) * query_count, s);
    try {
      timer.mark("upload");
      run_ranked_summaries(sc, d_query, (uint32_t)query_count, radius, (uint32_t)k_max, nullptr, aggregate_out, s,
                           &timer);
      timer.publish();
    } catch (...) {
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_query, s);
  }, error_out, error_size);
}

int rtdl_b200_queries_create(const void* points, size_t count, int dimension, int points_on_device, void* stream,
                             void** queries_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!queries_out) throw std::runtime_error("queries_out must not be null");
    *queries_out = nullptr;
    if (dimension != 2 && dimension != 3) throw std::runtime_error("dimension must be 2 or 3");
    if (!points && count != 0) throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    if (count > (size_t)UINT32_MAX) throw std::runtime_error("query_count exceeds uint32 limit");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : library_stream();
    int dev = 0;
    RTDL_CUDA_CHECK(cudaGetDevice(&dev));
    ensure_pool_configured(dev);
    const size_t bytes = record_size(dimension) * count;
    void* owned = dev_alloc(bytes ? bytes : 1, s);
    if (bytes)
      RTDL_CUDA_CHECK(cudaMemcpyAsync(owned, points, bytes, points_on_device ? cudaMemcpyDeviceToDevice
                                                                            : cudaMemcpyHostToDevice, s));
    PreparedQueries* pq = nullptr;
    try {
      pq = prepare_query_set(owned, (uint32_t)count, dimension, s);
      unsigned int bad = 0;
      RTDL_CUDA_CHECK(cudaMemcpyAsync(&bad, &pq->qst->bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
      RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      throw_if_bad(bad);
    } catch (...) {
      if (pq) destroy_query_set(pq); else dev_free(owned, s);
      sync_quietly(s);
      throw;
    }
    *queries_out = pq;
  }, error_out, error_size);
}

void rtdl_b200_queries_destroy(void* queries) {
  PreparedQueries* pq = static_cast<PreparedQueries*>(queries);
  if (!pq) return;
  cudaStream_t s = pq->stream;
  destroy_query_set(pq);
  if (s) cudaStreamSynchronize(s);
}

int rtdl_b200_prepare_fixed_radius_query_points_3d(const RtdlPoint3D* query_points, size_t query_count,
                                                   void** prepared_queries_out, char* error_out, size_t error_size) {
  return rtdl_b200_queries_create(query_points, query_count, 3, 0, nullptr, prepared_queries_out, error_out,
                                  error_size);
}

void rtdl_b200_destroy_prepared_fixed_radius_query_points_3d(void* prepared_queries) {
  rtdl_b200_queries_destroy(prepared_queries);
}

int rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d(
    void* prepared, void* prepared_queries, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!aggregate_out) throw std::runtime_error("aggregate_out must not be null");
    PreparedQueries* pq = static_cast<PreparedQueries*>(prepared_queries);
    if (!pq) throw std::runtime_error("prepared fixed-radius query handle must not be null");
    *aggregate_out = RtdlFixedRadiusRankedNeighborAggregate{pq->n, 0u, 0u, 0u, 0.0};
    Scene* sc = prepared_summary_scene(prepared, radius, pq->n, k_max);
    if (pq->dim != 3) throw std::runtime_error("prepared queries are not 3D");
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    run_ranked_summaries(sc, nullptr, pq->n, radius, (uint32_t)k_max, nullptr, aggregate_out, s, &timer, pq);
    timer.publish();
  }, error_out, error_size);
}

int rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d_f32(
    void* prepared, void* prepared_queries, double radius, size_t k_max,
    RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, char* error_out, size_t error_size) {
  return rtdl_b200_aggregate_prepared_query_ranked_fixed_radius_neighbor_summaries_3d(
      prepared, prepared_queries, radius, k_max, aggregate_out, error_out, error_size);
}

int rtdl_b200_scene_ranked_summaries_prepared_device(void* scene, void* queries, double radius, size_t k_max,
                                                     RtdlFixedRadiusRankedNeighborSummary* summaries_dev,
                                                     RtdlFixedRadiusRankedNeighborAggregate* aggregate_out,
                                                     void* stream, char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    PreparedQueries* pq = static_cast<PreparedQueries*>(queries);
    if (!sc || !pq) throw std::runtime_error("scene and queries must not be null");
    if (!aggregate_out) throw std::runtime_error("aggregate_out must not be null");
    validate_common(radius, k_max, pq->n, sc->n, true, "fixed_radius_neighbors", "k_max");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    run_ranked_summaries(sc, nullptr, pq->n, radius, (uint32_t)k_max, summaries_dev, aggregate_out, s, &timer, pq);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    timer.publish();
  }, error_out, error_size);
}

namespace {
std::vector<uint32_t> graph_k_values(const size_t* k_values, size_t request_count) {
  if (request_count > (size_t)UINT32_MAX)
    throw std::runtime_error("fixed_radius_neighbors_3d graph request_count exceeds uint32 limit");
  if (!k_values && request_count) throw std::runtime_error("k_values pointer must not be null when request_count is nonzero");
  std::vector<uint32_t> k(request_count);
  for (size_t r = 0; r < request_count; ++r) {
    if (k_values[r] > 64)
      throw std::runtime_error("prepared ranked fixed_radius_neighbors_3d aggregate currently supports k_max <= 64");
    k[r] = (uint32_t)k_values[r];
  }
  return k;
}
}  // namespace

int rtdl_b200_prepare_fixed_radius_ranked_summary_aggregate_batch_graph_3d(
    void* prepared, void* prepared_queries, const double* radii, const size_t* k_values, size_t request_count,
    void** graph_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!graph_out) throw std::runtime_error("graph_out must not be null");
    *graph_out = nullptr;
    if (!radii && request_count) throw std::runtime_error("radii pointer must not be null when request_count is nonzero");
    const std::vector<uint32_t> k = graph_k_values(k_values, request_count);
    Scene* sc = static_cast<Scene*>(prepared);
    if (sc && sc->dim != 3) throw std::runtime_error("prepared scene is not 3D");
    *graph_out = summary_graph_create(sc, static_cast<PreparedQueries*>(prepared_queries), radii, k.data(),
                                      (uint32_t)request_count);
  }, error_out, error_size);
}

int rtdl_b200_update_fixed_radius_ranked_summary_aggregate_batch_graph_3d(
    void* graph, const double* radii, const size_t* k_values, size_t request_count, char* error_out,
    size_t error_size) {
  return guarded([&]() {
    if (!radii && request_count) throw std::runtime_error("radii pointer must not be null when request_count is nonzero");
    const std::vector<uint32_t> k = graph_k_values(k_values, request_count);
    summary_graph_update(static_cast<SummaryGraph*>(graph), radii, k.data(), (uint32_t)request_count);
  }, error_out, error_size);
}

int rtdl_b200_replay_fixed_radius_ranked_summary_aggregate_batch_graph_3d(
    void* graph, RtdlFixedRadiusRankedNeighborAggregate* aggregates_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    SummaryGraph* g = static_cast<SummaryGraph*>(graph);
    if (!g) throw std::runtime_error("prepared fixed_radius_neighbors_3d graph handle must not be null");
    summary_graph_replay(g, aggregates_out);
  }, error_out, error_size);
}

int rtdl_b200_launch_fixed_radius_ranked_summary_aggregate_batch_graph_device_partials_3d(
    void* graph, uint64_t* partials_device_ptr_out, size_t* partial_count_out, size_t* request_count_out,
    size_t* query_block_count_out, uint64_t* cuda_stream_ptr_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    SummaryGraph* g = static_cast<SummaryGraph*>(graph);
    if (!g) throw std::runtime_error("prepared fixed_radius_neighbors_3d graph handle must not be null");
    if (!partials_device_ptr_out) throw std::runtime_error("partials_device_ptr_out must not be null");
    if (!partial_count_out) throw std::runtime_error("partial_count_out must not be null");
    if (!request_count_out) throw std::runtime_error("request_count_out must not be null");
    if (!query_block_count_out) throw std::runtime_error("query_block_count_out must not be null");
    if (!cuda_stream_ptr_out) throw std::runtime_error("cuda_stream_ptr_out must not be null");
    summary_graph_launch(g);
    const uint32_t R = summary_graph_requests(g);
    *partials_device_ptr_out = reinterpret_cast<uint64_t>(summary_graph_device_aggregates(g));
    *partial_count_out = R;
    *request_count_out = R;
    *query_block_count_out = 1;
    *cuda_stream_ptr_out = reinterpret_cast<uint64_t>(summary_graph_stream(g));
  }, error_out, error_size);
}

int rtdl_b200_fixed_radius_ranked_summary_aggregate_batch_graph_status_device_3d(
    void* graph, uint64_t* status_device_ptr_out, uint64_t* fallback_count_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    SummaryGraph* g = static_cast<SummaryGraph*>(graph);
    if (!g) throw std::runtime_error("prepared fixed_radius_neighbors_3d graph handle must not be null");
    if (status_device_ptr_out) *status_device_ptr_out = reinterpret_cast<uint64_t>(summary_graph_device_status(g));
    if (fallback_count_out) *fallback_count_out = summary_graph_fallbacks(g);
  }, error_out, error_size);
}

void rtdl_b200_destroy_fixed_radius_ranked_summary_aggregate_batch_graph_3d(void* graph) {
  summary_graph_destroy(static_cast<SummaryGraph*>(graph));
}

// ---- fixed_radius_count_threshold and the nearest witness ------------------------
namespace rtdl_b200 {
namespace {
void count_checks(double radius, size_t query_count, size_t threshold, const char* what) {
  const std::string w(what);
  if (radius < 0.0) throw std::runtime_error(w + " radius must be non-negative");
  if (query_count > (size_t)UINT32_MAX) throw std::runtime_error(w + " query_count exceeds uint32 limit");
  if (threshold > (size_t)UINT32_MAX) throw std::runtime_error(w + " threshold exceeds uint32 limit");
}

Scene* prepared_count_scene(void* prepared, int dim, double radius, const char* what, const char* null_msg) {
  Scene* sc = static_cast<Scene*>(prepared);
  if (!sc) throw std::runtime_error(null_msg);
  if (sc->dim != dim) throw std::runtime_error(dim == 3 ? "prepared scene is not 3D" : "prepared scene is not 2D");
  if (radius > sc->max_radius + 1.0e-7) throw std::runtime_error(std::string(what) + " radius exceeds prepared max_radius");
  return sc;
}

// Counts into 12-byte rows (device) and returns them in a pinned host buffer.
void count_rows_to_host(Scene* sc, const void* d_query, uint32_t nq, double radius, uint32_t threshold,
                        RtdlFixedRadiusCountRow** rows_out, size_t* row_count_out, cudaStream_t s) {
  RtdlFixedRadiusCountRow* d_rows =
      static_cast<RtdlFixedRadiusCountRow*>(dev_alloc(sizeof(RtdlFixedRadiusCountRow) * nq, s));
  try {
    CountOutputs out;
    out.rows = d_rows;
    run_count_threshold(sc, d_query, nq, radius, threshold, out, s);
    *rows_out = static_cast<RtdlFixedRadiusCountRow*>(download_rows(d_rows, sizeof(RtdlFixedRadiusCountRow) * nq, s));
    *row_count_out = nq;
  } catch (...) {
    dev_free(d_rows, s);
    throw;
  }
  dev_free(d_rows, s);
}

int prepare_count_scene(const void* points, size_t count, int dim, int on_device, double max_radius,
                        bool device_columns, void** prepared_out, char* error_out, size_t error_size) {
  void* scene = nullptr;
  char err[1024];
  if (scene_create_impl(points, count, dim, on_device, nullptr, &scene, err, sizeof(err)) != 0) {
    if (error_out && error_size) {
      std::strncpy(error_out, err, error_size - 1);
      error_out[error_size - 1] = 0;
    }
    return 1;
  }
  static_cast<Scene*>(scene)->max_radius = max_radius;
  static_cast<Scene*>(scene)->device_columns = device_columns;
  *prepared_out = scene;
  return 0;
}
}  // namespace
}  // namespace rtdl_b200

int rtdl_b200_run_fixed_radius_count_threshold(const RtdlPoint* query_points, size_t query_count,
                                               const RtdlPoint* search_points, size_t search_count, double radius,
                                               size_t threshold, RtdlFixedRadiusCountRow** rows_out,
                                               size_t* row_count_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    count_checks(radius, query_count, threshold, "fixed_radius_count_threshold");
    if (search_count > (size_t)UINT32_MAX)
      throw std::runtime_error("fixed_radius_count_threshold search_count exceeds uint32 limit");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || search_count == 0) return;
    if (!query_points || !search_points) throw std::runtime_error("point pointers must not be null when counts are nonzero");
    cudaStream_t s = library_stream();
    void* d_search = upload(search_points, sizeof(RtdlPoint) * search_count, s);
    void* d_query = nullptr;
    Scene* sc = nullptr;
    try {
      sc = build_scene(d_search, (uint32_t)search_count, 2, s, scene_leaf_size());
      d_query = upload(query_points, sizeof(RtdlPoint) * query_count, s);
      count_rows_to_host(sc, d_query, (uint32_t)query_count, radius, (uint32_t)threshold, rows_out, row_count_out, s);
    } catch (...) {
      destroy_scene(sc);
      dev_free(d_search, s);
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    destroy_scene(sc);
    dev_free(d_search, s);
    dev_free(d_query, s);
  }, error_out, error_size);
}

int rtdl_b200_prepare_fixed_radius_count_threshold_2d(const RtdlPoint* search_points, size_t search_count,
                                                      double max_radius, void** prepared_out, char* error_out,
                                                      size_t error_size) {
  if (!prepared_out) return guarded([] { throw std::runtime_error("prepared_out must not be null"); }, error_out, error_size);
  *prepared_out = nullptr;
  const int st = guarded([&]() {
    if (!search_points && search_count != 0)
      throw std::runtime_error("search_points pointer must not be null when search_count is nonzero");
    if (max_radius < 0.0) throw std::runtime_error("fixed_radius_count_threshold max_radius must be non-negative");
    if (search_count > (size_t)UINT32_MAX)
      throw std::runtime_error("fixed_radius_count_threshold search_count exceeds uint32 limit");
  }, error_out, error_size);
  if (st != 0) return st;
  return prepare_count_scene(search_points, search_count, 2, 0, max_radius, false, prepared_out, error_out, error_size);
}

int rtdl_b200_prepare_fixed_radius_count_threshold_2d_device_search_columns(
    const uint32_t* search_ids, const double* search_x, const double* search_y, size_t search_count,
    double max_radius, void** prepared_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!prepared_out) throw std::runtime_error("prepared_out must not be null");
    *prepared_out = nullptr;
    if ((!search_ids || !search_x || !search_y) && search_count != 0)
      throw std::runtime_error("search column pointers must not be null when search_count is nonzero");
    if (max_radius < 0.0) throw std::runtime_error("fixed_radius_count_threshold max_radius must be non-negative");
    if (search_count > (size_t)UINT32_MAX)
      throw std::runtime_error("fixed_radius_count_threshold search_count exceeds uint32 limit");
    cudaStream_t s = library_stream();
    void* recs = dev_alloc(sizeof(RtdlPoint) * (search_count ? search_count : 1), s);
    columns_to_records_2d(search_ids, search_x, search_y, (uint32_t)search_count, recs, s);
    char err[1024];
    const int st = prepare_count_scene(recs, search_count, 2, 1, max_radius, true, prepared_out, err, sizeof(err));
    dev_free(recs, s);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    if (st != 0) throw std::runtime_error(err);
  }, error_out, error_size);
}

int rtdl_b200_run_prepared_fixed_radius_count_threshold_2d(void* prepared, const RtdlPoint* query_points,
                                                           size_t query_count, double radius, size_t threshold,
                                                           RtdlFixedRadiusCountRow** rows_out, size_t* row_count_out,
                                                           char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX fixed-radius handle must not be null");
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    count_checks(radius, query_count, threshold, "fixed_radius_count_threshold");
    Scene* sc = prepared_count_scene(prepared, 2, radius, "fixed_radius_count_threshold",
                                     "prepared OptiX fixed-radius handle must not be null");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || sc->n == 0) return;
    cudaStream_t s = sc->stream;
    void* d_query = upload(query_points, sizeof(RtdlPoint) * query_count, s);
    try {
      count_rows_to_host(sc, d_query, (uint32_t)query_count, radius, (uint32_t)threshold, rows_out, row_count_out, s);
    } catch (...) {
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_query, s);
  }, error_out, error_size);
}

int rtdl_b200_write_prepared_fixed_radius_count_threshold_2d_device_query_columns(
    void* prepared, const uint32_t* query_ids, const double* query_x, const double* query_y, size_t query_count,
    double radius, size_t threshold, uint32_t* query_ids_out, uint32_t* neighbor_counts_out,
    uint32_t* threshold_flags_out, char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX fixed-radius handle must not be null");
    Scene* sc = static_cast<Scene*>(prepared);
    if (!sc->device_columns)
      throw std::runtime_error("fixed-radius device-column output requires a device-search-column prepared scene");
    count_checks(radius, query_count, threshold, "fixed_radius_count_threshold");
    prepared_count_scene(prepared, 2, radius, "fixed_radius_count_threshold", "");
    if (query_count == 0) return;
    if (!query_ids || !query_x || !query_y)
      throw std::runtime_error("query column pointers must not be null when query_count is nonzero");
    if (!query_ids_out || !neighbor_counts_out || !threshold_flags_out)
      throw std::runtime_error("device output pointers must not be null when query_count is nonzero");
    cudaStream_t s = sc->stream;
    void* recs = dev_alloc(sizeof(RtdlPoint) * query_count, s);
    try {
      columns_to_records_2d(query_ids, query_x, query_y, (uint32_t)query_count, recs, s);
      CountOutputs out;
      out.ids = query_ids_out;
      out.counts = neighbor_counts_out;
      out.flags = threshold_flags_out;
      run_count_threshold(sc, recs, (uint32_t)query_count, radius, (uint32_t)threshold, out, s);
    } catch (...) {
      dev_free(recs, s);
      sync_quietly(s);
      throw;
    }
    dev_free(recs, s);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  }, error_out, error_size);
}

int rtdl_b200_count_prepared_fixed_radius_threshold_reached_2d(void* prepared, const RtdlPoint* query_points,
                                                               size_t query_count, double radius, size_t threshold,
                                                               size_t* threshold_reached_count_out, char* error_out,
                                                               size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX fixed-radius handle must not be null");
    if (!threshold_reached_count_out) throw std::runtime_error("threshold_reached_count_out must not be null");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    count_checks(radius, query_count, threshold, "fixed_radius_count_threshold");
    Scene* sc = prepared_count_scene(prepared, 2, radius, "fixed_radius_count_threshold", "");
    *threshold_reached_count_out = 0;
    if (query_count == 0 || sc->n == 0) return;
    cudaStream_t s = sc->stream;
    void* d_query = upload(query_points, sizeof(RtdlPoint) * query_count, s);
    unsigned long long reached = 0;
    try {
      CountOutputs out;
      out.reached_host = &reached;
      run_count_threshold(sc, d_query, (uint32_t)query_count, radius, (uint32_t)threshold, out, s);
    } catch (...) {
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_query, s);
    *threshold_reached_count_out = (size_t)reached;
  }, error_out, error_size);
}

int rtdl_b200_run_prepared_fixed_radius_nearest_witness_2d(void* prepared, const RtdlPoint* query_points,
                                                           size_t query_count, double radius,
                                                           RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
                                                           char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX fixed-radius handle must not be null");
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    if (radius < 0.0) throw std::runtime_error("fixed_radius_nearest_witness radius must be non-negative");
    Scene* sc = prepared_count_scene(prepared, 2, radius, "fixed_radius_nearest_witness", "");
    if (query_count > (size_t)UINT32_MAX)
      throw std::runtime_error("fixed_radius_nearest_witness query_count exceeds uint32 limit");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || sc->n == 0) return;
    cudaStream_t s = sc->stream;
    PhaseTimer timer(s);
    timer.mark("begin");
    void* d_query = upload(query_points, sizeof(RtdlPoint) * query_count, s);
    void* d_rows = nullptr;
    try {
      QueryResult r = run_nearest_witness(sc, d_query, (uint32_t)query_count, radius, &d_rows, s, &timer);
      *rows_out = static_cast<RtdlFixedRadiusNeighborRow*>(
          download_rows(d_rows, sizeof(RtdlFixedRadiusNeighborRow) * r.rows, s));
      *row_count_out = (size_t)r.rows;
      timer.mark("download");
      timer.publish();
    } catch (...) {
      dev_free(d_rows, s);
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_rows, s);
    dev_free(d_query, s);
  }, error_out, error_size);
}

void rtdl_b200_destroy_prepared_fixed_radius_count_threshold_2d(void* prepared) { rtdl_b200_scene_destroy(prepared); }

int rtdl_b200_prepare_fixed_radius_count_threshold_3d(const RtdlPoint3D* search_points, size_t search_count,
                                                      double max_radius, void** prepared_out, char* error_out,
                                                      size_t error_size) {
  if (!prepared_out) return guarded([] { throw std::runtime_error("prepared_out must not be null"); }, error_out, error_size);
  *prepared_out = nullptr;
  const int st = guarded([&]() {
    if (!search_points && search_count != 0)
      throw std::runtime_error("search_points pointer must not be null when search_count is nonzero");
    if (!(max_radius > 0.0)) throw std::runtime_error("fixed_radius_count_threshold_3d max_radius must be positive");
    if (search_count > (size_t)UINT32_MAX)
      throw std::runtime_error("fixed_radius_count_threshold_3d search_count exceeds uint32 limit");
  }, error_out, error_size);
  if (st != 0) return st;
  return prepare_count_scene(search_points, search_count, 3, 0, max_radius, false, prepared_out, error_out, error_size);
}

int rtdl_b200_write_prepared_fixed_radius_count_threshold_3d_device_outputs(
    void* prepared, const RtdlPoint3D* query_points, size_t query_count, double radius, size_t threshold,
    uint32_t* query_ids_out, uint32_t* neighbor_counts_out, uint32_t* threshold_flags_out, char* error_out,
    size_t error_size) {
  return guarded([&]() {
    const char* null_msg = "prepared OptiX fixed-radius count-threshold 3D handle must not be null";
    if (!prepared) throw std::runtime_error(null_msg);
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    count_checks(radius, query_count, threshold, "fixed_radius_count_threshold_3d");
    Scene* sc = prepared_count_scene(prepared, 3, radius, "fixed_radius_count_threshold_3d", null_msg);
    if (query_count == 0) return;
    if (!query_ids_out || !neighbor_counts_out || !threshold_flags_out)
      throw std::runtime_error(
          "fixed_radius_count_threshold_3d device output pointers must not be null when query_count is nonzero");
    cudaStream_t s = sc->stream;
    void* d_query = upload(query_points, sizeof(RtdlPoint3D) * query_count, s);
    try {
      CountOutputs out;
      out.ids = query_ids_out;
      out.counts = neighbor_counts_out;
      out.flags = threshold_flags_out;
      if (threshold == 0)
        run_count_trivial(d_query, (uint32_t)query_count, 3, out, s);
      else
        run_count_threshold(sc, d_query, (uint32_t)query_count, radius, (uint32_t)threshold, out, s);
    } catch (...) {
      dev_free(d_query, s);
      sync_quietly(s);
      throw;
    }
    dev_free(d_query, s);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
  }, error_out, error_size);
}

void rtdl_b200_destroy_prepared_fixed_radius_count_threshold_3d(void* prepared) { rtdl_b200_scene_destroy(prepared); }

// ---- point-group witness ---------------------------------------------------------
namespace rtdl_b200 {
namespace {
PointGroupScene* point_group_checked(void* prepared, double radius, size_t query_count, const char* what) {
  PointGroupScene* pg = static_cast<PointGroupScene*>(prepared);
  if (!pg) throw std::runtime_error("prepared OptiX point-group handle must not be null");
  const std::string w(what);
  if (radius < 0.0) throw std::runtime_error(w + " radius must be non-negative");
  if (radius > pg->max_radius + 1.0e-7) throw std::runtime_error(w + " radius exceeds prepared max_radius");
  if (query_count > (size_t)UINT32_MAX) throw std::runtime_error(w + " query_count exceeds uint32 limit");
  return pg;
}

// Uploads host query records, runs `fn(d_query, s)`, releases them.
void with_queries(PointGroupScene* pg, const RtdlPoint* query_points, size_t query_count,
                  const std::function<void(const void*, cudaStream_t)>& fn) {
  cudaStream_t s = pg->sc->stream;
  void* d_query = upload(query_points, sizeof(RtdlPoint) * query_count, s);
  try {
    fn(d_query, s);
  } catch (...) {
    dev_free(d_query, s);
    sync_quietly(s);
    throw;
  }
  dev_free(d_query, s);
}
}  // namespace
}  // namespace rtdl_b200

int rtdl_b200_prepare_point_group_nearest_witness_2d(const RtdlPoint* search_points, size_t search_count,
                                                     const RtdlPointGroupBounds2D* groups, size_t group_count,
                                                     double max_radius, void** prepared_out, char* error_out,
                                                     size_t error_size) {
  return guarded([&]() {
    if (!prepared_out) throw std::runtime_error("prepared_out must not be null");
    *prepared_out = nullptr;
    if (!search_points && search_count != 0)
      throw std::runtime_error("point_group search_points pointer must not be null when search_count is nonzero");
    if (!groups && group_count != 0)
      throw std::runtime_error("point_group groups pointer must not be null when group_count is nonzero");
    if (max_radius < 0.0) throw std::runtime_error("point_group_nearest_witness max_radius must be non-negative");
    if (search_count > (size_t)UINT32_MAX)
      throw std::runtime_error("point_group_nearest_witness search_count exceeds uint32 limit");
    if (group_count > (size_t)UINT32_MAX)
      throw std::runtime_error("point_group_nearest_witness group_count exceeds uint32 limit");
    int dev = 0;
    RTDL_CUDA_CHECK(cudaGetDevice(&dev));
    ensure_pool_configured(dev);
    *prepared_out = point_group_create(search_points, search_count, groups, group_count, max_radius,
                                       scene_leaf_size(), library_stream());
  }, error_out, error_size);
}

int rtdl_b200_count_prepared_point_group_threshold_reached_2d(void* prepared, const RtdlPoint* query_points,
                                                              size_t query_count, double radius, size_t threshold,
                                                              size_t* threshold_reached_count_out, char* error_out,
                                                              size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX point-group handle must not be null");
    if (!threshold_reached_count_out) throw std::runtime_error("threshold_reached_count_out must not be null");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    PointGroupScene* pg = point_group_checked(prepared, radius, query_count, "point_group_threshold");
    if (threshold > (size_t)UINT32_MAX) throw std::runtime_error("point_group_threshold threshold exceeds uint32 limit");
    *threshold_reached_count_out = 0;
    if (query_count == 0 || pg->groups == 0) return;
    unsigned long long reached = 0;
    with_queries(pg, query_points, query_count, [&](const void* d_query, cudaStream_t s) {
      CountOutputs out;
      out.reached_host = &reached;
      point_group_count(pg, d_query, (uint32_t)query_count, radius, (uint32_t)threshold, out, s);
    });
    *threshold_reached_count_out = (size_t)reached;
  }, error_out, error_size);
}

int rtdl_b200_write_prepared_point_group_threshold_flags_2d(void* prepared, const RtdlPoint* query_points,
                                                            size_t query_count, double radius, size_t threshold,
                                                            uint32_t* threshold_flags_out, char* error_out,
                                                            size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX point-group handle must not be null");
    if (!threshold_flags_out && query_count != 0)
      throw std::runtime_error("threshold_flags_out must not be null when query_count is nonzero");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    PointGroupScene* pg = point_group_checked(prepared, radius, query_count, "point_group_threshold_flags");
    if (threshold > (size_t)UINT32_MAX)
      throw std::runtime_error("point_group_threshold_flags threshold exceeds uint32 limit");
    if (query_count == 0) return;
    if (pg->groups == 0) {  // as the reference: threshold 0 counts as reached without groups
      for (size_t i = 0; i < query_count; ++i) threshold_flags_out[i] = threshold == 0 ? 1u : 0u;
      return;
    }
    with_queries(pg, query_points, query_count, [&](const void* d_query, cudaStream_t s) {
      uint32_t* d_flags = static_cast<uint32_t*>(dev_alloc(sizeof(uint32_t) * query_count, s));
      try {
        CountOutputs out;
        out.flags = d_flags;
        point_group_count(pg, d_query, (uint32_t)query_count, radius, (uint32_t)threshold, out, s);
        RTDL_CUDA_CHECK(cudaMemcpyAsync(threshold_flags_out, d_flags, sizeof(uint32_t) * query_count,
                                        cudaMemcpyDeviceToHost, s));
        RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
      } catch (...) {
        dev_free(d_flags, s);
        throw;
      }
      dev_free(d_flags, s);
    });
  }, error_out, error_size);
}

int rtdl_b200_run_prepared_point_group_nearest_witness_2d(void* prepared, const RtdlPoint* query_points,
                                                          size_t query_count, double radius,
                                                          RtdlFixedRadiusNeighborRow** rows_out, size_t* row_count_out,
                                                          char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX point-group handle must not be null");
    if (!rows_out || !row_count_out) throw std::runtime_error("output pointers must not be null");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    PointGroupScene* pg = point_group_checked(prepared, radius, query_count, "point_group_nearest_witness");
    *rows_out = nullptr;
    *row_count_out = 0;
    if (query_count == 0 || pg->groups == 0) return;
    with_queries(pg, query_points, query_count, [&](const void* d_query, cudaStream_t s) {
      RtdlFixedRadiusNeighborRow* d_rows =
          static_cast<RtdlFixedRadiusNeighborRow*>(dev_alloc(sizeof(RtdlFixedRadiusNeighborRow) * query_count, s));
      try {
        point_group_nearest(pg, d_query, (uint32_t)query_count, radius, d_rows, nullptr, s);
        *rows_out = static_cast<RtdlFixedRadiusNeighborRow*>(
            download_rows(d_rows, sizeof(RtdlFixedRadiusNeighborRow) * query_count, s));
        *row_count_out = query_count;
      } catch (...) {
        dev_free(d_rows, s);
        throw;
      }
      dev_free(d_rows, s);
    });
  }, error_out, error_size);
}

int rtdl_b200_reduce_prepared_point_group_nearest_max_distance_2d(void* prepared, const RtdlPoint* query_points,
                                                                  size_t query_count, double radius,
                                                                  RtdlFixedRadiusNeighborRow* row_out,
                                                                  char* error_out, size_t error_size) {
  return guarded([&]() {
    if (!prepared) throw std::runtime_error("prepared OptiX point-group handle must not be null");
    if (!row_out) throw std::runtime_error("row_out must not be null");
    if (!query_points && query_count != 0)
      throw std::runtime_error("query_points pointer must not be null when query_count is nonzero");
    PointGroupScene* pg = point_group_checked(prepared, radius, query_count, "point_group_nearest_max_distance");
    *row_out = RtdlFixedRadiusNeighborRow{0xFFFFFFFFu, 0xFFFFFFFFu, std::numeric_limits<double>::infinity()};
    if (query_count == 0 || pg->groups == 0) return;
    with_queries(pg, query_points, query_count, [&](const void* d_query, cudaStream_t s) {
      RtdlFixedRadiusNeighborRow* d_rows =
          static_cast<RtdlFixedRadiusNeighborRow*>(dev_alloc(sizeof(RtdlFixedRadiusNeighborRow) * query_count, s));
      try {
        point_group_nearest(pg, d_query, (uint32_t)query_count, radius, d_rows, row_out, s);
      } catch (...) {
        dev_free(d_rows, s);
        throw;
      }
      dev_free(d_rows, s);
    });
  }, error_out, error_size);
}

void rtdl_b200_destroy_prepared_point_group_nearest_witness_2d(void* prepared) {
  point_group_destroy(static_cast<PointGroupScene*>(prepared));
}

int rtdl_b200_scene_query_prepared_device(void* scene, void* queries, double radius, size_t k_max, void* rows_dev,
                                          size_t rows_capacity, size_t* row_count_out, uint8_t* overflow_dev,
                                          void* stream, char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    PreparedQueries* pq = static_cast<PreparedQueries*>(queries);
    if (!sc || !pq) throw std::runtime_error("scene and queries must not be null");
    if (!row_count_out) throw std::runtime_error("row_count_out must not be null");
    validate_common(radius, k_max, pq->n, sc->n, true, "fixed_radius_neighbors", "k_max");
    *row_count_out = 0;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    QueryResult r = run_query_prepared(sc, pq, radius, (uint32_t)k_max, rows_dev, rows_capacity, overflow_dev, s,
                                       &timer);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    timer.publish();
    *row_count_out = (size_t)r.rows;
  }, error_out, error_size);
}

int rtdl_b200_scene_ranked_summaries_device(void* scene, const void* query_points_dev, size_t query_count,
                                            double radius, size_t k_max,
                                            RtdlFixedRadiusRankedNeighborSummary* summaries_dev,
                                            RtdlFixedRadiusRankedNeighborAggregate* aggregate_out, void* stream,
                                            char* error_out, size_t error_size) {
  return guarded([&]() {
    Scene* sc = static_cast<Scene*>(scene);
    if (!sc) throw std::runtime_error("scene must not be null");
    if (!aggregate_out) throw std::runtime_error("aggregate_out must not be null");
    validate_common(radius, k_max, query_count, sc->n, true, "fixed_radius_neighbors", "k_max");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sc->stream;
    PhaseTimer timer(s);
    run_ranked_summaries(sc, query_points_dev, (uint32_t)query_count, radius, (uint32_t)k_max, summaries_dev,
                         aggregate_out, s, &timer);
    RTDL_CUDA_CHECK(cudaStreamSynchronize(s));
    timer.publish();
  }, error_out, error_size);
}

}  // extern "C"
