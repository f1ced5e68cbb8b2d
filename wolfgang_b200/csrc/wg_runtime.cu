// wg_runtime.cu -- C-ABI runtime plumbing: errors, device discovery, the
// stream-ordered memory pool, copies and pointer validation.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wg_common.cuh"

namespace wg {

namespace {
thread_local std::string g_last_error;
std::atomic<long> g_fail_after{0};
std::mutex g_props_mu;
std::vector<DeviceProps> g_props;
std::vector<bool> g_pool_ready;
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }

namespace {
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {
struct ProfEntry {
  const char* name;
  cudaEvent_t a, b;
};
std::atomic<bool> g_prof_on{false};
std::mutex g_prof_mu;
std::vector<ProfEntry> g_prof;
std::vector<cudaEvent_t> g_prof_free;
thread_local std::vector<std::pair<const char*, cudaEvent_t>> g_prof_open;

cudaEvent_t prof_event() {
  if (!g_prof_free.empty()) {
    cudaEvent_t e = g_prof_free.back();
    g_prof_free.pop_back();
    return e;
  }
  cudaEvent_t e;
  check_cuda(cudaEventCreate(&e), "create profiling event");
  return e;
}
}  // namespace

bool profiling() { return g_prof_on.load(std::memory_order_relaxed); }

void prof_record(const char* name, cudaStream_t s, bool begin) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  cudaEvent_t e = prof_event();
  if (cudaEventRecord(e, s) != cudaSuccess) {
    (void)cudaGetLastError();
    g_prof_free.push_back(e);
    return;
  }
  if (begin) {
    g_prof_open.emplace_back(name, e);
    return;
  }
  for (size_t i = g_prof_open.size(); i-- > 0;) {
    if (g_prof_open[i].first == name) {
      g_prof.push_back(ProfEntry{name, g_prof_open[i].second, e});
      g_prof_open.erase(g_prof_open.begin() + static_cast<long>(i));
      return;
    }
  }
  g_prof_free.push_back(e);
}

int current_device() {
  int d = 0;
  check_cuda(cudaGetDevice(&d), "get current device");
  return d;
}

const DeviceProps& device_props(int device) {
  std::lock_guard<std::mutex> lk(g_props_mu);
  if (device < 0) throw_invalid("CUDA device ordinal is out of range");
  if (static_cast<size_t>(device) >= g_props.size()) {
    g_props.resize(device + 1);
    g_pool_ready.resize(device + 1, false);
  }
  DeviceProps& p = g_props[device];
  if (p.sm_count == 0) {
    int v = 0;
    check_cuda(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device), "query SM count");
    p.sm_count = v;
    check_cuda(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device),
               "query shared memory");
    p.max_smem_optin = v;
    check_cuda(cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, device), "query L2 size");
    p.l2_bytes = static_cast<size_t>(v);
    cudaDeviceProp dp{};
    check_cuda(cudaGetDeviceProperties(&dp, device), "query device memory");
    p.total_mem = dp.totalGlobalMem;
  }
  if (!g_pool_ready[device]) {
    // Keep freed blocks cached in the pool instead of returning them to the
    // driver at every synchronisation: repeated calls reuse scratch without
    // cudaMalloc cost.
    cudaMemPool_t pool;
    check_cuda(cudaDeviceGetDefaultMemPool(&pool, device), "get default memory pool");
    uint64_t thr = UINT64_MAX;
    check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr),
               "set pool release threshold");
    g_pool_ready[device] = true;
  }
  return p;
}

void* pool_alloc(size_t bytes, cudaStream_t s) {
  if (bytes == 0) return nullptr;
  long f = g_fail_after.load();
  if (f > 0) {
    f = g_fail_after.fetch_sub(1);
    if (f == 1) throw Error(WG_ERR_OOM, "CUDA allocate device buffer failed: out of memory (injected)");
  }
  void* p = nullptr;
  check_cuda(cudaMallocAsync(&p, bytes, s), "allocate device buffer");
  return p;
}

void pool_free(void* p, cudaStream_t s) noexcept {
  if (p != nullptr) {
    if (cudaFreeAsync(p, s) != cudaSuccess) (void)cudaGetLastError();
  }
}

// ------------------------------------------------------------ staged copies
//
// Large copies between the device and pageable host memory go through two
// pinned 64 MiB staging buffers: the DMA engine fills (or drains) one while
// host threads copy the other, so the transfer runs near the link rate
// instead of the driver's single-threaded pageable path.
namespace {
constexpr size_t kStageBytes = size_t{64} << 20;
struct Staging {
  std::mutex mu;
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
};
Staging g_staging;

void parallel_memcpy(char* dst, const char* src, size_t bytes) {
  static const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  if (nt == 1 || bytes < (size_t{4} << 20)) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t part = (bytes + nt - 1) / nt;
  std::vector<std::thread> th;
  for (unsigned i = 1; i < nt; ++i) {
    const size_t o = i * part;
    if (o >= bytes) break;
    const size_t len = std::min(part, bytes - o);
    th.emplace_back([=] { std::memcpy(dst + o, src + o, len); });
  }
  std::memcpy(dst, src, std::min(part, bytes));
  for (auto& t : th) t.join();
}
// Staging for chunked downloads: a ring of small pinned buffers, their events
// and a stream per concurrent call, kept for reuse.  The chunks are small and
// the ring shallow so that a chunk is consumed soon after its DMA lands.
constexpr size_t kChunkBytes = size_t{8} << 20;
constexpr int kChunkRing = 3;
struct ChunkStage {
  void* buf[kChunkRing] = {};
  cudaEvent_t done[kChunkRing] = {};
  cudaEvent_t ready = nullptr;  // recorded on the caller's stream: src is complete
  cudaStream_t stream = nullptr;
  int device = -1;
};
std::mutex g_chunk_mu;
std::vector<ChunkStage*> g_chunk_free;

ChunkStage* take_chunk_stage(int device) {
  {
    std::lock_guard<std::mutex> lk(g_chunk_mu);
    for (size_t i = 0; i < g_chunk_free.size(); ++i) {
      if (g_chunk_free[i]->device == device) {
        ChunkStage* c = g_chunk_free[i];
        g_chunk_free.erase(g_chunk_free.begin() + static_cast<std::ptrdiff_t>(i));
        return c;
      }
    }
  }
  auto* c = new ChunkStage;
  c->device = device;
  try {
    for (int i = 0; i < kChunkRing; ++i) {
      check_cuda(cudaHostAlloc(&c->buf[i], kChunkBytes, cudaHostAllocPortable), "allocate pinned staging");
      check_cuda(cudaEventCreateWithFlags(&c->done[i], cudaEventDisableTiming), "create staging event");
    }
    check_cuda(cudaEventCreateWithFlags(&c->ready, cudaEventDisableTiming), "create staging event");
    check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "create staging stream");
  } catch (...) {
    for (int i = 0; i < kChunkRing; ++i) {
      if (c->buf[i]) (void)cudaFreeHost(c->buf[i]);
      if (c->done[i]) (void)cudaEventDestroy(c->done[i]);
    }
    if (c->ready) (void)cudaEventDestroy(c->ready);
    delete c;
    throw;
  }
  return c;
}

void give_chunk_stage(ChunkStage* c) {
  std::lock_guard<std::mutex> lk(g_chunk_mu);
  g_chunk_free.push_back(c);
}
}  // namespace

void chunked_download(int device, const void* src, size_t bytes, wg_chunk_fn fn, void* user, cudaStream_t after) {
  ChunkStage* c = take_chunk_stage(device);
  const char* const sp = static_cast<const char*>(src);
  const size_t chunks = (bytes + kChunkBytes - 1) / kChunkBytes;
  auto len_of = [&](size_t k) { return std::min(kChunkBytes, bytes - k * kChunkBytes); };
  constexpr size_t ahead = kChunkRing - 1;  // chunks in flight while the caller consumes one
  try {
    // The staging stream is a non-blocking stream of its own: order its copies
    // after everything already enqueued on the caller's stream (the work that
    // writes src), or they could read src before that work has finished.
    check_cuda(cudaEventRecord(c->ready, after), "record download order");
    check_cuda(cudaStreamWaitEvent(c->stream, c->ready, 0), "order download after the caller's stream");
    // DMA chunk k into ring buffer k % kChunkRing while the caller consumes chunk k - ahead
    for (size_t k = 0; k < chunks + ahead; ++k) {
      if (k < chunks) {
        check_cuda(cudaMemcpyAsync(c->buf[k % kChunkRing], sp + k * kChunkBytes, len_of(k),
                                   cudaMemcpyDeviceToHost, c->stream),
                   "copy device buffer to staging");
        check_cuda(cudaEventRecord(c->done[k % kChunkRing], c->stream), "record staging event");
      }
      if (k >= ahead) {
        const size_t j = k - ahead;
        check_cuda(cudaEventSynchronize(c->done[j % kChunkRing]), "wait for staging");
        fn(user, c->buf[j % kChunkRing], len_of(j));
      }
    }
  } catch (...) {
    (void)cudaStreamSynchronize(c->stream);
    give_chunk_stage(c);
    throw;
  }
  give_chunk_stage(c);
}

bool pinned_host(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

void staged_copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_staging.mu);
  for (int i = 0; i < 2; ++i) {
    if (!g_staging.buf[i]) {
      check_cuda(cudaHostAlloc(&g_staging.buf[i], kStageBytes, cudaHostAllocPortable), "allocate pinned staging");
      check_cuda(cudaEventCreateWithFlags(&g_staging.done[i], cudaEventDisableTiming), "create staging event");
    }
  }
  char* const d = static_cast<char*>(dst);
  const char* const sp = static_cast<const char*>(src);
  const size_t chunks = (bytes + kStageBytes - 1) / kStageBytes;
  auto len_of = [&](size_t k) { return std::min(kStageBytes, bytes - k * kStageBytes); };
  if (kind == cudaMemcpyDeviceToHost) {
    // DMA chunk k into buffer k%2 while the host drains chunk k-1
    for (size_t k = 0; k <= chunks; ++k) {
      if (k < chunks) {
        char* b = static_cast<char*>(g_staging.buf[k & 1]);
        check_cuda(cudaMemcpyAsync(b, sp + k * kStageBytes, len_of(k), cudaMemcpyDeviceToHost, s),
                   "copy device buffer to staging");
        check_cuda(cudaEventRecord(g_staging.done[k & 1], s), "record staging event");
      }
      if (k > 0) {
        const size_t j = k - 1;
        check_cuda(cudaEventSynchronize(g_staging.done[j & 1]), "wait for staging");
        parallel_memcpy(d + j * kStageBytes, static_cast<const char*>(g_staging.buf[j & 1]), len_of(j));
      }
    }
  } else {
    // the host fills buffer k%2 once the DMA of chunk k-2 has drained it
    for (size_t k = 0; k < chunks; ++k) {
      if (k >= 2) check_cuda(cudaEventSynchronize(g_staging.done[k & 1]), "wait for staging");
      char* b = static_cast<char*>(g_staging.buf[k & 1]);
      parallel_memcpy(b, sp + k * kStageBytes, len_of(k));
      check_cuda(cudaMemcpyAsync(d + k * kStageBytes, b, len_of(k), cudaMemcpyHostToDevice, s),
                 "copy staging to device buffer");
      check_cuda(cudaEventRecord(g_staging.done[k & 1], s), "record staging event");
    }
  }
  check_cuda(cudaStreamSynchronize(s), "synchronize staged copy");
}

namespace {
constexpr int kMaxDevices = 64;
struct WorkspaceSlot {
  std::mutex mu;
  void* base = nullptr;
  size_t cap = 0;
};
WorkspaceSlot g_workspace[kMaxDevices];
}  // namespace

Workspace::Workspace(int device, size_t bytes, cudaStream_t s) : device_(device) {
  if (device < 0 || device >= kMaxDevices) throw_invalid("CUDA device ordinal is out of range");
  WorkspaceSlot& w = g_workspace[device];
  w.mu.lock();
  try {
    if (w.cap < bytes) {
      if (w.base) pool_free(w.base, s);
      w.base = nullptr;
      w.cap = 0;
      // some headroom, so that slightly larger calls reuse the block
      const size_t want = bytes + bytes / 8;
      w.base = pool_alloc(want, s);
      w.cap = want;
    }
  } catch (...) {
    w.mu.unlock();
    throw;
  }
  p_ = static_cast<char*>(w.base);
  end_ = p_ + w.cap;
}

Workspace::~Workspace() { g_workspace[device_].mu.unlock(); }

void* Workspace::take(size_t bytes) {
  const size_t r = rounded(bytes);
  if (static_cast<size_t>(end_ - p_) < r) throw Error(WG_ERR_INVALID, "internal: workspace piece exceeds its reservation");
  void* out = p_;
  p_ += r;
  return out;
}

void Scratch::reset(size_t bytes, cudaStream_t s) {
  release();
  s_ = s;
  p_ = pool_alloc(bytes, s);
  n_ = bytes;
}

void Scratch::release() noexcept {
  pool_free(p_, s_);
  p_ = nullptr;
  n_ = 0;
}

}  // namespace wg

using namespace wg;

extern "C" {

const char* wg_last_error(void) { return g_last_error.c_str(); }

int wg_abi_version(void) { return 1; }

int wg_device_count(int* count) {
  return guarded([&] {
    int c = 0;
    const cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      c = 0;
    }
    *count = c;
  });
}

int wg_runtime_versions(int* runtime_version, int* driver_version) {
  return guarded([&] {
    *runtime_version = 0;
    *driver_version = 0;
    (void)cudaRuntimeGetVersion(runtime_version);
    (void)cudaDriverGetVersion(driver_version);
  });
}

int wg_device_info(int ordinal, char* name, size_t name_cap, int* cc_major, int* cc_minor,
                   size_t* total_mem, int* sm_count) {
  return guarded([&] {
    cudaDeviceProp p{};
    check_cuda(cudaGetDeviceProperties(&p, ordinal), "query device properties");
    if (name && name_cap) {
      std::strncpy(name, p.name, name_cap - 1);
      name[name_cap - 1] = 0;
    }
    *cc_major = p.major;
    *cc_minor = p.minor;
    *total_mem = p.totalGlobalMem;
    *sm_count = p.multiProcessorCount;
  });
}

int wg_malloc(int device, size_t bytes, wg_stream_t stream, void** out) {
  return guarded([&] {
    DeviceGuard g(device);
    *out = pool_alloc(bytes, stream);
  });
}

int wg_free(int device, void* ptr, wg_stream_t stream) {
  return guarded([&] {
    if (ptr == nullptr) return;
    DeviceGuard g(device);
    check_cuda(cudaFreeAsync(ptr, stream), "free device buffer");
  });
}

int wg_memcpy_htod(int device, void* dst, const void* src, size_t bytes, wg_stream_t stream) {
  return guarded([&] {
    if (bytes == 0) return;
    DeviceGuard g(device);
    if (bytes >= kStagedMin && !wg::pinned_host(src)) {
      wg::staged_copy(dst, src, bytes, cudaMemcpyHostToDevice, stream);
      return;
    }
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), "copy host buffer to device");
  });
}

int wg_memcpy_dtoh(int device, void* dst, const void* src, size_t bytes, wg_stream_t stream) {
  return guarded([&] {
    if (bytes == 0) return;
    DeviceGuard g(device);
    if (bytes >= kStagedMin && !wg::pinned_host(dst)) {
      wg::staged_copy(dst, src, bytes, cudaMemcpyDeviceToHost, stream);
      return;
    }
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream), "copy device buffer to host");
    check_cuda(cudaStreamSynchronize(stream), "synchronize copy to host");
  });
}

int wg_memcpy_dtoh_chunked(int device, const void* src, size_t bytes, wg_chunk_fn fn, void* user,
                           wg_stream_t stream) {
  return guarded([&] {
    if (bytes == 0) return;
    if (fn == nullptr) throw_invalid("chunked download needs a chunk callback");
    DeviceGuard g(device);
    wg::chunked_download(device, src, bytes, fn, user, stream);
  });
}

int wg_memcpy_dtod(int device, void* dst, const void* src, size_t bytes, wg_stream_t stream) {
  return guarded([&] {
    if (bytes == 0) return;
    DeviceGuard g(device);
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream), "copy device buffer");
  });
}

int wg_memset(int device, void* dst, int value, size_t bytes, wg_stream_t stream) {
  return guarded([&] {
    if (bytes == 0) return;
    DeviceGuard g(device);
    check_cuda(cudaMemsetAsync(dst, value, bytes, stream), "fill device buffer");
  });
}

int wg_stream_synchronize(int device, wg_stream_t stream) {
  return guarded([&] {
    DeviceGuard g(device);
    check_cuda(cudaStreamSynchronize(stream), "synchronize stream");
  });
}

int wg_device_synchronize(int device) {
  return guarded([&] {
    DeviceGuard g(device);
    check_cuda(cudaDeviceSynchronize(), "synchronize device");
  });
}

int wg_pointer_check(const void* ptr, size_t bytes, int* is_device, int* device, int* in_one_allocation) {
  return guarded([&] {
    *is_device = -1;
    *device = -1;
    *in_one_allocation = 0;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
      (void)cudaGetLastError();
      return;
    }
    *is_device = 0;
    if (a.type != cudaMemoryTypeDevice) return;
    *is_device = 1;
    *device = a.device;
    // Driver entry point resolved through the runtime, so the library does not
    // link libcuda and still loads on machines without a driver.
    using range_fn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static range_fn get_range = [] {
      void* fn = nullptr;
      cudaDriverEntryPointQueryResult q{};
      if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) != cudaSuccess ||
          q != cudaDriverEntryPointSuccess) {
        (void)cudaGetLastError();
        return static_cast<range_fn>(nullptr);
      }
      return reinterpret_cast<range_fn>(fn);
    }();
    if (!get_range) return;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (get_range(&base, &size, reinterpret_cast<CUdeviceptr>(ptr)) != CUDA_SUCCESS) return;
    const uintptr_t p = reinterpret_cast<uintptr_t>(ptr);
    if (p < base) return;
    const uintptr_t off = p - base;
    *in_one_allocation = (off <= size && bytes <= size - off) ? 1 : 0;
  });
}

int wg_profile_enable(int on) {
  g_prof_on.store(on != 0);
  return WG_OK;
}

int wg_profile_report(char* buf, size_t cap) {
  return guarded([&] {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    struct Acc {
      unsigned long long count = 0;
      double ms = 0.0;
    };
    std::vector<std::pair<std::string, Acc>> acc;
    for (const ProfEntry& p : g_prof) {
      check_cuda(cudaEventSynchronize(p.b), "synchronize profiling event");
      float ms = 0.0f;
      check_cuda(cudaEventElapsedTime(&ms, p.a, p.b), "read profiling event");
      auto it = std::find_if(acc.begin(), acc.end(), [&](const auto& kv) { return kv.first == p.name; });
      if (it == acc.end()) {
        acc.emplace_back(p.name, Acc{});
        it = acc.end() - 1;
      }
      it->second.count += 1;
      it->second.ms += ms;
      g_prof_free.push_back(p.a);
      g_prof_free.push_back(p.b);
    }
    g_prof.clear();
    std::string out;
    for (const auto& [name, a] : acc)
      out += name + ":" + std::to_string(a.count) + ":" + std::to_string(a.ms) + ";";
    if (cap) {
      std::strncpy(buf, out.c_str(), cap - 1);
      buf[cap - 1] = 0;
    }
  });
}

int wg_kernel_launches(unsigned long long* count) {
  *count = g_launches.load(std::memory_order_relaxed);
  return WG_OK;
}

int wg_inject_alloc_failure(long n) {
  g_fail_after.store(n > 0 ? n : 0);
  return WG_OK;
}

}  // extern "C"
