// wg_common.cuh -- shared host/device plumbing for the sm_100a packed-Pauli kernels.
//
// Host side: thread-local error text, status codes, checked CUDA calls, and the
// device-property cache used to size grids in multiples of the SM count.
// Device side: exact-rounding FP64 complex helpers and key utilities.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "wg_pauli.h"

namespace wg {

// ---------------------------------------------------------------- host errors

void set_error(const std::string& msg);

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void throw_invalid(const std::string& m) { throw Error(WG_ERR_INVALID, m); }

inline void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  (void)cudaGetLastError();
  const int code = (e == cudaErrorMemoryAllocation) ? WG_ERR_OOM : WG_ERR_CUDA;
  throw Error(code, std::string("CUDA ") + what + " failed: " + cudaGetErrorString(e));
}

// Optional per-kernel timing (wg_profile_enable): a ProfRange placed before a
// launch records CUDA events on the launch stream around it; durations are
// summed per kernel name by wg_profile_report.
bool profiling();
void prof_record(const char* name, cudaStream_t s, bool begin);
struct ProfRange {
  const char* name;
  cudaStream_t s;
  bool on;
  ProfRange(const char* n, cudaStream_t st) : name(n), s(st), on(profiling()) {
    if (on) prof_record(name, s, true);
  }
  ~ProfRange() {
    if (on) prof_record(name, s, false);
  }
};

// Launch wrapped in a timing range named `name` on `stream`.
#define WG_TIMED(name, stream, ...)       \
  do {                                    \
    ::wg::ProfRange wg_prof_(name, stream); \
    __VA_ARGS__;                          \
  } while (0)

// Every kernel launch site calls check_launch, which also counts launches
// (wg_kernel_launches reports the total).
void count_launch();
inline void check_launch(const char* what) {
  count_launch();
  check_cuda(cudaGetLastError(), what);
}

// Runs f(), mapping exceptions onto the C-ABI status convention.
template <typename F>
int guarded(F&& f) {
  try {
    f();
    return WG_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return WG_ERR_OOM;
  } catch (const std::exception& e) {
    set_error(e.what());
    return WG_ERR_INVALID;
  }
}

// Per-device properties, cached after the first query.
struct DeviceProps {
  int sm_count = 0;
  int max_smem_optin = 0;
  size_t l2_bytes = 0;
  size_t total_mem = 0;
};
const DeviceProps& device_props(int device);
int current_device();

// Grid size for a grid-stride kernel: a whole number of waves of `per_sm`
// resident CTAs on every SM, never more blocks than work items need.
inline unsigned grid_for(size_t items, unsigned block_items, int device, int per_sm) {
  const size_t need = (items + block_items - 1) / block_items;
  const size_t wave = static_cast<size_t>(device_props(device).sm_count) * per_sm;
  size_t g = need < wave ? need : wave;
  if (g == 0) g = 1;
  return static_cast<unsigned>(g);
}

// Stream-ordered scratch from the device's default memory pool (cached by the
// pool between calls).  Freed on the same stream when the holder dies.
class Scratch {
 public:
  Scratch() = default;
  Scratch(size_t bytes, cudaStream_t s) { reset(bytes, s); }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  Scratch(Scratch&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; }
  Scratch& operator=(Scratch&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_;
      n_ = o.n_;
      s_ = o.s_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  ~Scratch() { release(); }
  void reset(size_t bytes, cudaStream_t s);
  void release() noexcept;
  void* get() const { return p_; }
  template <typename T>
  T* as() const { return static_cast<T*>(p_); }
  size_t size() const { return n_; }
  // Stream on which the buffer is released (for buffers that outlive the
  // stream they were allocated on).
  void rebind(cudaStream_t s) { s_ = s; }
  // Hands ownership to the caller (the result buffers of an entry point).
  void* detach() {
    void* p = p_;
    p_ = nullptr;
    n_ = 0;
    return p;
  }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};

// RAII device switch for entry points that take an explicit ordinal.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int device) {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      (void)cudaGetLastError();
      throw Error(WG_ERR_NO_DEVICE, "no CUDA device is available");
    }
    if (device < 0 || device >= count) throw_invalid("CUDA device ordinal is out of range");
    check_cuda(cudaGetDevice(&prev), "get current device");
    if (prev != device) check_cuda(cudaSetDevice(device), "set device");
    (void)device_props(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) (void)cudaSetDevice(prev);
  }
};

void* pool_alloc(size_t bytes, cudaStream_t s);
void pool_free(void* p, cudaStream_t s) noexcept;

// Copies of at least kStagedMin bytes between the device and pageable host
// memory run through pinned staging (wg_runtime.cu); both synchronise s.
constexpr size_t kStagedMin = size_t{32} << 20;
bool pinned_host(const void* p);
void staged_copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s);
// Device-to-host copy through a pinned staging pair of its own; fn gets each
// chunk in order on the calling thread.  The copies start after all work
// enqueued on `after` so far.
void chunked_download(int device, const void* src, size_t bytes, wg_chunk_fn fn, void* user, cudaStream_t after);

// Per-device grow-only workspace for an entry point's intermediates.  It is
// held for the whole call (calls on one device take turns on it) and kept for
// later calls, so large scratch of varying sizes does not fragment the memory
// pool: every call that uses it synchronises its stream before returning.
class Workspace {
 public:
  Workspace(int device, size_t bytes, cudaStream_t s);
  ~Workspace();
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;
  // 256-byte aligned piece of the reserved bytes.
  void* take(size_t bytes);
  template <typename T>
  T* take_as(size_t count) { return static_cast<T*>(take(sizeof(T) * count)); }
  static size_t rounded(size_t bytes) { return (bytes + 255) & ~size_t{255}; }

 private:
  int device_;
  char* p_ = nullptr;
  char* end_ = nullptr;
};

// Stable LSD radix sort of n items by K structure-of-arrays key words (word 0
// most significant) carrying a 32-bit item index (wg_simplify.cu).
void radix_sort_keys(int device, size_t n, int K, Scratch& keys, Scratch& idx, cudaStream_t s);

// Bucketed sort-reduce (wg_bucket.cu).  thr_mode: 0 cull at thr_fixed, 1 at
// atol + rtol*max|c|, 2 at atol (empty result when some |c| is infinite).
// Each returns false when the inputs are outside the bucketed path's limits;
// the caller then runs the LSD pipeline.
bool bucket_products(int device, int W, const uint64_t* lx, const uint64_t* lz, const double* lc, size_t n_l,
                     const uint64_t* rx, const uint64_t* rz, const double* rc, size_t n_r, int thr_mode, double atol,
                     double rtol, double thr_fixed, uint64_t** ox, uint64_t** oz, double** oc, size_t* U,
                     cudaStream_t s);
bool bucket_simplify(int device, int W, const uint64_t* x, const uint64_t* z, const double* c, size_t n,
                     int thr_mode, double atol, double rtol, uint64_t** ox, uint64_t** oz, double** oc, size_t* U,
                     cudaStream_t s);
int sort_algorithm();     // WG_SORT_* setting
void note_sort(int algo);  // records the algorithm of the thread's last result

// ------------------------------------------------------------- autotuner
// Tile shapes and schedules chosen per shape class (wg_tune.cu).  A class is
// (operation, mask words, a, b) with a and b the ceiling log2 of the sizes
// that set the work (e.g. lhs and rhs terms).  In WG_TUNE_SEARCH mode the
// first call of a class without a cached choice runs every candidate on its
// own inputs, times each on its stream with CUDA events (best of two runs),
// synchronising, and caches the fastest; WG_TUNE_CACHED (default) uses cached
// choices and the measured defaults elsewhere; WG_TUNE_OFF always the
// defaults.  Every candidate of an operation produces identical results.
enum TuneOp : int { kTuneCommute = 1, kTuneBucket = 2, kTuneGroupQwc = 3, kTuneGroupFull = 4 };
int tune_mode();
int tune_lookup(int op, int words, int a, int b);  // -1 when the class has no cached choice
void tune_store(int op, int words, int a, int b, int choice);
int tune_candidates(int op);  // number of candidates of an operation
int ceil_log2(size_t n);
// Milliseconds of run() on stream s (CUDA events; synchronises s); run()
// returns false when its candidate cannot serve the inputs (infinite time).
float tune_time(cudaStream_t s, bool (*run)(void*), void* ctx);

// The choice for one call: the class's cached choice, else (search mode, and
// allow_search) the fastest candidate, else `fallback`.  run(c) does the
// call's whole work with candidate c and returns false if c cannot serve it;
// after a search the last candidate's run has produced the call's results
// (all candidates' results are identical), and *done says so.
template <class Run>
int tune_choose(int op, int words, int a, int b, int fallback, bool allow_search, cudaStream_t s, Run&& run,
                bool* done) {
  *done = false;
  const int mode = tune_mode();
  if (mode == WG_TUNE_OFF) return fallback;
  const int cached = tune_lookup(op, words, a, b);
  if (cached >= 0) return cached;
  if (mode != WG_TUNE_SEARCH || !allow_search) return fallback;
  const int n = tune_candidates(op);
  int best = -1;
  float best_ms = 0.0f;
  for (int c = 0; c < n; ++c) {
    struct Ctx {
      std::remove_reference_t<Run>* run;
      int c;
    } ctx{&run, c};
    auto thunk = [](void* p) -> bool {
      auto* k = static_cast<Ctx*>(p);
      return (*k->run)(k->c);
    };
    float ms = tune_time(s, thunk, &ctx);
    const float ms2 = tune_time(s, thunk, &ctx);  // the first run may carry one-time set-up
    if (ms2 < ms) ms = ms2;
    if (ms >= 0.0f && (best < 0 || ms < best_ms)) {
      best = c;
      best_ms = ms;
    }
  }
  if (best < 0) return fallback;
  *done = true;  // the last successful run left the results in place
  tune_store(op, words, a, b, best);
  return best;
}

inline size_t checked_mul(size_t a, size_t b, const char* what) {
  if (a != 0 && b > SIZE_MAX / a) throw_invalid(std::string(what) + " size overflows size_t");
  return a * b;
}

}  // namespace wg

// ============================================================== device helpers
namespace wgd {

struct c128 {
  double re, im;
};

// IEEE operations with explicit round-to-nearest and no contraction, so each
// product or sum rounds once, as in the reference's g++ -O2 build (x86-64
// baseline code generation has no FMA).
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ c128 cadd(c128 a, c128 b) { return {add(a.re, b.re), add(a.im, b.im)}; }

// std::complex<double> multiplication as g++ evaluates it without
// -ffast-math / -fcx-limited-range: (ac - bd, ad + bc), and when both parts are
// NaN the recovery procedure of ISO C Annex G.5.1 (the algorithm libgcc's
// __muldc3 implements) to recover infinities.
__device__ __forceinline__ c128 cmul(c128 z, c128 w) {
  double a = z.re, b = z.im, c = w.re, d = w.im;
  const double ac = mul(a, c), bd = mul(b, d), ad = mul(a, d), bc = mul(b, c);
  double x = sub(ac, bd), y = add(ad, bc);
  if (isnan(x) && isnan(y)) {
    bool recalc = false;
    if (isinf(a) || isinf(b)) {
      a = copysign(isinf(a) ? 1.0 : 0.0, a);
      b = copysign(isinf(b) ? 1.0 : 0.0, b);
      if (isnan(c)) c = copysign(0.0, c);
      if (isnan(d)) d = copysign(0.0, d);
      recalc = true;
    }
    if (isinf(c) || isinf(d)) {
      c = copysign(isinf(c) ? 1.0 : 0.0, c);
      d = copysign(isinf(d) ? 1.0 : 0.0, d);
      if (isnan(a)) a = copysign(0.0, a);
      if (isnan(b)) b = copysign(0.0, b);
      recalc = true;
    }
    if (!recalc && (isinf(ac) || isinf(bd) || isinf(ad) || isinf(bc))) {
      if (isnan(a)) a = copysign(0.0, a);
      if (isnan(b)) b = copysign(0.0, b);
      if (isnan(c)) c = copysign(0.0, c);
      if (isnan(d)) d = copysign(0.0, d);
      recalc = true;
    }
    if (recalc) {
      x = mul(__longlong_as_double(0x7ff0000000000000LL), sub(mul(a, c), mul(b, d)));
      y = mul(__longlong_as_double(0x7ff0000000000000LL), add(mul(a, d), mul(b, c)));
    }
  }
  return {x, y};
}

// Multiplication by i^e (exact sign swaps).
__device__ __forceinline__ c128 rotate(c128 v, unsigned e) {
  switch (e & 3U) {
    case 0: return v;
    case 1: return {-v.im, v.re};
    case 2: return {-v.re, -v.im};
    default: return {v.im, -v.re};
  }
}

// |z| with the rounding of glibc's hypot, which std::abs(std::complex<double>)
// calls in the reference.  The method is the corrected square root of
// C. F. Borges, "An Improved Algorithm for hypot(a,b)" (arXiv:1904.09481), in
// its variant without fused multiply-add, with power-of-two rescaling outside
// [2^-500, 2^500] and the large-ratio shortcut; checked bit-for-bit against the
// host libm across the full exponent range by the test suite.
__device__ __forceinline__ double borges_kernel(double ax, double ay) {
  double h = __dsqrt_rn(add(mul(ax, ax), mul(ay, ay)));
  double t1, t2;
  if (h <= mul(2.0, ay)) {
    const double delta = sub(h, ay);
    t1 = mul(ax, sub(mul(2.0, delta), ax));
    t2 = mul(sub(delta, mul(2.0, sub(ax, ay))), delta);
  } else {
    const double delta = sub(h, ax);
    t1 = mul(mul(2.0, delta), sub(ax, mul(2.0, ay)));
    t2 = add(mul(sub(mul(4.0, delta), ay), ay), mul(delta, delta));
  }
  return sub(h, __ddiv_rn(add(t1, t2), mul(2.0, h)));
}

__device__ __forceinline__ double hypot_ref(double x, double y) {
  if (isinf(x) || isinf(y)) return __longlong_as_double(0x7ff0000000000000LL);
  if (isnan(x) || isnan(y)) return __longlong_as_double(0x7ff8000000000000LL);
  double ax = fabs(x), ay = fabs(y);
  if (ax < ay) {
    const double t = ax;
    ax = ay;
    ay = t;
  }
  if (ay == 0.0) return ax;
  if (ax > mul(ay, 0x1p54)) return add(ax, ay);
  if (ax > 0x1p500) return mul(borges_kernel(mul(ax, 0x1p-600), mul(ay, 0x1p-600)), 0x1p600);
  if (ay < 0x1p-500) return mul(borges_kernel(mul(ax, 0x1p600), mul(ay, 0x1p600)), 0x1p-600);
  return borges_kernel(ax, ay);
}

__device__ __forceinline__ unsigned popc64(uint64_t v) { return __popcll(v); }

// Strict canonical comparison of two keys held as 2*W words in significance
// order (x0, z0, x1, z1, ...).
template <int W>
__device__ __forceinline__ bool key_less(const uint64_t (&a)[2 * W], const uint64_t (&b)[2 * W]) {
#pragma unroll
  for (int i = 0; i < 2 * W; ++i)
    if (a[i] != b[i]) return a[i] < b[i];
  return false;
}

}  // namespace wgd
