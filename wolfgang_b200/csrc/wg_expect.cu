// wg_expect.cu -- x-grouped statevector expectation, its adjoint, and the
// batched persistent form.
//
// Convention (reference src/expectation.cpp:121-150):
//   P|b> = i^y (-1)^{popc(z&b)} |b^x>,  y = popc(x&z),
//   e_k = <psi|P_k|psi> = sum_b conj(psi[b^x]) i^y (-1)^{popc(z&b)} psi[b]  (real),
//   E = sum_k c_k e_k.
// Terms sharing an x-mask form a group.  For x != 0 the pair (b, b^x) with the
// lowest x bit of b clear gives t = conj(psi[b^x]) psi[b] and, since
// (-1)^{popc(z&(b^x))} = (-1)^{popc(z&b)} (-1)^y,
//   e_k = {2R, -2I, -2R, 2I}[y mod 4],  R = sum s_k(b) Re t,  I = sum s_k(b) Im t,
// over the half basis; so one pass reading every amplitude once serves every
// term of the group.  For x == 0, e_k = sum_b s_k(b) |psi_b|^2.
//
// Adjoint: (H psi)[j] = sum_g psi[j^x_g] F_g(j^x_g),
//   F_g(b) = sum_{k in g} c_k i^{y_k} (-1)^{popc(z_k&b)}  (output-stationary: each
// output amplitude is written once).  dE/dc_k = e_k, dE/dpsi* = H psi.
//
// Work is split into items (plan, group, chunk); a persistent grid pulls items
// from a device counter, so one launch covers any mix of operators and sizes.
// Per-term partial sums are stored per chunk and reduced in a fixed order:
// results are deterministic run to run.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "wg_common.cuh"
#include "wg_scan.cuh"

namespace {

using wgd::c128;

constexpr int kThreads = 256;
constexpr int kTermChunk = 16;            // per-thread term accumulators
constexpr size_t kMaxChunkPairs = 1u << 16;
constexpr uint32_t kDiagFlag = 4;         // ty bit: the term's group has x == 0

// Device-side description of one operator's grouping.
struct PlanDev {
  int n;                   // qubits
  int C;                   // chunks per group
  uint64_t CH;             // pairs per chunk (singles per chunk = 2*CH for x == 0)
  uint32_t G;              // groups
  uint32_t T;              // terms
  const uint64_t* gx;      // [G] group x-mask
  const uint32_t* gstart;  // [G+1] group start in sorted term order
  const uint64_t* tz;      // [T] sorted z-masks
  const uint32_t* ty;      // [T] sorted y mod 4, | kDiagFlag for x == 0
  const double* td;        // [2T] sorted c_k * i^y
  const uint32_t* torig;   // [T] original index of sorted term
  const double* coeffs;    // [2T] original-order coefficients
  double* partial;         // [T*C] per-chunk partial sums (sorted order)
};

struct wg_plan_host {
  int device;
  PlanDev dev;
  wg::Scratch gx, gstart, tz, ty, td, torig, coeffs, partial;
};

}  // namespace

struct wg_expect_plan_s {
  wg_plan_host h;
};

namespace {

__device__ __forceinline__ uint64_t insert_zero(uint64_t h, int p) {
  const uint64_t lo = h & ((uint64_t{1} << p) - 1);
  return ((h >> p) << (p + 1)) | lo;
}

template <typename Amp>
__device__ __forceinline__ c128 load_amp(const void* psi, uint64_t i);

template <>
__device__ __forceinline__ c128 load_amp<double2>(const void* psi, uint64_t i) {
  const double2 v = __ldg(static_cast<const double2*>(psi) + i);
  return {v.x, v.y};
}

template <>
__device__ __forceinline__ c128 load_amp<float2>(const void* psi, uint64_t i) {
  const float2 v = __ldg(static_cast<const float2*>(psi) + i);
  return {static_cast<double>(v.x), static_cast<double>(v.y)};
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Device work tables of one batched launch (kernel parameter, by value).
struct BatchDev {
  const PlanDev* plans;       // [np]
  const uint64_t* item_base;  // [np+1] forward items (group x chunk) per pair
  const uint64_t* term_base;  // [np+1] flat term offsets
  const uint64_t* tile_base;  // [np+1] adjoint tiles (0 for pairs without H psi)
  const void* const* psis;    // [np]
  double* const* evals;       // [np] e_k outputs (original order)
  double* const* results;     // [np] E outputs or null
  double* const* hpsis;       // [np] H psi outputs or null
  unsigned long long* counters;  // [2] forward / adjoint work queues
  uint32_t np;
  uint64_t n_items, n_terms, n_tiles;
};

__device__ __forceinline__ uint32_t find_pair(const uint64_t* base, uint32_t np, uint64_t v) {
  uint32_t lo = 0, hi = np;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (base[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <typename Amp>
__global__ void __launch_bounds__(kThreads) expect_forward_kernel(BatchDev B) {
  __shared__ double red[kThreads / 32][kTermChunk];
  __shared__ uint64_t s_item;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(B.counters, 1ull);
    __syncthreads();
    const uint64_t item = s_item;
    __syncthreads();
    if (item >= B.n_items) break;
    const uint32_t p = find_pair(B.item_base, B.np, item);
    const PlanDev& P = B.plans[p];
    const void* psi = B.psis[p];
    const uint64_t local = item - B.item_base[p];
    const uint32_t g = static_cast<uint32_t>(local / P.C);
    const uint32_t c = static_cast<uint32_t>(local - static_cast<uint64_t>(g) * P.C);
    const uint64_t x = P.gx[g];
    const uint32_t t0 = P.gstart[g], t1 = P.gstart[g + 1];
    const bool diag = x == 0;
    const uint64_t span = diag ? (uint64_t{1} << P.n) : (P.n > 0 ? uint64_t{1} << (P.n - 1) : 1);
    const uint64_t per = diag ? 2 * P.CH : P.CH;
    const uint64_t h0 = static_cast<uint64_t>(c) * per;
    const uint64_t h1 = min(span, h0 + per);
    const int pivot = diag ? 0 : __ffsll(static_cast<long long>(x)) - 1;
    for (uint32_t tc = t0; tc < t1; tc += kTermChunk) {
      const int nk = min(kTermChunk, static_cast<int>(t1 - tc));
      uint64_t zk[kTermChunk];
      bool imag[kTermChunk];
#pragma unroll
      for (int kk = 0; kk < kTermChunk; ++kk) {
        zk[kk] = kk < nk ? P.tz[tc + kk] : 0;
        imag[kk] = kk < nk ? (P.ty[tc + kk] & 1u) : false;
      }
      double acc[kTermChunk];
#pragma unroll
      for (int kk = 0; kk < kTermChunk; ++kk) acc[kk] = 0.0;
      for (uint64_t h = h0 + threadIdx.x; h < h1; h += kThreads) {
        double vre, vim;
        uint64_t b;
        if (diag) {
          b = h;
          const c128 a = load_amp<Amp>(psi, b);
          vre = a.re * a.re + a.im * a.im;
          vim = 0.0;
        } else {
          b = insert_zero(h, pivot);
          const c128 a = load_amp<Amp>(psi, b);
          const c128 q = load_amp<Amp>(psi, b ^ x);
          // t = conj(q) * a
          vre = q.re * a.re + q.im * a.im;
          vim = q.re * a.im - q.im * a.re;
        }
#pragma unroll
        for (int kk = 0; kk < kTermChunk; ++kk) {
          const double v = imag[kk] ? vim : vre;
          acc[kk] += (__popcll(zk[kk] & b) & 1u) ? -v : v;
        }
      }
#pragma unroll
      for (int kk = 0; kk < kTermChunk; ++kk) {
        const double s = warp_sum(acc[kk]);
        if (lane == 0) red[warp][kk] = s;
      }
      __syncthreads();
      if (threadIdx.x < nk) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
        P.partial[static_cast<size_t>(tc + threadIdx.x) * P.C + c] = s;
      }
      __syncthreads();
    }
  }
}

// e_k from the chunk partials (summed in chunk order), scaled by the pairing
// factor and scattered to original term order; flat over every pair's terms.
__global__ void __launch_bounds__(kThreads) expect_finish_terms_kernel(BatchDev B) {
  for (uint64_t f = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; f < B.n_terms;
       f += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t p = find_pair(B.term_base, B.np, f);
    const PlanDev& P = B.plans[p];
    const uint32_t k = static_cast<uint32_t>(f - B.term_base[p]);
    double s = 0.0;
    for (int c = 0; c < P.C; ++c) s += P.partial[static_cast<size_t>(k) * P.C + c];
    const uint32_t ty = P.ty[k];
    double e;
    if (ty & kDiagFlag) {
      e = s;
    } else {
      switch (ty & 3u) {
        case 0: e = 2.0 * s; break;
        case 1: e = -2.0 * s; break;
        case 2: e = -2.0 * s; break;
        default: e = 2.0 * s; break;
      }
    }
    B.evals[p][P.torig[k]] = e;
  }
}

// E_p = sum_k c_k e_k, one block per pair, tree reduction in a fixed order.
__global__ void __launch_bounds__(kThreads) expect_total_kernel(BatchDev B) {
  __shared__ double sre[kThreads / 32], sim[kThreads / 32];
  for (uint32_t p = blockIdx.x; p < B.np; p += gridDim.x) {
    double* out = B.results[p];
    if (!out) continue;
    const PlanDev& P = B.plans[p];
    const double* ev = B.evals[p];
    double re = 0.0, im = 0.0;
    for (uint32_t k = threadIdx.x; k < P.T; k += blockDim.x) {
      re += P.coeffs[2 * k] * ev[k];
      im += P.coeffs[2 * k + 1] * ev[k];
    }
    re = warp_sum(re);
    im = warp_sum(im);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      sre[warp] = re;
      sim[warp] = im;
    }
    __syncthreads();
    if (warp == 0) {
      re = lane < kThreads / 32 ? sre[lane] : 0.0;
      im = lane < kThreads / 32 ? sim[lane] : 0.0;
      re = warp_sum(re);
      im = warp_sum(im);
      if (lane == 0) {
        out[0] = re;
        out[1] = im;
      }
    }
    __syncthreads();
  }
}

// Output-stationary adjoint over all pairs' tiles (persistent work queue):
// thread owns amplitudes j = tile0 + t + 256 r of one pair's H psi.
constexpr int kAdjR = 4;
constexpr uint64_t kAdjTile = static_cast<uint64_t>(kThreads) * kAdjR;

template <typename Amp>
__global__ void __launch_bounds__(kThreads) expect_adjoint_kernel(BatchDev B) {
  __shared__ uint64_t s_item;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(B.counters + 1, 1ull);
    __syncthreads();
    const uint64_t item = s_item;
    __syncthreads();
    if (item >= B.n_tiles) break;
    const uint32_t p = find_pair(B.tile_base, B.np, item);
    const PlanDev& P = B.plans[p];
    const void* psi = B.psis[p];
    double* hpsi = B.hpsis[p];
    const uint64_t N = uint64_t{1} << P.n;
    const uint64_t t0 = (item - B.tile_base[p]) * kAdjTile;
    c128 acc[kAdjR];
#pragma unroll
    for (int r = 0; r < kAdjR; ++r) acc[r] = {0.0, 0.0};
    for (uint32_t g = 0; g < P.G; ++g) {
      const uint64_t x = P.gx[g];
      c128 u[kAdjR], F[kAdjR];
      uint64_t b[kAdjR];
#pragma unroll
      for (int r = 0; r < kAdjR; ++r) {
        const uint64_t j = t0 + threadIdx.x + static_cast<uint64_t>(kThreads) * r;
        b[r] = j ^ x;
        u[r] = j < N ? load_amp<Amp>(psi, b[r]) : c128{0.0, 0.0};
        F[r] = {0.0, 0.0};
      }
      for (uint32_t k = P.gstart[g]; k < P.gstart[g + 1]; ++k) {
        const uint64_t z = P.tz[k];
        const double dre = P.td[2 * k], dim = P.td[2 * k + 1];
#pragma unroll
        for (int r = 0; r < kAdjR; ++r) {
          const bool neg = __popcll(z & b[r]) & 1u;
          F[r].re += neg ? -dre : dre;
          F[r].im += neg ? -dim : dim;
        }
      }
#pragma unroll
      for (int r = 0; r < kAdjR; ++r) {
        acc[r].re += u[r].re * F[r].re - u[r].im * F[r].im;
        acc[r].im += u[r].re * F[r].im + u[r].im * F[r].re;
      }
    }
#pragma unroll
    for (int r = 0; r < kAdjR; ++r) {
      const uint64_t j = t0 + threadIdx.x + static_cast<uint64_t>(kThreads) * r;
      if (j < N) reinterpret_cast<double2*>(hpsi)[j] = make_double2(acc[r].re, acc[r].im);
    }
  }
}

// ------------------------------------------------------------- plan build

// OR of all x and z masks: the kernels index psi[b ^ x], so masks must stay
// below 2^n; the plan rejects anything else before a kernel reads psi.
__global__ void mask_or_kernel(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z, uint32_t T,
                               unsigned long long* __restrict__ out) {
  uint64_t acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) acc |= x[i] | z[i];
#pragma unroll
  for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicOr(out, static_cast<unsigned long long>(acc));
}

__global__ void iota_kernel(uint32_t* __restrict__ v, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

__global__ void plan_group_heads_kernel(const uint64_t* __restrict__ sx, uint32_t T, uint32_t* __restrict__ flags) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x)
    flags[i] = (i == 0 || sx[i] != sx[i - 1]) ? 1u : 0u;
}

__global__ void plan_fill_kernel(const uint64_t* __restrict__ sx, const uint32_t* __restrict__ perm,
                                 const uint32_t* __restrict__ flags, const uint32_t* __restrict__ gpos, uint32_t T,
                                 const uint64_t* __restrict__ z, const double* __restrict__ c, int words,
                                 uint64_t* __restrict__ gx, uint32_t* __restrict__ gstart, uint64_t* __restrict__ tz,
                                 uint32_t* __restrict__ ty, double* __restrict__ td, uint32_t* __restrict__ torig) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
    const uint32_t o = perm[i];
    const uint64_t xm = sx[i];
    const uint64_t zm = words ? z[o] : 0;
    const unsigned y = __popcll(xm & zm) & 3u;
    tz[i] = zm;
    ty[i] = y | (xm == 0 ? kDiagFlag : 0u);
    torig[i] = o;
    const c128 d = wgd::rotate(c128{c[2 * o], c[2 * o + 1]}, y);
    td[2 * i] = d.re;
    td[2 * i + 1] = d.im;
    if (flags[i]) {
      gx[gpos[i]] = xm;
      gstart[gpos[i]] = i;
    }
  }
}

__global__ void plan_refresh_coeffs_kernel(PlanDev P) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.T; i += gridDim.x * blockDim.x) {
    const uint32_t o = P.torig[i];
    const c128 d = wgd::rotate(c128{P.coeffs[2 * o], P.coeffs[2 * o + 1]}, P.ty[i] & 3u);
    const_cast<double*>(P.td)[2 * i] = d.re;
    const_cast<double*>(P.td)[2 * i + 1] = d.im;
  }
}

wg_plan_host* make_plan(int device, size_t n, size_t T, const uint64_t* x, const uint64_t* z, const double* c,
                        cudaStream_t s) {
  if (n > 63) wg::throw_invalid("expectation_statevector requires num_qubits <= 63");
  if (T > 0xffffffffull) wg::throw_invalid("expectation supports at most 2^32-1 terms");
  std::unique_ptr<wg_plan_host> p(new wg_plan_host());
  p->device = device;
  PlanDev& d = p->dev;
  d.n = static_cast<int>(n);
  d.T = static_cast<uint32_t>(T);
  const int words = n == 0 ? 0 : 1;
  const uint64_t half = n > 0 ? (uint64_t{1} << (n - 1)) : 1;
  d.CH = std::min<uint64_t>(half, kMaxChunkPairs);
  d.C = static_cast<int>((half + d.CH - 1) / d.CH);
  p->coeffs.reset(std::max<size_t>(16, 16 * T), s);
  if (T) wg::check_cuda(cudaMemcpyAsync(p->coeffs.get(), c, 16 * T, cudaMemcpyDeviceToDevice, s), "copy coefficients");
  if (T == 0) {
    d.G = 0;
    d.coeffs = p->coeffs.as<double>();
    wg::check_cuda(cudaStreamSynchronize(s), "build plan");
    p->coeffs.rebind(nullptr);
    return p.release();
  }
  // sort terms by x (stable) -> groups
  wg::Scratch keys(8 * T, s), idx(4 * T, s);
  if (words)
    wg::check_cuda(cudaMemcpyAsync(keys.get(), x, 8 * T, cudaMemcpyDeviceToDevice, s), "copy x masks");
  else
    wg::check_cuda(cudaMemsetAsync(keys.get(), 0, 8 * T, s), "clear x masks");
  iota_kernel<<<wg::grid_for(T, kThreads, device, 4), kThreads, 0, s>>>(idx.as<uint32_t>(), d.T);
  wg::check_launch("launch permutation init");
  if (words) {
    wg::Scratch orv(8, s);
    wg::check_cuda(cudaMemsetAsync(orv.get(), 0, 8, s), "clear mask check");
    mask_or_kernel<<<wg::grid_for(T, kThreads, device, 4), kThreads, 0, s>>>(x, z, d.T,
                                                                              orv.as<unsigned long long>());
    wg::check_launch("launch mask check");
    unsigned long long bits = 0;
    wg::check_cuda(cudaMemcpyAsync(&bits, orv.get(), 8, cudaMemcpyDeviceToHost, s), "read mask check");
    wg::check_cuda(cudaStreamSynchronize(s), "read mask check");
    if (n < 64 && (bits >> n) != 0) {
      wg::throw_invalid("Pauli masks set bits at or above num_qubits");
    }
  }
  wg::radix_sort_keys(device, T, 1, keys, idx, s);
  wg::Scratch flags(4 * T, s), gpos(4 * T, s), cnt(4, s);
  const unsigned grid = wg::grid_for(T, kThreads, device, 4);
  plan_group_heads_kernel<<<grid, kThreads, 0, s>>>(keys.as<uint64_t>(), d.T, flags.as<uint32_t>());
  wg::check_launch("launch plan group heads");
  wgs::exclusive_scan<uint32_t>(flags.as<uint32_t>(), gpos.as<uint32_t>(), T, cnt.as<uint32_t>(), s);
  uint32_t G = 0;
  wg::check_cuda(cudaMemcpyAsync(&G, cnt.get(), 4, cudaMemcpyDeviceToHost, s), "read group count");
  wg::check_cuda(cudaStreamSynchronize(s), "read group count");
  d.G = G;
  p->gx.reset(8 * G, s);
  p->gstart.reset(4 * (G + 1), s);
  p->tz.reset(8 * T, s);
  p->ty.reset(4 * T, s);
  p->td.reset(16 * T, s);
  p->torig.reset(4 * T, s);
  p->partial.reset(8 * T * static_cast<size_t>(d.C), s);
  plan_fill_kernel<<<grid, kThreads, 0, s>>>(keys.as<uint64_t>(), idx.as<uint32_t>(), flags.as<uint32_t>(),
                                             gpos.as<uint32_t>(), d.T, z, c, words, p->gx.as<uint64_t>(),
                                             p->gstart.as<uint32_t>(), p->tz.as<uint64_t>(), p->ty.as<uint32_t>(),
                                             p->td.as<double>(), p->torig.as<uint32_t>());
  wg::check_launch("launch plan fill");
  const uint32_t Tv = d.T;
  wg::check_cuda(cudaMemcpyAsync(p->gstart.as<uint32_t>() + G, &Tv, 4, cudaMemcpyHostToDevice, s), "group end");
  wg::check_cuda(cudaStreamSynchronize(s), "build plan");
  d.gx = p->gx.as<uint64_t>();
  d.gstart = p->gstart.as<uint32_t>();
  d.tz = p->tz.as<uint64_t>();
  d.ty = p->ty.as<uint32_t>();
  d.td = p->td.as<double>();
  d.torig = p->torig.as<uint32_t>();
  d.coeffs = p->coeffs.as<double>();
  d.partial = p->partial.as<double>();
  // The plan outlives the caller's stream: release its buffers on the legacy
  // default stream.
  for (wg::Scratch* b : {&p->gx, &p->gstart, &p->tz, &p->ty, &p->td, &p->torig, &p->coeffs, &p->partial})
    b->rebind(nullptr);
  return p.release();
}

struct RunSpec {
  wg_plan_host* plan;
  const void* psi;
  double* result;
  double* term_values;
  double* hpsi;
};

}  // namespace

// A prepared batch: device work tables for fixed (plan, psi, outputs) pairs.
// Running it only enqueues kernels (no host synchronisation, no host copies),
// so a run can be captured in a CUDA graph and replayed.
struct wg_expect_batch_s {
  int device = 0;
  int dtype = WG_DTYPE_C128;
  int sms = 0;
  BatchDev dev{};
  wg::Scratch table;
  std::vector<wg::Scratch> evtmp;
};

namespace {

wg_expect_batch_s* make_batch(int device, const std::vector<RunSpec>& specs, int dtype, cudaStream_t s) {
  if (dtype != WG_DTYPE_C128 && dtype != WG_DTYPE_C64) wg::throw_invalid("psi dtype must be complex64 or complex128");
  std::unique_ptr<wg_expect_batch_s> b(new wg_expect_batch_s());
  b->device = device;
  b->dtype = dtype;
  b->sms = wg::device_props(device).sm_count;
  const size_t np = specs.size();
  if (np > 0xffffffffull) wg::throw_invalid("too many pairs in one batch");
  std::vector<PlanDev> plans(np);
  std::vector<uint64_t> item_base(np + 1, 0), term_base(np + 1, 0), tile_base(np + 1, 0);
  std::vector<const void*> psis(np);
  std::vector<double*> evals(np), results(np), hpsis(np);
  b->evtmp.resize(np);
  for (size_t i = 0; i < np; ++i) {
    const PlanDev& P = specs[i].plan->dev;
    plans[i] = P;
    psis[i] = specs[i].psi;
    item_base[i + 1] = item_base[i] + static_cast<uint64_t>(P.G) * P.C;
    term_base[i + 1] = term_base[i] + P.T;
    const uint64_t N = uint64_t{1} << P.n;
    const bool adj = specs[i].hpsi != nullptr;
    tile_base[i + 1] = tile_base[i] + (adj ? (N + kAdjTile - 1) / kAdjTile : 0);
    if (specs[i].term_values) {
      evals[i] = specs[i].term_values;
    } else {
      b->evtmp[i].reset(8 * std::max<uint32_t>(1, P.T), s);
      b->evtmp[i].rebind(nullptr);
      evals[i] = b->evtmp[i].as<double>();
    }
    results[i] = specs[i].result;
    hpsis[i] = specs[i].hpsi;
  }
  // one device block: plans | item_base | term_base | tile_base | psis | evals | results | hpsis | counters
  const size_t bytes = sizeof(PlanDev) * np + 8 * 3 * (np + 1) + 8 * 4 * np + 16;
  std::vector<unsigned char> host(bytes, 0);
  size_t off = 0;
  auto put = [&](const void* src, size_t n) {
    std::memcpy(host.data() + off, src, n);
    const size_t at = off;
    off += n;
    return at;
  };
  const size_t o_plans = put(plans.data(), sizeof(PlanDev) * np);
  const size_t o_item = put(item_base.data(), 8 * (np + 1));
  const size_t o_term = put(term_base.data(), 8 * (np + 1));
  const size_t o_tile = put(tile_base.data(), 8 * (np + 1));
  const size_t o_psis = put(psis.data(), 8 * np);
  const size_t o_evals = put(evals.data(), 8 * np);
  const size_t o_res = put(results.data(), 8 * np);
  const size_t o_hpsi = put(hpsis.data(), 8 * np);
  const size_t o_cnt = off;
  b->table.reset(bytes, s);
  b->table.rebind(nullptr);
  // pageable source: the call returns once the bytes are staged
  wg::check_cuda(cudaMemcpyAsync(b->table.get(), host.data(), bytes, cudaMemcpyHostToDevice, s), "upload work table");
  auto* base = static_cast<unsigned char*>(b->table.get());
  BatchDev& d = b->dev;
  d.plans = reinterpret_cast<const PlanDev*>(base + o_plans);
  d.item_base = reinterpret_cast<const uint64_t*>(base + o_item);
  d.term_base = reinterpret_cast<const uint64_t*>(base + o_term);
  d.tile_base = reinterpret_cast<const uint64_t*>(base + o_tile);
  d.psis = reinterpret_cast<const void* const*>(base + o_psis);
  d.evals = reinterpret_cast<double* const*>(base + o_evals);
  d.results = reinterpret_cast<double* const*>(base + o_res);
  d.hpsis = reinterpret_cast<double* const*>(base + o_hpsi);
  d.counters = reinterpret_cast<unsigned long long*>(base + o_cnt);
  d.np = static_cast<uint32_t>(np);
  d.n_items = item_base[np];
  d.n_terms = term_base[np];
  d.n_tiles = tile_base[np];
  return b.release();
}

// Enqueues forward, finish, totals and adjoint; no host synchronisation.
void run_batch(const wg_expect_batch_s& b, cudaStream_t s) {
  const BatchDev& d = b.dev;
  if (d.np == 0) return;
  wg::check_cuda(cudaMemsetAsync(d.counters, 0, 16, s), "reset work queues");
  const unsigned persistent = static_cast<unsigned>(b.sms) * 8;
  if (d.n_items) {
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(d.n_items, persistent));
    if (b.dtype == WG_DTYPE_C128)
      WG_TIMED("expect_forward_kernel", s, expect_forward_kernel<double2><<<grid, kThreads, 0, s>>>(d));
    else
      WG_TIMED("expect_forward_kernel", s, expect_forward_kernel<float2><<<grid, kThreads, 0, s>>>(d));
    wg::check_launch("launch expectation forward");
  }
  if (d.n_terms) {
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((d.n_terms + kThreads - 1) / kThreads, persistent));
    WG_TIMED("expect_finish_terms_kernel", s, expect_finish_terms_kernel<<<grid, kThreads, 0, s>>>(d));
    wg::check_launch("launch expectation finish");
  }
  WG_TIMED("expect_total_kernel", s,
           expect_total_kernel<<<std::min<uint32_t>(d.np, 65535u), kThreads, 0, s>>>(d));
  wg::check_launch("launch expectation total");
  if (d.n_tiles) {
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(d.n_tiles, persistent));
    if (b.dtype == WG_DTYPE_C128)
      WG_TIMED("expect_adjoint_kernel", s, expect_adjoint_kernel<double2><<<grid, kThreads, 0, s>>>(d));
    else
      WG_TIMED("expect_adjoint_kernel", s, expect_adjoint_kernel<float2><<<grid, kThreads, 0, s>>>(d));
    wg::check_launch("launch expectation adjoint");
  }
}

// Pairs whose operator has no terms: E = 0, e = {}, H psi = 0.
void clear_empty(const std::vector<RunSpec>& specs, cudaStream_t s) {
  for (const RunSpec& r : specs) {
    if (r.plan->dev.T != 0) continue;
    if (r.result) wg::check_cuda(cudaMemsetAsync(r.result, 0, 16, s), "clear expectation");
    if (r.hpsi) wg::check_cuda(cudaMemsetAsync(r.hpsi, 0, 16ull << r.plan->dev.n, s), "clear H psi");
  }
}

void run_specs(int device, const std::vector<RunSpec>& specs, int dtype, cudaStream_t s) {
  std::unique_ptr<wg_expect_batch_s> b(make_batch(device, specs, dtype, s));
  clear_empty(specs, s);
  run_batch(*b, s);
  // stream-ordered release after the kernels that read the tables
  b->table.rebind(s);
  for (auto& e : b->evtmp) e.rebind(s);
}

std::vector<RunSpec> batch_specs(int device, size_t n_pairs, const wg_expect_plan_t* plans, const void* const* psis,
                                 double* const* results, double* const* term_values, double* const* hpsis) {
  std::vector<RunSpec> specs(n_pairs);
  for (size_t i = 0; i < n_pairs; ++i) {
    if (!plans[i]) wg::throw_invalid("expectation plan is null");
    if (plans[i]->h.device != device) wg::throw_invalid("expectation plan belongs to another device");
    if (!psis[i]) wg::throw_invalid("CUDA statevector data pointer must be non-null");
    for (size_t j = 0; j < i; ++j)
      if (plans[j] == plans[i]) wg::throw_invalid("a plan may appear at most once per batched launch");
    specs[i] = RunSpec{&plans[i]->h, psis[i], results ? results[i] : nullptr, term_values ? term_values[i] : nullptr,
                       hpsis ? hpsis[i] : nullptr};
  }
  return specs;
}

}  // namespace

extern "C" {

int wg_expect_plan_create(int device, size_t n_qubits, size_t n_terms, const uint64_t* x, const uint64_t* z,
                          const double* coeffs, wg_expect_plan_t* plan, wg_stream_t stream) {
  return wg::guarded([&] {
    *plan = nullptr;
    if (n_qubits > 63) wg::throw_invalid("expectation_statevector requires num_qubits <= 63");
    wg::DeviceGuard g(device);
    std::unique_ptr<wg_plan_host> p(make_plan(device, n_qubits, n_terms, x, z, coeffs, stream));
    *plan = reinterpret_cast<wg_expect_plan_t>(new wg_expect_plan_s{std::move(*p)});
  });
}

int wg_expect_plan_destroy(wg_expect_plan_t plan) {
  return wg::guarded([&] {
    if (!plan) return;
    wg::DeviceGuard g(plan->h.device);
    delete plan;
  });
}

int wg_expect_plan_set_coeffs(wg_expect_plan_t plan, const double* coeffs, wg_stream_t stream) {
  return wg::guarded([&] {
    if (!plan) wg::throw_invalid("expectation plan is null");
    wg::DeviceGuard g(plan->h.device);
    const PlanDev& P = plan->h.dev;
    if (P.T == 0) return;
    wg::check_cuda(cudaMemcpyAsync(plan->h.coeffs.get(), coeffs, 16ull * P.T, cudaMemcpyDeviceToDevice, stream),
                   "copy coefficients");
    plan_refresh_coeffs_kernel<<<wg::grid_for(P.T, kThreads, plan->h.device, 4), kThreads, 0, stream>>>(P);
    wg::check_launch("launch coefficient refresh");
  });
}

int wg_expect_plan_info(wg_expect_plan_t plan, size_t* n_groups, size_t* n_terms) {
  return wg::guarded([&] {
    if (!plan) wg::throw_invalid("expectation plan is null");
    *n_groups = plan->h.dev.G;
    *n_terms = plan->h.dev.T;
  });
}

int wg_expect_plan_run(wg_expect_plan_t plan, const void* psi, int psi_dtype, double* result, double* term_values,
                       double* hpsi, wg_stream_t stream) {
  return wg::guarded([&] {
    if (!plan) wg::throw_invalid("expectation plan is null");
    if (!psi) wg::throw_invalid("CUDA statevector data pointer must be non-null");
    wg::DeviceGuard g(plan->h.device);
    run_specs(plan->h.device, {RunSpec{&plan->h, psi, result, term_values, hpsi}}, psi_dtype, stream);
  });
}

int wg_expectation(int device, size_t n_qubits, size_t n_terms, const uint64_t* x, const uint64_t* z,
                   const double* coeffs, const void* psi, int psi_dtype, double* result_host, wg_stream_t stream) {
  return wg::guarded([&] {
    if (n_qubits > 63) wg::throw_invalid("expectation_statevector requires num_qubits <= 63");
    if (psi_dtype != WG_DTYPE_C128 && psi_dtype != WG_DTYPE_C64)
      wg::throw_invalid("psi dtype must be complex64 or complex128");
    result_host[0] = result_host[1] = 0.0;
    if (n_terms == 0) return;
    if (!psi) wg::throw_invalid("CUDA statevector data pointer must be non-null");
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    std::unique_ptr<wg_plan_host> p(make_plan(device, n_qubits, n_terms, x, z, coeffs, s));
    wg::Scratch res(16, s);
    run_specs(device, {RunSpec{p.get(), psi, res.as<double>(), nullptr, nullptr}}, psi_dtype, s);
    wg::check_cuda(cudaMemcpyAsync(result_host, res.get(), 16, cudaMemcpyDeviceToHost, s), "read expectation");
    wg::check_cuda(cudaStreamSynchronize(s), "read expectation");
  });
}

int wg_expect_batched(int device, size_t n_pairs, const wg_expect_plan_t* plans, const void* const* psis,
                      int psi_dtype, double* const* results, double* const* term_values, double* const* hpsis,
                      wg_stream_t stream) {
  return wg::guarded([&] {
    if (n_pairs == 0) return;
    wg::DeviceGuard g(device);
    run_specs(device, batch_specs(device, n_pairs, plans, psis, results, term_values, hpsis), psi_dtype, stream);
  });
}

int wg_expect_batch_create(int device, size_t n_pairs, const wg_expect_plan_t* plans, const void* const* psis,
                           int psi_dtype, double* const* results, double* const* term_values,
                           double* const* hpsis, wg_expect_batch_t* batch, wg_stream_t stream) {
  return wg::guarded([&] {
    *batch = nullptr;
    wg::DeviceGuard g(device);
    const auto specs = batch_specs(device, n_pairs, plans, psis, results, term_values, hpsis);
    for (const RunSpec& r : specs)
      if (r.plan->dev.T == 0) wg::throw_invalid("a prepared batch needs operators with at least one term");
    *batch = make_batch(device, specs, psi_dtype, stream);
    wg::check_cuda(cudaStreamSynchronize(stream), "prepare batch");
  });
}

int wg_expect_batch_run(wg_expect_batch_t batch, wg_stream_t stream) {
  return wg::guarded([&] {
    if (!batch) wg::throw_invalid("expectation batch is null");
    wg::DeviceGuard g(batch->device);
    run_batch(*batch, stream);
  });
}

int wg_expect_batch_destroy(wg_expect_batch_t batch) {
  return wg::guarded([&] {
    if (!batch) return;
    wg::DeviceGuard g(batch->device);
    delete batch;
  });
}

}  // extern "C"
