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

// Items of pair p span [item_base[p], item_base[p+1]); item -> (group, chunk).
struct ItemTable {
  const PlanDev* plans;
  const uint64_t* item_base;  // [n_plans + 1]
  const void* const* psis;
  uint32_t n_plans;
  unsigned long long* counter;
};

template <typename Amp>
__global__ void __launch_bounds__(kThreads) expect_forward_kernel(ItemTable tab, uint64_t n_items) {
  __shared__ double red[kThreads / 32][kTermChunk];
  __shared__ uint64_t s_item;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(tab.counter, 1ull);
    __syncthreads();
    const uint64_t item = s_item;
    __syncthreads();
    if (item >= n_items) break;
    // plan lookup (few plans: binary search over item_base)
    uint32_t lo = 0, hi = tab.n_plans;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (tab.item_base[mid] <= item) lo = mid;
      else hi = mid;
    }
    const PlanDev& P = tab.plans[lo];
    const void* psi = tab.psis[lo];
    const uint64_t local = item - tab.item_base[lo];
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
// factor and scattered to original term order.
__global__ void __launch_bounds__(kThreads) expect_finish_terms_kernel(PlanDev P, double* __restrict__ evals) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < P.T; k += gridDim.x * blockDim.x) {
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
    evals[P.torig[k]] = e;
  }
}

__global__ void __launch_bounds__(1024) expect_total_kernel(const double* __restrict__ coeffs,
                                                            const double* __restrict__ evals, uint32_t T,
                                                            double* __restrict__ result) {
  __shared__ double sre[32], sim[32];
  double re = 0.0, im = 0.0;
  for (uint32_t k = threadIdx.x; k < T; k += blockDim.x) {
    re += coeffs[2 * k] * evals[k];
    im += coeffs[2 * k + 1] * evals[k];
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
    const int nw = blockDim.x >> 5;
    re = lane < nw ? sre[lane] : 0.0;
    im = lane < nw ? sim[lane] : 0.0;
    re = warp_sum(re);
    im = warp_sum(im);
    if (lane == 0) {
      result[0] = re;
      result[1] = im;
    }
  }
}

// Output-stationary adjoint: thread owns amplitudes j = tile0 + t + 256 r.
constexpr int kAdjR = 4;
template <typename Amp>
__global__ void __launch_bounds__(kThreads) expect_adjoint_kernel(PlanDev P, const void* psi, double* hpsi) {
  const uint64_t N = uint64_t{1} << P.n;
  const uint64_t tile = static_cast<uint64_t>(kThreads) * kAdjR;
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * tile; t0 < N; t0 += static_cast<uint64_t>(gridDim.x) * tile) {
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

// Forward pass for any number of (plan, psi) pairs in one persistent launch,
// then per-pair finishing kernels and (optionally) the adjoint.
void run_specs(int device, const std::vector<RunSpec>& specs, int dtype, cudaStream_t s) {
  if (dtype != WG_DTYPE_C128 && dtype != WG_DTYPE_C64)
    wg::throw_invalid("psi dtype must be complex64 or complex128");
  const size_t np = specs.size();
  std::vector<PlanDev> plans(np);
  std::vector<uint64_t> base(np + 1, 0);
  std::vector<const void*> psis(np);
  for (size_t i = 0; i < np; ++i) {
    plans[i] = specs[i].plan->dev;
    psis[i] = specs[i].psi;
    base[i + 1] = base[i] + static_cast<uint64_t>(plans[i].G) * plans[i].C;
  }
  const uint64_t n_items = base[np];
  // temporaries per pair for e_k when the caller does not want them
  std::vector<wg::Scratch> evtmp(np);
  std::vector<double*> evals(np);
  for (size_t i = 0; i < np; ++i) {
    if (specs[i].term_values) {
      evals[i] = specs[i].term_values;
    } else {
      evtmp[i].reset(8 * std::max<uint32_t>(1, plans[i].T), s);
      evals[i] = evtmp[i].as<double>();
    }
  }
  if (n_items > 0) {
    const size_t bytes = sizeof(PlanDev) * np + 8 * (np + 1) + sizeof(void*) * np + 8;
    wg::Scratch meta(bytes, s);
    std::vector<unsigned char> host(bytes, 0);
    std::memcpy(host.data(), plans.data(), sizeof(PlanDev) * np);
    std::memcpy(host.data() + sizeof(PlanDev) * np, base.data(), 8 * (np + 1));
    std::memcpy(host.data() + sizeof(PlanDev) * np + 8 * (np + 1), psis.data(), sizeof(void*) * np);
    wg::check_cuda(cudaMemcpyAsync(meta.get(), host.data(), bytes, cudaMemcpyHostToDevice, s), "upload work table");
    auto* mb = static_cast<unsigned char*>(meta.get());
    ItemTable tab;
    tab.plans = reinterpret_cast<const PlanDev*>(mb);
    tab.item_base = reinterpret_cast<const uint64_t*>(mb + sizeof(PlanDev) * np);
    tab.psis = reinterpret_cast<const void* const*>(mb + sizeof(PlanDev) * np + 8 * (np + 1));
    tab.n_plans = static_cast<uint32_t>(np);
    tab.counter = reinterpret_cast<unsigned long long*>(mb + bytes - 8);
    const int sms = wg::device_props(device).sm_count;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(n_items, static_cast<uint64_t>(sms) * 8));
    if (dtype == WG_DTYPE_C128)
      WG_TIMED("expect_forward_kernel", s,
        expect_forward_kernel<double2><<<grid, kThreads, 0, s>>>(tab, n_items));
    else
      WG_TIMED("expect_forward_kernel", s,
        expect_forward_kernel<float2><<<grid, kThreads, 0, s>>>(tab, n_items));
    wg::check_launch("launch expectation forward");
    // keep the table alive until the kernel has run
    wg::check_cuda(cudaStreamSynchronize(s), "expectation forward");
  }
  for (size_t i = 0; i < np; ++i) {
    const PlanDev& P = plans[i];
    if (P.T > 0) {
      const unsigned g = wg::grid_for(P.T, kThreads, device, 4);
      WG_TIMED("expect_finish_terms_kernel", s,
        expect_finish_terms_kernel<<<g, kThreads, 0, s>>>(P, evals[i]));
      wg::check_launch("launch expectation finish");
    }
    if (specs[i].result) {
      if (P.T > 0) {
        WG_TIMED("expect_total_kernel", s,
          expect_total_kernel<<<1, 1024, 0, s>>>(P.coeffs, evals[i], P.T, specs[i].result));
        wg::check_launch("launch expectation total");
      } else {
        wg::check_cuda(cudaMemsetAsync(specs[i].result, 0, 16, s), "clear expectation");
      }
    }
    if (specs[i].hpsi) {
      const uint64_t N = uint64_t{1} << P.n;
      if (P.T == 0) {
        wg::check_cuda(cudaMemsetAsync(specs[i].hpsi, 0, 16 * N, s), "clear H psi");
      } else {
        const uint64_t tiles = (N + kThreads * kAdjR - 1) / (kThreads * kAdjR);
        const unsigned g = static_cast<unsigned>(std::min<uint64_t>(tiles, wg::device_props(device).sm_count * 8ull));
        if (dtype == WG_DTYPE_C128)
          WG_TIMED("expect_adjoint_kernel", s,
            expect_adjoint_kernel<double2><<<g, kThreads, 0, s>>>(P, specs[i].psi, specs[i].hpsi));
        else
          WG_TIMED("expect_adjoint_kernel", s,
            expect_adjoint_kernel<float2><<<g, kThreads, 0, s>>>(P, specs[i].psi, specs[i].hpsi));
        wg::check_launch("launch expectation adjoint");
      }
    }
  }
  // evtmp buffers are released stream-ordered after the kernels that use them
}

}  // namespace

extern "C" {

int wg_expect_plan_create(int device, size_t n_qubits, size_t n_terms, const uint64_t* x, const uint64_t* z,
                          const double* coeffs, wg_expect_plan_t* plan, wg_stream_t stream) {
  return wg::guarded([&] {
    *plan = nullptr;
    if (n_qubits > 63) wg::throw_invalid("expectation_statevector requires num_qubits <= 63");
    wg::DeviceGuard g(device);
    wg_plan_host* p = make_plan(device, n_qubits, n_terms, x, z, coeffs, stream);
    *plan = reinterpret_cast<wg_expect_plan_t>(new wg_expect_plan_s{std::move(*p)});
    delete p;
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
    std::vector<RunSpec> specs(n_pairs);
    for (size_t i = 0; i < n_pairs; ++i) {
      if (!plans[i]) wg::throw_invalid("expectation plan is null");
      if (plans[i]->h.device != device) wg::throw_invalid("expectation plan belongs to another device");
      if (!psis[i]) wg::throw_invalid("CUDA statevector data pointer must be non-null");
      for (size_t j = 0; j < i; ++j)
        if (plans[j] == plans[i]) wg::throw_invalid("a plan may appear at most once per batched launch");
      specs[i] = RunSpec{&plans[i]->h, psis[i], results ? results[i] : nullptr,
                         term_values ? term_values[i] : nullptr, hpsis ? hpsis[i] : nullptr};
    }
    run_specs(device, specs, psi_dtype, stream);
  });
}

}  // extern "C"
