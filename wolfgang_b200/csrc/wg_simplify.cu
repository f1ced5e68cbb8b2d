// wg_simplify.cu -- all-pairs Pauli products and simplify (sort, reduce, cull).
//
// Semantics (reference src/simplify.cpp:147-430, src/multiply.cpp:73-402):
//  * product (l, r): x = lx ^ rx, z = lz ^ rz,
//      e = sum_w popc(x&z) - popc(lx&lz) - popc(rx&rz) + 2 popc(lx&rz)  (mod 4),
//      c = (cl * cr) * i^e, with std::complex<double> rounding;
//    products are numbered l*n_r + r (nested-loop order, lhs outer).
//  * simplify: equal keys are summed in input order, kept iff
//    |sum| > atol + rtol*max|c_in| (|.| = glibc hypot), emitted in canonical
//    key order (x0, z0, x1, z1, ... as unsigned words).
//
// Pipeline (all on device, 64-bit sizes, 32-bit item indices):
//  1. keys as structure-of-arrays words K[k][i] in significance order plus
//     item index; for products the keys, indices and coefficients are
//     generated straight into that layout;
//  2. a stable multi-word LSD radix sort (8-bit digits) over only the digits
//     in which some key differs from the first key; stability keeps equal
//     keys in input order, which is the reference's summation order;
//  3. segment heads, then one thread per segment sums its run left to right
//     (the exact reference order and rounding), culls with the reference
//     hypot, and survivors are compacted in sorted order.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "wg_common.cuh"
#include "wg_scan.cuh"

namespace {

using wgd::c128;

constexpr int kThreads = 256;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kTileItems = 4096;                  // items per radix block
constexpr int kRounds = kTileItems / kThreads;    // 16 rounds of 256 items

// ------------------------------------------------------------- key building

// Splits AoS term words into SoA key words: K[2w][i] = x[i*W+w], K[2w+1][i] = z[i*W+w].
__global__ void build_keys_kernel(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z, size_t n,
                                  int W, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    for (int w = 0; w < W; ++w) {
      keys[(2 * w) * n + i] = x[i * W + w];
      keys[(2 * w + 1) * n + i] = z[i * W + w];
    }
    idx[i] = static_cast<uint32_t>(i);
  }
}

// Product generation.  Thread handles products p = l*n_r + r.  When keys is
// non-null it writes SoA sort keys + index; otherwise AoS output terms.
template <int W>
__device__ __forceinline__ void product_term(const uint64_t* __restrict__ lx, const uint64_t* __restrict__ lz,
                                             const double* __restrict__ lc, const uint64_t* __restrict__ rx,
                                             const uint64_t* __restrict__ rz, const double* __restrict__ rc,
                                             size_t l, size_t r, int Wrt, uint64_t* ox, uint64_t* oz, c128& c) {
  const int WW = W > 0 ? W : Wrt;
  unsigned e = 0;
  for (int w = 0; w < WW; ++w) {
    const uint64_t ax = __ldg(lx + l * WW + w), az = __ldg(lz + l * WW + w);
    const uint64_t bx = __ldg(rx + r * WW + w), bz = __ldg(rz + r * WW + w);
    const uint64_t px = ax ^ bx, pz = az ^ bz;
    ox[w] = px;
    oz[w] = pz;
    e += __popcll(px & pz) - __popcll(ax & az) - __popcll(bx & bz) + 2u * __popcll(ax & bz);
  }
  const c128 a{__ldg(lc + 2 * l), __ldg(lc + 2 * l + 1)};
  const c128 b{__ldg(rc + 2 * r), __ldg(rc + 2 * r + 1)};
  c = wgd::rotate(wgd::cmul(a, b), e);
}

template <int W>
__global__ void __launch_bounds__(kThreads) products_kernel(
    const uint64_t* __restrict__ lx, const uint64_t* __restrict__ lz, const double* __restrict__ lc, size_t n_l,
    const uint64_t* __restrict__ rx, const uint64_t* __restrict__ rz, const double* __restrict__ rc, size_t n_r,
    int Wrt, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx, uint64_t* __restrict__ out_x,
    uint64_t* __restrict__ out_z, double* __restrict__ out_c, unsigned long long* __restrict__ max_bits) {
  const size_t P = n_l * n_r;
  const int WW = W > 0 ? W : Wrt;
  double mx = 0.0;
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < P;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t l = p / n_r;
    const size_t r = p - l * n_r;
    c128 c;
    if constexpr (W < 0) {
      // any width: each word's product is stored as soon as it is formed
      unsigned e = 0;
      for (int w = 0; w < WW; ++w) {
        const uint64_t ax = __ldg(lx + l * WW + w), az = __ldg(lz + l * WW + w);
        const uint64_t bx = __ldg(rx + r * WW + w), bz = __ldg(rz + r * WW + w);
        const uint64_t px = ax ^ bx, pz = az ^ bz;
        e += __popcll(px & pz) - __popcll(ax & az) - __popcll(bx & bz) + 2u * __popcll(ax & bz);
        if (keys) {
          keys[(2 * w) * P + p] = px;
          keys[(2 * w + 1) * P + p] = pz;
        } else {
          out_x[p * WW + w] = px;
          out_z[p * WW + w] = pz;
        }
      }
      const c128 a{__ldg(lc + 2 * l), __ldg(lc + 2 * l + 1)};
      const c128 b{__ldg(rc + 2 * r), __ldg(rc + 2 * r + 1)};
      c = wgd::rotate(wgd::cmul(a, b), e);
      if (keys) idx[p] = static_cast<uint32_t>(p);
    } else {
    uint64_t px[W > 0 ? W : 1], pz[W > 0 ? W : 1];
    product_term<W>(lx, lz, lc, rx, rz, rc, l, r, Wrt, px, pz, c);
    if (keys) {
      for (int w = 0; w < WW; ++w) {
        keys[(2 * w) * P + p] = px[w];
        keys[(2 * w + 1) * P + p] = pz[w];
      }
      idx[p] = static_cast<uint32_t>(p);
    } else {
      for (int w = 0; w < WW; ++w) {
        out_x[p * WW + w] = px[w];
        out_z[p * WW + w] = pz[w];
      }
    }
    }
    out_c[2 * p] = c.re;
    out_c[2 * p + 1] = c.im;
    if (max_bits) {
      const double a = wgd::hypot_ref(c.re, c.im);
      if (mx < a) mx = a;  // std::max semantics: a NaN never replaces the running max
    }
  }
  if (max_bits) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, mx, o);
      if (mx < other) mx = other;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(max_bits, static_cast<unsigned long long>(__double_as_longlong(mx)));
  }
}

// max over hypot_ref(c) of an input coefficient array (non-negative doubles
// order like their bit patterns, so an integer atomicMax works).
__global__ void max_abs_kernel(const double* __restrict__ c, size_t n, unsigned long long* __restrict__ max_bits) {
  double mx = 0.0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double a = wgd::hypot_ref(c[2 * i], c[2 * i + 1]);
    if (mx < a) mx = a;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, mx, o);
    if (mx < other) mx = other;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(max_bits, static_cast<unsigned long long>(__double_as_longlong(mx)));
}

// OR over items of (K[k][i] ^ K[k][0]): the bits in which keys differ.
__global__ void key_diff_kernel(const uint64_t* __restrict__ keys, size_t n, int K,
                                unsigned long long* __restrict__ diff) {
  for (int k = 0; k < K; ++k) {
    const uint64_t first = keys[static_cast<size_t>(k) * n];
    uint64_t acc = 0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
      acc |= keys[static_cast<size_t>(k) * n + i] ^ first;
#pragma unroll
    for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicOr(diff + k, static_cast<unsigned long long>(acc));
  }
}

// ------------------------------------------------------------- radix passes

__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const uint64_t* __restrict__ word, size_t n, int shift,
                                                             uint32_t* __restrict__ hist, size_t nblocks) {
  __shared__ uint32_t h[kRadix];
  for (int d = threadIdx.x; d < kRadix; d += kThreads) h[d] = 0;
  __syncthreads();
  const size_t base = static_cast<size_t>(blockIdx.x) * kTileItems;
#pragma unroll 4
  for (int r = 0; r < kRounds; ++r) {
    const size_t i = base + static_cast<size_t>(r) * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(word[i] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kThreads) hist[static_cast<size_t>(d) * nblocks + blockIdx.x] = h[d];
}

// Stable scatter of one tile.  Items are taken in rounds of 256 consecutive
// positions; within a round, lanes with equal digits are ranked with
// __match_any_sync and warps are ordered by a per-digit prefix over warps, so
// the output order of equal digits is the input order.
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(
    const uint64_t* __restrict__ keys_in, uint64_t* __restrict__ keys_out, int K, size_t n,
    const uint32_t* __restrict__ idx_in, uint32_t* __restrict__ idx_out, int word, int shift,
    const uint32_t* __restrict__ offsets, size_t nblocks) {
  __shared__ uint32_t s_base[kRadix];
  __shared__ uint32_t s_cnt[kThreads / 32][kRadix];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kRadix; d += kThreads)
    s_base[d] = offsets[static_cast<size_t>(d) * nblocks + blockIdx.x];
  const size_t base = static_cast<size_t>(blockIdx.x) * kTileItems;
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (int r = 0; r < kRounds; ++r) {
    const size_t i = base + static_cast<size_t>(r) * kThreads + threadIdx.x;
    const bool valid = i < n;
    const uint32_t d = valid ? static_cast<uint32_t>((keys_in[static_cast<size_t>(word) * n + i] >> shift) &
                                                     (kRadix - 1))
                             : 0xffffffffu;
    for (int e = threadIdx.x; e < (kThreads / 32) * kRadix; e += kThreads) (&s_cnt[0][0])[e] = 0;
    __syncthreads();
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t wrank = __popc(peers & lt_mask);
    if (valid && wrank == 0) s_cnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      // thread t owns digit t: exclusive prefix over warps, then advance base
      uint32_t run = s_base[threadIdx.x];
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) {
        const uint32_t c = s_cnt[w][threadIdx.x];
        s_cnt[w][threadIdx.x] = run;
        run += c;
      }
      s_base[threadIdx.x] = run;
    }
    __syncthreads();
    if (valid) {
      const size_t pos = static_cast<size_t>(s_cnt[warp][d]) + wrank;
      for (int k = 0; k < K; ++k) keys_out[static_cast<size_t>(k) * n + pos] = keys_in[static_cast<size_t>(k) * n + i];
      idx_out[pos] = idx_in[i];
    }
    __syncthreads();
  }
}
static_assert(kThreads == kRadix, "radix_scatter_kernel maps one thread per digit");

// ------------------------------------------------------------- reduction

__global__ void seg_head_kernel(const uint64_t* __restrict__ keys, size_t n, int K, uint32_t* __restrict__ flags) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint32_t head = i == 0;
    if (!head)
      for (int k = 0; k < K; ++k)
        if (keys[static_cast<size_t>(k) * n + i] != keys[static_cast<size_t>(k) * n + i - 1]) {
          head = 1;
          break;
        }
    flags[i] = head;
  }
}

__global__ void seg_start_kernel(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ pos, size_t n,
                                 uint32_t* __restrict__ starts) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    if (flags[i]) starts[pos[i]] = static_cast<uint32_t>(i);
}

// One thread per segment: left-to-right sum in input order (the run is sorted
// stably, so idx increases along it), then the cull.
__global__ void seg_reduce_kernel(const uint32_t* __restrict__ starts, size_t nseg, size_t n,
                                  const uint32_t* __restrict__ idx, const double* __restrict__ coeffs, double thr,
                                  double* __restrict__ segsum, uint32_t* __restrict__ keep) {
  for (size_t s = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; s < nseg;
       s += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t b = starts[s];
    const size_t e = (s + 1 < nseg) ? starts[s + 1] : n;
    c128 acc{0.0, 0.0};
    for (size_t p = b; p < e; ++p) {
      const size_t j = idx[p];
      acc = wgd::cadd(acc, c128{coeffs[2 * j], coeffs[2 * j + 1]});
    }
    segsum[2 * s] = acc.re;
    segsum[2 * s + 1] = acc.im;
    keep[s] = wgd::hypot_ref(acc.re, acc.im) > thr;
  }
}

__global__ void write_out_kernel(const uint64_t* __restrict__ keys, size_t n, int W,
                                 const uint32_t* __restrict__ starts, size_t nseg, const uint32_t* __restrict__ keep,
                                 const uint32_t* __restrict__ outpos, const double* __restrict__ segsum,
                                 uint64_t* __restrict__ ox, uint64_t* __restrict__ oz, double* __restrict__ oc) {
  for (size_t s = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; s < nseg;
       s += static_cast<size_t>(gridDim.x) * blockDim.x) {
    if (!keep[s]) continue;
    const size_t o = outpos[s];
    const size_t i = starts[s];
    for (int w = 0; w < W; ++w) {
      ox[o * W + w] = keys[static_cast<size_t>(2 * w) * n + i];
      oz[o * W + w] = keys[static_cast<size_t>(2 * w + 1) * n + i];
    }
    oc[2 * o] = segsum[2 * s];
    oc[2 * o + 1] = segsum[2 * s + 1];
  }
}

// ------------------------------------------------------------- host driver

struct Outputs {
  uint64_t** x;
  uint64_t** z;
  double** c;
  size_t* n;
};

template <typename T>
T read_scalar(const T* dev, cudaStream_t s) {
  T h{};
  wg::check_cuda(cudaMemcpyAsync(&h, dev, sizeof(T), cudaMemcpyDeviceToHost, s), "read back scalar");
  wg::check_cuda(cudaStreamSynchronize(s), "read back scalar");
  return h;
}

}  // namespace

namespace wg {

// Stable LSD radix sort of n items by K SoA key words (word 0 most
// significant) carrying a 32-bit index; only digits in which some key differs
// from the first key are sorted.  keys/idx are replaced by the sorted arrays.
void radix_sort_keys(int device, size_t n, int K, Scratch& keys, Scratch& idx, cudaStream_t s) {
  if (n <= 1 || K == 0) return;
  // bits in which keys differ
  std::vector<unsigned long long> diff(K, 0);
  {
    Scratch d(sizeof(unsigned long long) * K, s);
    check_cuda(cudaMemsetAsync(d.get(), 0, sizeof(unsigned long long) * K, s), "clear key diff");
    WG_TIMED("key_diff_kernel", s,
      key_diff_kernel<<<grid_for(n, kThreads, device, 8), kThreads, 0, s>>>(keys.as<uint64_t>(), n, K,
                                                                            d.as<unsigned long long>()));
    check_launch("launch key diff");
    check_cuda(cudaMemcpyAsync(diff.data(), d.get(), sizeof(unsigned long long) * K, cudaMemcpyDeviceToHost, s),
               "read key diff");
    check_cuda(cudaStreamSynchronize(s), "read key diff");
  }
  // LSD passes, least significant word (k = K-1) first
  const size_t nblocks = (n + kTileItems - 1) / kTileItems;
  if (nblocks > 0x7fffffffu) throw_invalid("sort item count exceeds the launch grid");
  std::vector<std::pair<int, int>> passes;
  for (int k = K - 1; k >= 0; --k)
    for (int sh = 0; sh < 64; sh += kRadixBits)
      if ((diff[k] >> sh) & (kRadix - 1)) passes.emplace_back(k, sh);
  if (passes.empty()) return;
  Scratch keys2(keys.size(), s), idx2(idx.size(), s);
  Scratch hist(sizeof(uint32_t) * kRadix * nblocks, s);
  uint64_t* kin = keys.as<uint64_t>();
  uint64_t* kout = keys2.as<uint64_t>();
  uint32_t* iin = idx.as<uint32_t>();
  uint32_t* iout = idx2.as<uint32_t>();
  for (const auto& [k, sh] : passes) {
    WG_TIMED("radix_hist_kernel", s,
      radix_hist_kernel<<<static_cast<unsigned>(nblocks), kThreads, 0, s>>>(kin + static_cast<size_t>(k) * n, n, sh,
                                                                           hist.as<uint32_t>(), nblocks));
    check_launch("launch radix histogram");
    wgs::exclusive_scan<uint32_t>(hist.as<uint32_t>(), hist.as<uint32_t>(), kRadix * nblocks, nullptr, s);
    WG_TIMED("radix_scatter_kernel", s,
      radix_scatter_kernel<<<static_cast<unsigned>(nblocks), kThreads, 0, s>>>(kin, kout, K, n, iin, iout, k, sh,
                                                                              hist.as<uint32_t>(), nblocks));
    check_launch("launch radix scatter");
    std::swap(kin, kout);
    std::swap(iin, iout);
  }
  if (kin != keys.as<uint64_t>()) {
    std::swap(keys, keys2);
    std::swap(idx, idx2);
  }
}

}  // namespace wg

namespace {

// Sort (keys, idx) of n items by K key words, reduce equal runs of the sorted
// order, cull at thr and write the survivors to freshly allocated outputs.
void sort_reduce(int device, int W, size_t n, wg::Scratch& keys, wg::Scratch& idx, const double* coeffs,
                 double thr, const Outputs& out, cudaStream_t s) {
  const int K = 2 * W;
  wg::radix_sort_keys(device, n, K, keys, idx, s);
  // 3. segments
  wg::Scratch flags(sizeof(uint32_t) * n, s), pos(sizeof(uint32_t) * n, s), cnt(sizeof(uint32_t), s);
  const unsigned g = wg::grid_for(n, kThreads, device, 8);
  WG_TIMED("seg_head_kernel", s,
    seg_head_kernel<<<g, kThreads, 0, s>>>(keys.as<uint64_t>(), n, K, flags.as<uint32_t>()));
  wg::check_launch("launch segment heads");
  wgs::exclusive_scan<uint32_t>(flags.as<uint32_t>(), pos.as<uint32_t>(), n, cnt.as<uint32_t>(), s);
  const size_t nseg = read_scalar(cnt.as<uint32_t>(), s);
  wg::Scratch starts(sizeof(uint32_t) * nseg, s);
  WG_TIMED("seg_start_kernel", s,
    seg_start_kernel<<<g, kThreads, 0, s>>>(flags.as<uint32_t>(), pos.as<uint32_t>(), n, starts.as<uint32_t>()));
  wg::check_launch("launch segment starts");
  flags.release();
  wg::Scratch segsum(sizeof(double) * 2 * nseg, s), keep(sizeof(uint32_t) * nseg, s);
  const unsigned gs = wg::grid_for(nseg, kThreads, device, 8);
  WG_TIMED("seg_reduce_kernel", s,
    seg_reduce_kernel<<<gs, kThreads, 0, s>>>(starts.as<uint32_t>(), nseg, n, idx.as<uint32_t>(), coeffs, thr,
                                              segsum.as<double>(), keep.as<uint32_t>()));
  wg::check_launch("launch segment reduce");
  wgs::exclusive_scan<uint32_t>(keep.as<uint32_t>(), pos.as<uint32_t>(), nseg, cnt.as<uint32_t>(), s);
  const size_t U = read_scalar(cnt.as<uint32_t>(), s);
  *out.n = U;
  *out.x = *out.z = nullptr;
  *out.c = nullptr;
  if (U == 0) return;
  wg::Scratch ox(sizeof(uint64_t) * U * W, s), oz(sizeof(uint64_t) * U * W, s), oc(sizeof(double) * 2 * U, s);
  WG_TIMED("write_out_kernel", s,
    write_out_kernel<<<gs, kThreads, 0, s>>>(keys.as<uint64_t>(), n, W, starts.as<uint32_t>(), nseg,
                                             keep.as<uint32_t>(), pos.as<uint32_t>(), segsum.as<double>(),
                                             ox.as<uint64_t>(), oz.as<uint64_t>(), oc.as<double>()));
  wg::check_launch("launch simplify output");
  wg::check_cuda(cudaStreamSynchronize(s), "synchronize simplify");
  *out.x = static_cast<uint64_t*>(ox.detach());
  *out.z = static_cast<uint64_t*>(oz.detach());
  *out.c = static_cast<double*>(oc.detach());
}

double threshold(double atol, double rtol, unsigned long long max_bits) {
  // atol + rtol * max|c| evaluated exactly as the reference does
  // (src/simplify.cpp:156-160): one product, one sum, no contraction.
  double max_abs;
  std::memcpy(&max_abs, &max_bits, sizeof(max_abs));
  volatile double prod = rtol * max_abs;
  return atol + prod;
}

// Bucketed sort-reduce for 1-2 mask words: chosen by WG_SORT_BUCKET, or by
// WG_SORT_AUTO from 2^20 items on (below that the LSD passes are cheap).
bool use_bucket(int W, size_t n) {
  const int algo = wg::sort_algorithm();
  if (algo == WG_SORT_LSD || W < 1 || W > 2) return false;
  return algo == WG_SORT_BUCKET || n >= (size_t{1} << 20);
}

void validate_tolerances(double atol, double rtol) {
  // src/simplify.cpp:148-150
  if (atol < 0.0 || rtol < 0.0 || !std::isfinite(atol) || !std::isfinite(rtol))
    wg::throw_invalid("simplify tolerances must be non-negative finite values");
}

template <int W>
void launch_products(const uint64_t* lx, const uint64_t* lz, const double* lc, size_t n_l, const uint64_t* rx,
                     const uint64_t* rz, const double* rc, size_t n_r, int Wrt, uint64_t* keys, uint32_t* idx,
                     uint64_t* ox, uint64_t* oz, double* oc, unsigned long long* max_bits, int device,
                     cudaStream_t s) {
  const unsigned g = wg::grid_for(n_l * n_r, kThreads, device, 8);
  WG_TIMED("products_kernel", s,
    products_kernel<W><<<g, kThreads, 0, s>>>(lx, lz, lc, n_l, rx, rz, rc, n_r, Wrt, keys, idx, ox, oz, oc, max_bits));
  wg::check_launch("launch products");
}

void products_dispatch(int W, const uint64_t* lx, const uint64_t* lz, const double* lc, size_t n_l,
                       const uint64_t* rx, const uint64_t* rz, const double* rc, size_t n_r, uint64_t* keys,
                       uint32_t* idx, uint64_t* ox, uint64_t* oz, double* oc, unsigned long long* max_bits,
                       int device, cudaStream_t s) {
  switch (W) {
    case 0: launch_products<0>(lx, lz, lc, n_l, rx, rz, rc, n_r, 0, keys, idx, ox, oz, oc, max_bits, device, s); break;
    case 1: launch_products<1>(lx, lz, lc, n_l, rx, rz, rc, n_r, 1, keys, idx, ox, oz, oc, max_bits, device, s); break;
    case 2: launch_products<2>(lx, lz, lc, n_l, rx, rz, rc, n_r, 2, keys, idx, ox, oz, oc, max_bits, device, s); break;
    default:
      launch_products<-1>(lx, lz, lc, n_l, rx, rz, rc, n_r, W, keys, idx, ox, oz, oc, max_bits, device, s);
  }
}

}  // namespace

extern "C" {

int wg_simplify(int device, size_t words, size_t n_terms, const uint64_t* x, const uint64_t* z,
                const double* coeffs, double atol, double rtol, uint64_t** out_x, uint64_t** out_z,
                double** out_coeffs, size_t* out_terms, wg_stream_t stream) {
  return wg::guarded([&] {
    validate_tolerances(atol, rtol);
    *out_x = *out_z = nullptr;
    *out_coeffs = nullptr;
    *out_terms = 0;
    if (n_terms == 0) return;
    if (n_terms > 0xffffffffull) wg::throw_invalid("simplify supports at most 2^32-1 terms on the device");
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    const int W = static_cast<int>(words);
    if (use_bucket(W, n_terms) &&
        wg::bucket_simplify(device, W, x, z, coeffs, n_terms, rtol > 0.0 ? 1 : 2, atol, rtol, out_x, out_z,
                            out_coeffs, out_terms, s)) {
      wg::note_sort(WG_SORT_BUCKET);
      return;
    }
    wg::note_sort(WG_SORT_LSD);
    wg::Scratch mx(sizeof(unsigned long long), s);
    wg::check_cuda(cudaMemsetAsync(mx.get(), 0, sizeof(unsigned long long), s), "clear max");
    WG_TIMED("max_abs_kernel", s,
      max_abs_kernel<<<wg::grid_for(n_terms, kThreads, device, 8), kThreads, 0, s>>>(coeffs, n_terms,
                                                                                     mx.as<unsigned long long>()));
    wg::check_launch("launch max abs");
    const double thr = threshold(atol, rtol, read_scalar(mx.as<unsigned long long>(), s));
    wg::Scratch keys(sizeof(uint64_t) * std::max<size_t>(1, 2 * words * n_terms), s);
    wg::Scratch idx(sizeof(uint32_t) * n_terms, s);
    WG_TIMED("build_keys_kernel", s,
      build_keys_kernel<<<wg::grid_for(n_terms, kThreads, device, 8), kThreads, 0, s>>>(x, z, n_terms, W,
                                                                                        keys.as<uint64_t>(),
                                                                                        idx.as<uint32_t>()));
    wg::check_launch("launch build keys");
    sort_reduce(device, W, n_terms, keys, idx, coeffs, thr, Outputs{out_x, out_z, out_coeffs, out_terms}, s);
  });
}

int wg_pauli_products(int device, size_t words, const uint64_t* lhs_x, const uint64_t* lhs_z, const double* lhs_c,
                      size_t n_lhs, const uint64_t* rhs_x, const uint64_t* rhs_z, const double* rhs_c,
                      size_t n_rhs, int mode, double atol, double rtol, uint64_t** out_x, uint64_t** out_z,
                      double** out_coeffs, size_t* out_terms, wg_stream_t stream) {
  return wg::guarded([&] {
    if (mode != WG_PRODUCTS_RAW && mode != WG_PRODUCTS_SIMPLIFY && mode != WG_PRODUCTS_FUSED)
      wg::throw_invalid("products mode must be raw, simplify or fused");
    if (mode == WG_PRODUCTS_SIMPLIFY) validate_tolerances(atol, rtol);
    *out_x = *out_z = nullptr;
    *out_coeffs = nullptr;
    *out_terms = 0;
    const size_t P = wg::checked_mul(n_lhs, n_rhs, "matmul intermediate term count");
    if (P == 0) return;
    if (P > 0xffffffffull) wg::throw_invalid("matmul intermediate term count exceeds the device index range (2^32-1)");
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    const int W = static_cast<int>(words);
    if (mode == WG_PRODUCTS_RAW) {
      wg::Scratch ox(sizeof(uint64_t) * P * words, s), oz(sizeof(uint64_t) * P * words, s),
          oc(sizeof(double) * 2 * P, s);
      products_dispatch(W, lhs_x, lhs_z, lhs_c, n_lhs, rhs_x, rhs_z, rhs_c, n_rhs, nullptr, nullptr,
                        ox.as<uint64_t>(), oz.as<uint64_t>(), oc.as<double>(), nullptr, device, s);
      wg::check_cuda(cudaStreamSynchronize(s), "synchronize products");
      *out_x = static_cast<uint64_t*>(ox.detach());
      *out_z = static_cast<uint64_t*>(oz.detach());
      *out_coeffs = static_cast<double*>(oc.detach());
      *out_terms = P;
      return;
    }
    // The fused hash path of the reference culls at a hard-coded 1e-12
    // (src/multiply.cpp:144, :226); simplify() uses atol + rtol*max|c|.
    const int thr_mode = mode == WG_PRODUCTS_FUSED ? 0 : (rtol > 0.0 ? 1 : 2);
    if (use_bucket(W, P) &&
        wg::bucket_products(device, W, lhs_x, lhs_z, lhs_c, n_lhs, rhs_x, rhs_z, rhs_c, n_rhs, thr_mode, atol, rtol,
                            1.0e-12, out_x, out_z, out_coeffs, out_terms, s)) {
      wg::note_sort(WG_SORT_BUCKET);
      return;
    }
    wg::note_sort(WG_SORT_LSD);
    wg::Scratch keys(sizeof(uint64_t) * std::max<size_t>(1, 2 * words * P), s);
    wg::Scratch idx(sizeof(uint32_t) * P, s);
    wg::Scratch pc(sizeof(double) * 2 * P, s);
    wg::Scratch mx(sizeof(unsigned long long), s);
    wg::check_cuda(cudaMemsetAsync(mx.get(), 0, sizeof(unsigned long long), s), "clear max");
    const bool need_max = mode == WG_PRODUCTS_SIMPLIFY;
    products_dispatch(W, lhs_x, lhs_z, lhs_c, n_lhs, rhs_x, rhs_z, rhs_c, n_rhs, keys.as<uint64_t>(),
                      idx.as<uint32_t>(), nullptr, nullptr, pc.as<double>(),
                      need_max ? mx.as<unsigned long long>() : nullptr, device, s);
    const double thr = need_max ? threshold(atol, rtol, read_scalar(mx.as<unsigned long long>(), s)) : 1.0e-12;
    sort_reduce(device, W, P, keys, idx, pc.as<double>(), thr, Outputs{out_x, out_z, out_coeffs, out_terms}, s);
  });
}

}  // extern "C"
