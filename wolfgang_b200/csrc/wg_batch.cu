// wg_batch.cu -- prepared batches of Pauli products: many lhs_p * rhs_p pairs
// of uneven sizes, simplified, in one capturable sequence of launches.
//
// Every pair's result is PauliSum::matmul(simplify) of the reference
// (src/multiply.cpp:73-402, src/simplify.cpp:147-430): products (l, r) in
// nested-loop order, equal keys summed left to right in that order, culled at
// |sum| > thr, emitted in canonical key order.  What a product's key and
// phase are depends only on the operands' masks, so the batch splits the work
// the way a sparse factorisation splits symbolic from numeric work:
//
//  create (symbolic, once): every product of every pair gets the key
//    (pair, x0, z0, ..., x_{W-1}, z_{W-1}); one stable LSD radix sort over all
//    pairs' products groups equal keys of a pair, in nested-loop order; each
//    sorted product keeps its pair-local index and phase (one 32-bit code),
//    each run of equal keys (a segment) its start, pair and key.  All scratch
//    of the numeric pass and the outputs (one slot per segment) are sized here.
//  run (numeric, any number of times): one thread per segment forms its
//    products' coefficients from the operands' current coefficient buffers and
//    sums them in order; the cull threshold per pair (atol + rtol*max|c| over
//    the pair's products, or the fused path's 1e-12); a scan of the survivors
//    and their write-out in canonical order.  No allocation, no host copy, no
//    host synchronisation: a run can be captured in a CUDA graph and replayed
//    after the coefficients change.
//
// Sizes: each pair has at most 2^30 products (index and phase share 32 bits)
// and the batch fewer than 2^32 products in all.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "wg_common.cuh"
#include "wg_scan.cuh"

namespace {

using wgd::c128;

constexpr int kThreads = 256;

// Operand masks of one pair (create only).
struct PairMasks {
  const uint64_t* lx;
  const uint64_t* lz;
  const uint64_t* rx;
  const uint64_t* rz;
  uint64_t n_r;
  uint64_t item_base;  // first product of the pair in the batch
};

// What a run needs of one pair.  q / n_r is computed as the high word of
// q * div_m (div_m = floor((2^64 - 1) / n_r) + 1, exact for q, n_r < 2^32;
// n_r = 1 divides trivially).
struct PairNum {
  const double* lc;
  const double* rc;
  uint64_t n_r;
  uint64_t div_m;
  uint64_t seg_base;  // first segment of the pair = first output slot
  uint64_t n_seg;
};

// How a run forms each pair's largest |product| (the rtol threshold):
enum MaxMode : int {
  kMaxNone = 0,  // fused mode: fixed threshold
  kMaxInf = 1,   // rtol == 0: atol + 0 * max is atol unless some |product| is infinite
  kMaxFull = 2,  // rtol > 0: the maximum itself
};

// ------------------------------------------------------------- symbolic pass

// Keys of every product: word 0 = pair, then the canonical key words (SoA);
// code = pair-local product index << 2 | phase exponent (mod 4).
__global__ void pbatch_keys_kernel(const PairMasks* __restrict__ pairs, const uint64_t* __restrict__ item_base,
                                   uint32_t n_pairs, size_t N, int W, uint64_t* __restrict__ keys,
                                   uint32_t* __restrict__ idx, uint32_t* __restrict__ code) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < N;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    // the last pair whose first product is at or before i (empty pairs share bases)
    uint32_t lo = 0, hi = n_pairs;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (item_base[mid] <= i) lo = mid;
      else hi = mid;
    }
    const PairMasks P = pairs[lo];
    const uint64_t q = i - P.item_base;
    const uint64_t l = q / P.n_r, r = q - l * P.n_r;
    keys[i] = lo;
    unsigned e = 0;
    for (int w = 0; w < W; ++w) {
      const uint64_t ax = P.lx[l * W + w], az = P.lz[l * W + w];
      const uint64_t bx = P.rx[r * W + w], bz = P.rz[r * W + w];
      const uint64_t px = ax ^ bx, pz = az ^ bz;
      keys[static_cast<size_t>(1 + 2 * w) * N + i] = px;
      keys[static_cast<size_t>(2 + 2 * w) * N + i] = pz;
      e += __popcll(px & pz) - __popcll(ax & az) - __popcll(bx & bz) + 2u * __popcll(ax & bz);
    }
    code[i] = static_cast<uint32_t>(q << 2) | (e & 3u);
    idx[i] = static_cast<uint32_t>(i);
  }
}

__global__ void pbatch_gather_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ in, size_t N,
                                     uint32_t* __restrict__ out) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < N;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[i] = in[idx[i]];
}

__global__ void pbatch_head_kernel(const uint64_t* __restrict__ keys, size_t N, int K, uint32_t* __restrict__ flags) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < N;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint32_t head = i == 0;
    for (int k = 0; k < K && !head; ++k)
      head = keys[static_cast<size_t>(k) * N + i] != keys[static_cast<size_t>(k) * N + i - 1];
    flags[i] = head;
  }
}

// Per segment: start, pair and key (AoS, x words then z words).
__global__ void pbatch_segments_kernel(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ segid,
                                       const uint64_t* __restrict__ keys, size_t N, int W,
                                       uint32_t* __restrict__ seg_start, uint32_t* __restrict__ seg_pair,
                                       uint64_t* __restrict__ seg_keys) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < N;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    if (!flags[i]) continue;
    const size_t s = segid[i];
    seg_start[s] = static_cast<uint32_t>(i);
    seg_pair[s] = static_cast<uint32_t>(keys[i]);
    for (int w = 0; w < W; ++w) {
      seg_keys[s * (2 * W) + w] = keys[static_cast<size_t>(1 + 2 * w) * N + i];
      seg_keys[s * (2 * W) + W + w] = keys[static_cast<size_t>(2 + 2 * w) * N + i];
    }
  }
}

// Segments per pair (segments of a pair are contiguous: one atomic per
// warp-run of equal pairs).
__global__ void pbatch_count_kernel(const uint32_t* __restrict__ seg_pair, size_t S, unsigned* __restrict__ cnt) {
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t base = static_cast<size_t>(blockIdx.x) * blockDim.x; base < S; base += stride) {
    const size_t s = base + threadIdx.x;
    const uint32_t p = s < S ? seg_pair[s] : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, p);
    if (s < S && (threadIdx.x & 31) == static_cast<unsigned>(__ffs(peers) - 1)) atomicAdd(cnt + p, __popc(peers));
  }
}

// ------------------------------------------------------------- numeric pass

// The magnitude of a product, out of line: kMaxInf needs it only for the rare
// product with a part beyond 2^1022 or not finite.
__device__ __noinline__ double product_magnitude(double re, double im) { return wgd::hypot_ref(re, im); }

// One thread per segment (a warp takes 32 consecutive segments): the
// segment's products formed from the current coefficients and summed left to
// right (FP64, no FMA: the reference's rounding); in SIMPLIFY mode the
// largest |product| of each pair, for the rtol threshold (non-negative
// doubles order like their bits; a NaN never replaces the running maximum,
// std::max's rule) -- with rtol = 0 only the magnitudes that may be infinite
// (a part beyond 2^1022 or not finite) are formed, since a finite maximum
// leaves the threshold at atol.  want_max is a MaxMode.
template <int want_max>
__global__ void __launch_bounds__(kThreads) pbatch_sums_kernel(
    const PairNum* __restrict__ pairs, const uint32_t* __restrict__ seg_start, const uint32_t* __restrict__ seg_pair,
    const uint32_t* __restrict__ code, size_t S, double* __restrict__ segsum,
    unsigned long long* __restrict__ pair_max) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5;
  const size_t nwarps = (static_cast<size_t>(gridDim.x) * blockDim.x) >> 5;
  for (size_t chunk = warp; chunk * 32 < S; chunk += nwarps) {
    const size_t s = chunk * 32 + lane;
    const bool valid = s < S;
    const uint32_t p = valid ? seg_pair[s] : 0xffffffffu;
    double mx = 0.0;
    if (valid) {
      const PairNum P = pairs[p];
      const uint32_t b = seg_start[s], e = seg_start[s + 1];
      const uint32_t nr = static_cast<uint32_t>(P.n_r);  // below 2^30
      c128 acc{0.0, 0.0};
      for (uint32_t j = b; j < e; ++j) {
        const uint32_t cj = __ldg(code + j);
        const uint32_t q = cj >> 2;
        const uint32_t l = nr == 1 ? q : static_cast<uint32_t>(__umul64hi(static_cast<uint64_t>(q), P.div_m));
        const uint32_t r = q - l * nr;
        const double2 av = __ldg(reinterpret_cast<const double2*>(P.lc) + l);
        const double2 bv = __ldg(reinterpret_cast<const double2*>(P.rc) + r);
        const c128 prod = wgd::rotate(wgd::cmul(c128{av.x, av.y}, c128{bv.x, bv.y}), cj & 3u);
        acc = wgd::cadd(acc, prod);
        if (want_max == kMaxFull) {
          const double m = wgd::hypot_ref(prod.re, prod.im);
          if (mx < m) mx = m;
        } else if (want_max == kMaxInf && !(fabs(prod.re) <= 0x1p1022 && fabs(prod.im) <= 0x1p1022)) {
          const double m = product_magnitude(prod.re, prod.im);
          if (mx < m) mx = m;
        }
      }
      segsum[2 * s] = acc.re;
      segsum[2 * s + 1] = acc.im;
    }
    if (want_max) {
      const uint32_t p0 = __shfl_sync(0xffffffffu, p, 0);
      if (__all_sync(0xffffffffu, p == p0 || !valid)) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          const double other = __shfl_xor_sync(0xffffffffu, mx, o);
          if (mx < other) mx = other;
        }
        if (lane == 0 && mx > 0.0) atomicMax(pair_max + p0, static_cast<unsigned long long>(__double_as_longlong(mx)));
      } else if (valid && mx > 0.0) {
        atomicMax(pair_max + p, static_cast<unsigned long long>(__double_as_longlong(mx)));
      }
    }
  }
}

// keep[s] = |sum| > threshold of the segment's pair (|.| = glibc's hypot).
__global__ void pbatch_keep_kernel(const uint32_t* __restrict__ seg_pair, const double* __restrict__ segsum, size_t S,
                                   int fused, double atol, double rtol, const unsigned long long* __restrict__ pair_max,
                                   uint32_t* __restrict__ keep) {
  for (size_t s = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; s < S;
       s += static_cast<size_t>(gridDim.x) * blockDim.x) {
    double thr = 1.0e-12;  // the fused path's fixed cull (src/multiply.cpp:144, :226)
    if (!fused) {
      // atol + rtol * max|c| with one rounding each (src/simplify.cpp:156-160)
      const double mx = __longlong_as_double(static_cast<long long>(pair_max[seg_pair[s]]));
      thr = __dadd_rn(atol, __dmul_rn(rtol, mx));
    }
    // without NaNs the rounded |s| is never below max(|re|, |im|): most sums are
    // decided without the full hypot
    const double re = segsum[2 * s], im = segsum[2 * s + 1];
    const bool plain = !isnan(re) && !isnan(im);
    keep[s] = (plain && (fabs(re) > thr || fabs(im) > thr)) || wgd::hypot_ref(re, im) > thr;
  }
}

// Survivor s of pair p goes to output slot seg_base[p] + its rank in the pair.
// WT = W for 1 or 2 mask words (16-byte loads and stores), 0 for any width.
template <int WT>
__global__ void pbatch_write_kernel(const PairNum* __restrict__ pairs, const uint32_t* __restrict__ seg_pair,
                                    const uint64_t* __restrict__ seg_keys, const double* __restrict__ segsum,
                                    const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos, size_t S,
                                    int Wrt, uint64_t* __restrict__ ox, uint64_t* __restrict__ oz,
                                    double* __restrict__ oc) {
  const int W = WT > 0 ? WT : Wrt;
  for (size_t s = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; s < S;
       s += static_cast<size_t>(gridDim.x) * blockDim.x) {
    if (!keep[s]) continue;
    const uint64_t base = pairs[seg_pair[s]].seg_base;
    const size_t o = base + (pos[s] - pos[base]);
    const double2 c = reinterpret_cast<const double2*>(segsum)[s];
    if constexpr (WT == 1) {
      const ulonglong2 k = reinterpret_cast<const ulonglong2*>(seg_keys)[s];
      ox[o] = k.x;
      oz[o] = k.y;
    } else if constexpr (WT == 2) {
      const ulonglong2 kx = reinterpret_cast<const ulonglong2*>(seg_keys)[2 * s];
      const ulonglong2 kz = reinterpret_cast<const ulonglong2*>(seg_keys)[2 * s + 1];
      reinterpret_cast<ulonglong2*>(ox)[o] = kx;
      reinterpret_cast<ulonglong2*>(oz)[o] = kz;
    } else {
      for (int w = 0; w < W; ++w) {
        ox[o * W + w] = seg_keys[s * (2 * W) + w];
        oz[o * W + w] = seg_keys[s * (2 * W) + W + w];
      }
    }
    reinterpret_cast<double2*>(oc)[o] = c;
  }
}

__global__ void pbatch_counts_kernel(const PairNum* __restrict__ pairs, const uint32_t* __restrict__ pos,
                                     size_t n_pairs, uint64_t* __restrict__ counts) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n_pairs;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const PairNum P = pairs[p];
    counts[p] = pos[P.seg_base + P.n_seg] - pos[P.seg_base];
  }
}

}  // namespace

// Allocations of a batch come from the device pool on the legacy default
// stream; create ends with a device synchronisation, so they are complete
// before any stream uses them, and destroy synchronises the device first.
struct wg_products_batch_s {
  int device = 0;
  int W = 0;
  int mode = WG_PRODUCTS_SIMPLIFY;
  double atol = 0.0, rtol = 0.0;
  size_t n_pairs = 0, N = 0, S = 0;
  unsigned sum_blocks = 0;  // grid of the segment-sum kernel
  std::vector<uint64_t> seg_base, n_seg;
  wg::Scratch pairs;            // PairNum[n_pairs]
  wg::Scratch code;             // uint32[N]: sorted products' index << 2 | phase
  wg::Scratch seg_start;        // uint32[S + 1]
  wg::Scratch seg_pair;         // uint32[S]
  wg::Scratch seg_keys;         // uint64[S][2W]
  wg::Scratch segsum, keep, pos, scan_ws, pair_max;
  wg::Scratch out_x, out_z, out_c, counts;
};

namespace {

void build_batch(wg_products_batch_s& b, const uint64_t* const* lhs_x, const uint64_t* const* lhs_z,
                 const double* const* lhs_c, const size_t* n_lhs, const uint64_t* const* rhs_x,
                 const uint64_t* const* rhs_z, const double* const* rhs_c, const size_t* n_rhs) {
  const int device = b.device;
  const int W = b.W;
  const size_t np = b.n_pairs;
  cudaStream_t s = nullptr;  // see the note above wg_products_batch_s
  std::vector<PairMasks> masks(np);
  std::vector<PairNum> nums(np);
  std::vector<uint64_t> item_base(np + 1, 0);
  for (size_t p = 0; p < np; ++p) {
    const size_t P = wg::checked_mul(n_lhs[p], n_rhs[p], "matmul intermediate term count");
    if (P > (size_t{1} << 30))
      wg::throw_invalid("a product batch takes at most 2^30 products per pair (pair " + std::to_string(p) +
                        " has " + std::to_string(P) + "); use wg_pauli_products for it");
    if (P > 0) {
      if (!lhs_c[p] || !rhs_c[p]) wg::throw_invalid("product batch pair has a null coefficient buffer");
      // runs read a coefficient (re, im) as one 16-byte load
      if ((reinterpret_cast<uintptr_t>(lhs_c[p]) | reinterpret_cast<uintptr_t>(rhs_c[p])) & 15u)
        wg::throw_invalid("product batch coefficient buffers must be 16-byte aligned (complex128 arrays)");
      if (W > 0 && (!lhs_x[p] || !lhs_z[p] || !rhs_x[p] || !rhs_z[p]))
        wg::throw_invalid("product batch pair has a null mask buffer");
    }
    masks[p] = PairMasks{lhs_x[p], lhs_z[p], rhs_x[p], rhs_z[p], n_rhs[p], item_base[p]};
    const uint64_t div_m = n_rhs[p] > 1 ? ~0ull / n_rhs[p] + 1 : 0ull;
    nums[p] = PairNum{lhs_c[p], rhs_c[p], n_rhs[p], div_m, 0, 0};
    item_base[p + 1] = item_base[p] + P;
    if (item_base[p + 1] > 0xffffffffull) wg::throw_invalid("a product batch takes fewer than 2^32 products in all");
  }
  const size_t N = item_base[np];
  b.N = N;
  b.seg_base.assign(np, 0);
  b.n_seg.assign(np, 0);
  if (N == 0) {
    b.S = 0;
  } else {
    const int K = 1 + 2 * W;
    wg::Scratch dmasks(sizeof(PairMasks) * np, s), dbase(sizeof(uint64_t) * (np + 1), s);
    wg::check_cuda(cudaMemcpyAsync(dmasks.get(), masks.data(), dmasks.size(), cudaMemcpyHostToDevice, s),
                   "upload batch masks");
    wg::check_cuda(cudaMemcpyAsync(dbase.get(), item_base.data(), dbase.size(), cudaMemcpyHostToDevice, s),
                   "upload batch bases");
    wg::Scratch keys(sizeof(uint64_t) * K * N, s), idx(sizeof(uint32_t) * N, s), raw(sizeof(uint32_t) * N, s);
    const unsigned g = wg::grid_for(N, kThreads, device, 8);
    WG_TIMED("pbatch_keys_kernel", s,
      pbatch_keys_kernel<<<g, kThreads, 0, s>>>(dmasks.as<PairMasks>(), dbase.as<uint64_t>(),
                                                static_cast<uint32_t>(np), N, W, keys.as<uint64_t>(),
                                                idx.as<uint32_t>(), raw.as<uint32_t>()));
    wg::check_launch("launch batch keys");
    wg::radix_sort_keys(device, N, K, keys, idx, s);  // stable: nested-loop order within equal keys
    b.code.reset(sizeof(uint32_t) * N, s);
    pbatch_gather_kernel<<<g, kThreads, 0, s>>>(idx.as<uint32_t>(), raw.as<uint32_t>(), N, b.code.as<uint32_t>());
    wg::check_launch("launch batch gather");
    raw.release();
    idx.release();
    wg::Scratch flags(sizeof(uint32_t) * N, s), segid(sizeof(uint32_t) * N, s), total(sizeof(uint32_t), s);
    pbatch_head_kernel<<<g, kThreads, 0, s>>>(keys.as<uint64_t>(), N, K, flags.as<uint32_t>());
    wg::check_launch("launch batch segment heads");
    wgs::exclusive_scan<uint32_t>(flags.as<uint32_t>(), segid.as<uint32_t>(), N, total.as<uint32_t>(), s);
    uint32_t S = 0;
    wg::check_cuda(cudaMemcpyAsync(&S, total.get(), sizeof(S), cudaMemcpyDeviceToHost, s), "read segment count");
    wg::check_cuda(cudaStreamSynchronize(s), "read segment count");
    b.S = S;
    b.seg_start.reset(sizeof(uint32_t) * (size_t(S) + 1), s);
    b.seg_pair.reset(sizeof(uint32_t) * S, s);
    b.seg_keys.reset(sizeof(uint64_t) * std::max<size_t>(1, size_t(S) * 2 * W), s);
    pbatch_segments_kernel<<<g, kThreads, 0, s>>>(flags.as<uint32_t>(), segid.as<uint32_t>(), keys.as<uint64_t>(), N,
                                                  W, b.seg_start.as<uint32_t>(), b.seg_pair.as<uint32_t>(),
                                                  b.seg_keys.as<uint64_t>());
    wg::check_launch("launch batch segments");
    const uint32_t n32 = static_cast<uint32_t>(N);
    wg::check_cuda(cudaMemcpyAsync(b.seg_start.as<uint32_t>() + S, &n32, sizeof(n32), cudaMemcpyHostToDevice, s),
                   "write segment end");
    wg::Scratch cnt(sizeof(unsigned) * np, s);
    wg::check_cuda(cudaMemsetAsync(cnt.get(), 0, cnt.size(), s), "clear segment counts");
    pbatch_count_kernel<<<wg::grid_for(S, kThreads, device, 8), kThreads, 0, s>>>(b.seg_pair.as<uint32_t>(), S,
                                                                                 cnt.as<unsigned>());
    wg::check_launch("launch batch segment counts");
    std::vector<unsigned> hcnt(np);
    wg::check_cuda(cudaMemcpyAsync(hcnt.data(), cnt.get(), cnt.size(), cudaMemcpyDeviceToHost, s),
                   "read segment counts");
    wg::check_cuda(cudaStreamSynchronize(s), "read segment counts");
    uint64_t run = 0;
    for (size_t p = 0; p < np; ++p) {
      b.seg_base[p] = run;
      b.n_seg[p] = hcnt[p];
      nums[p].seg_base = run;
      nums[p].n_seg = hcnt[p];
      run += hcnt[p];
    }
    if (run != S) wg::throw_invalid("product batch segment count mismatch");
  }
  const size_t S = b.S;
  b.pairs.reset(sizeof(PairNum) * std::max<size_t>(np, 1), s);
  wg::check_cuda(cudaMemcpyAsync(b.pairs.get(), nums.data(), sizeof(PairNum) * np, cudaMemcpyHostToDevice, s),
                 "upload batch pairs");
  b.segsum.reset(sizeof(double) * 2 * S, s);
  b.keep.reset(sizeof(uint32_t) * S, s);
  b.pos.reset(sizeof(uint32_t) * (S + 1), s);
  b.scan_ws.reset(sizeof(uint32_t) * wgs::scan_workspace(S), s);
  b.pair_max.reset(sizeof(unsigned long long) * std::max<size_t>(np, 1), s);
  b.out_x.reset(sizeof(uint64_t) * S * W, s);
  b.out_z.reset(sizeof(uint64_t) * S * W, s);
  b.out_c.reset(sizeof(double) * 2 * S, s);
  b.counts.reset(sizeof(uint64_t) * std::max<size_t>(np, 1), s);
  wg::check_cuda(cudaMemsetAsync(b.counts.get(), 0, b.counts.size(), s), "clear batch counts");
  b.sum_blocks = wg::grid_for(S, kThreads, device, 8);
  wg::check_cuda(cudaDeviceSynchronize(), "prepare product batch");
}

void run_batch(wg_products_batch_s& b, cudaStream_t s) {
  const int device = b.device;
  const size_t S = b.S;
  if (b.n_pairs == 0) return;
  if (S == 0) {
    wg::check_cuda(cudaMemsetAsync(b.counts.get(), 0, sizeof(uint64_t) * b.n_pairs, s), "clear batch counts");
    return;
  }
  const bool fused = b.mode == WG_PRODUCTS_FUSED;
  const int max_mode = fused ? kMaxNone : b.rtol > 0.0 ? kMaxFull : kMaxInf;
  if (!fused)
    wg::check_cuda(cudaMemsetAsync(b.pair_max.get(), 0, sizeof(unsigned long long) * b.n_pairs, s), "clear maxima");
  auto* sums = max_mode == kMaxNone ? pbatch_sums_kernel<kMaxNone>
               : max_mode == kMaxInf ? pbatch_sums_kernel<kMaxInf> : pbatch_sums_kernel<kMaxFull>;
  WG_TIMED("pbatch_sums_kernel", s,
    sums<<<b.sum_blocks, kThreads, 0, s>>>(b.pairs.as<PairNum>(), b.seg_start.as<uint32_t>(),
                                           b.seg_pair.as<uint32_t>(), b.code.as<uint32_t>(), S,
                                           b.segsum.as<double>(), b.pair_max.as<unsigned long long>()));
  wg::check_launch("launch batch sums");
  const unsigned g = wg::grid_for(S, kThreads, device, 8);
  WG_TIMED("pbatch_keep_kernel", s,
    pbatch_keep_kernel<<<g, kThreads, 0, s>>>(b.seg_pair.as<uint32_t>(), b.segsum.as<double>(), S, fused ? 1 : 0,
                                              b.atol, b.rtol, b.pair_max.as<unsigned long long>(),
                                              b.keep.as<uint32_t>()));
  wg::check_launch("launch batch cull");
  wgs::exclusive_scan_ws<uint32_t>(b.keep.as<uint32_t>(), b.pos.as<uint32_t>(), S, b.pos.as<uint32_t>() + S,
                                   b.scan_ws.as<uint32_t>(), s);
  auto* write = b.W == 1 ? pbatch_write_kernel<1> : b.W == 2 ? pbatch_write_kernel<2> : pbatch_write_kernel<0>;
  WG_TIMED("pbatch_write_kernel", s,
    write<<<g, kThreads, 0, s>>>(b.pairs.as<PairNum>(), b.seg_pair.as<uint32_t>(), b.seg_keys.as<uint64_t>(),
                                 b.segsum.as<double>(), b.keep.as<uint32_t>(), b.pos.as<uint32_t>(), S, b.W,
                                 b.out_x.as<uint64_t>(), b.out_z.as<uint64_t>(), b.out_c.as<double>()));
  wg::check_launch("launch batch write-out");
  pbatch_counts_kernel<<<wg::grid_for(b.n_pairs, kThreads, device, 1), kThreads, 0, s>>>(
      b.pairs.as<PairNum>(), b.pos.as<uint32_t>(), b.n_pairs, b.counts.as<uint64_t>());
  wg::check_launch("launch batch counts");
}

}  // namespace

extern "C" {

int wg_products_batch_create(int device, size_t words, size_t n_pairs, const uint64_t* const* lhs_x,
                             const uint64_t* const* lhs_z, const double* const* lhs_c, const size_t* n_lhs,
                             const uint64_t* const* rhs_x, const uint64_t* const* rhs_z,
                             const double* const* rhs_c, const size_t* n_rhs, int mode, double atol, double rtol,
                             wg_products_batch_t* batch, wg_stream_t stream) {
  return wg::guarded([&] {
    if (!batch) wg::throw_invalid("product batch output handle is null");
    *batch = nullptr;
    if (mode != WG_PRODUCTS_SIMPLIFY && mode != WG_PRODUCTS_FUSED)
      wg::throw_invalid("a product batch runs in simplify or fused mode");
    if (mode == WG_PRODUCTS_SIMPLIFY &&
        (atol < 0.0 || rtol < 0.0 || !std::isfinite(atol) || !std::isfinite(rtol)))
      wg::throw_invalid("simplify tolerances must be non-negative finite values");
    if (n_pairs > 0xfffffffeull) wg::throw_invalid("too many pairs in one product batch");
    if (n_pairs > 0 && (!n_lhs || !n_rhs || !lhs_c || !rhs_c || !lhs_x || !lhs_z || !rhs_x || !rhs_z))
      wg::throw_invalid("product batch pointer arrays must not be null");
    wg::DeviceGuard g(device);
    // the caller's operands may still be in flight on its stream
    wg::check_cuda(cudaStreamSynchronize(stream), "synchronize before a product batch");
    std::unique_ptr<wg_products_batch_s> b(new wg_products_batch_s());
    b->device = device;
    b->W = static_cast<int>(words);
    b->mode = mode;
    b->atol = atol;
    b->rtol = rtol;
    b->n_pairs = n_pairs;
    build_batch(*b, lhs_x, lhs_z, lhs_c, n_lhs, rhs_x, rhs_z, rhs_c, n_rhs);
    *batch = b.release();
  });
}

int wg_products_batch_run(wg_products_batch_t batch, wg_stream_t stream) {
  return wg::guarded([&] {
    if (!batch) wg::throw_invalid("product batch is null");
    wg::DeviceGuard g(batch->device);
    run_batch(*batch, stream);
  });
}

int wg_products_batch_result(wg_products_batch_t batch, size_t pair, uint64_t** x, uint64_t** z, double** coeffs,
                             size_t* capacity) {
  return wg::guarded([&] {
    if (!batch) wg::throw_invalid("product batch is null");
    if (pair >= batch->n_pairs) wg::throw_invalid("product batch pair index is out of range");
    const size_t base = batch->seg_base[pair];
    const size_t W = static_cast<size_t>(batch->W);
    if (x) *x = batch->n_seg[pair] && W ? batch->out_x.as<uint64_t>() + base * W : nullptr;
    if (z) *z = batch->n_seg[pair] && W ? batch->out_z.as<uint64_t>() + base * W : nullptr;
    if (coeffs) *coeffs = batch->n_seg[pair] ? batch->out_c.as<double>() + 2 * base : nullptr;
    if (capacity) *capacity = batch->n_seg[pair];
  });
}

int wg_products_batch_counts(wg_products_batch_t batch, uint64_t** counts) {
  return wg::guarded([&] {
    if (!batch) wg::throw_invalid("product batch is null");
    if (!counts) wg::throw_invalid("product batch counts output is null");
    *counts = batch->counts.as<uint64_t>();
  });
}

int wg_products_batch_info(wg_products_batch_t batch, size_t* n_products, size_t* n_keys) {
  return wg::guarded([&] {
    if (!batch) wg::throw_invalid("product batch is null");
    if (n_products) *n_products = batch->N;
    if (n_keys) *n_keys = batch->S;
  });
}

int wg_products_batch_destroy(wg_products_batch_t batch) {
  return wg::guarded([&] {
    if (!batch) return;
    wg::DeviceGuard g(batch->device);
    wg::check_cuda(cudaDeviceSynchronize(), "finish product batch runs");
    delete batch;
  });
}

}  // extern "C"
