// wg_group.cu -- greedy commuting groups and the Z-count expectation.
//
// group_commuting (reference src/grouping.cpp:197-290):
//   order = terms sorted by (weight desc, canonical key, index)   (:36-62)
//   qwc : a term joins the first group whose OR-basis has no conflict
//         ((tx & gz) ^ (tz & gx)) == 0 in every word               (:64-84)
//   full: a term joins the first group all of whose members commute with it
//                                                                  (:96-126)
//   otherwise it opens a new group.  Groups list members in placement order.
// The greedy is inherently sequential over terms; per term, one CTA of 1024
// threads examines all existing groups in parallel and takes the smallest
// accepting group index, so the result equals the sequential first-fit.

#include <cuda_runtime.h>

#include <climits>
#include <vector>

#include "wg_common.cuh"
#include "wg_scan.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kGreedyThreads = 1024;

// Sort keys for the deterministic order: word 0 = (maxw - weight) so that an
// ascending sort puts heavier terms first, then the canonical key words.
__global__ void order_keys_kernel(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z, size_t T, int W,
                                  uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < T;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint64_t wgt = 0;
    for (int w = 0; w < W; ++w) {
      const uint64_t a = x[i * W + w], b = z[i * W + w];
      wgt += __popcll(a | b);
      keys[static_cast<size_t>(1 + 2 * w) * T + i] = a;
      keys[static_cast<size_t>(2 + 2 * w) * T + i] = b;
    }
    keys[i] = ~wgt;  // larger weight -> smaller key
    idx[i] = static_cast<uint32_t>(i);
  }
}

__global__ void gather_terms_kernel(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z,
                                    const uint32_t* __restrict__ order, size_t T, int W, uint64_t* __restrict__ ox,
                                    uint64_t* __restrict__ oz) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < T;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t t = order[i];
    for (int w = 0; w < W; ++w) {
      ox[i * W + w] = x[t * W + w];
      oz[i * W + w] = z[t * W + w];
    }
  }
}

// Sequential first-fit over ordered terms (ox/oz in processing order).
// qwc state: bx/bz [G][W] group bases.  full state: first[g] / next[pos]
// singly linked member lists (positions in processing order).
template <int W, bool FULL>
__global__ void __launch_bounds__(kGreedyThreads) greedy_kernel(const uint64_t* __restrict__ ox,
                                                               const uint64_t* __restrict__ oz, uint32_t T,
                                                               uint64_t* __restrict__ bx, uint64_t* __restrict__ bz,
                                                               uint32_t* __restrict__ first, uint32_t* __restrict__ last,
                                                               uint32_t* __restrict__ next, uint32_t* __restrict__ group_of,
                                                               uint32_t* __restrict__ n_groups) {
  __shared__ unsigned s_best;
  uint32_t G = 0;
  for (uint32_t i = 0; i < T; ++i) {
    uint64_t tx[W], tz[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      tx[w] = ox[static_cast<size_t>(i) * W + w];
      tz[w] = oz[static_cast<size_t>(i) * W + w];
    }
    if (threadIdx.x == 0) s_best = UINT_MAX;
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += kGreedyThreads) {
      if (g >= *static_cast<volatile unsigned*>(&s_best)) break;
      bool accept = true;
      if (!FULL) {
#pragma unroll
        for (int w = 0; w < W; ++w)
          accept = accept && (((tx[w] & bz[static_cast<size_t>(g) * W + w]) ^ (tz[w] & bx[static_cast<size_t>(g) * W + w])) == 0);
      } else {
        for (uint32_t m = first[g]; m != UINT_MAX; m = next[m]) {
          uint64_t acc = 0;
#pragma unroll
          for (int w = 0; w < W; ++w)
            acc ^= (tx[w] & oz[static_cast<size_t>(m) * W + w]) ^ (tz[w] & ox[static_cast<size_t>(m) * W + w]);
          if (__popcll(acc) & 1u) {
            accept = false;
            break;
          }
        }
      }
      if (accept) {
        atomicMin(&s_best, g);
        break;
      }
    }
    __syncthreads();
    uint32_t best = s_best;
    const bool fresh = best == UINT_MAX;
    if (fresh) best = G;
    if (threadIdx.x == 0) {
      group_of[i] = best;
      if (!FULL) {
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const size_t o = static_cast<size_t>(best) * W + w;
          bx[o] = fresh ? tx[w] : (bx[o] | tx[w]);
          bz[o] = fresh ? tz[w] : (bz[o] | tz[w]);
        }
      } else {
        next[i] = UINT_MAX;
        if (fresh) first[best] = i;
        else next[last[best]] = i;
        last[best] = i;
      }
      __threadfence_block();
    }
    if (fresh) ++G;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_groups = G;
}

// 64-bit sort keys from group ids; carried index = processing position.
__global__ void widen_ids_kernel(const uint32_t* __restrict__ gid, size_t T, uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ pos) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < T;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    keys[i] = gid[i];
    pos[i] = static_cast<uint32_t>(i);
  }
}

__global__ void group_head_kernel(const uint64_t* __restrict__ sorted_gid, size_t T, uint32_t* __restrict__ flags) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < T;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    flags[i] = (i == 0 || sorted_gid[i] != sorted_gid[i - 1]) ? 1u : 0u;
}

__global__ void group_out_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ pos_sorted,
                                 const uint32_t* __restrict__ flags, const uint32_t* __restrict__ fpos, size_t T,
                                 uint64_t* __restrict__ order_out, uint64_t* __restrict__ starts) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < T;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    order_out[i] = order[pos_sorted[i]];
    if (flags[i]) starts[fpos[i]] = i;
  }
}

template <int W>
void launch_greedy(bool full, const uint64_t* ox, const uint64_t* oz, uint32_t T, uint64_t* bx, uint64_t* bz,
                   uint32_t* first, uint32_t* last, uint32_t* next, uint32_t* gid, uint32_t* ng, cudaStream_t s) {
  if (full)
    WG_TIMED("greedy_kernel", s,
      greedy_kernel<W, true><<<1, kGreedyThreads, 0, s>>>(ox, oz, T, bx, bz, first, last, next, gid, ng));
  else
    WG_TIMED("greedy_kernel", s,
      greedy_kernel<W, false><<<1, kGreedyThreads, 0, s>>>(ox, oz, T, bx, bz, first, last, next, gid, ng));
  wg::check_launch("launch group greedy");
}

// ---------------------------------------------------------------- Z counts

__global__ void or_reduce_kernel(const uint64_t* __restrict__ v, size_t n, unsigned long long* __restrict__ out) {
  uint64_t acc = 0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    acc |= v[i];
#pragma unroll
  for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicOr(out, static_cast<unsigned long long>(acc));
}

// Block per term: weighted parity sum over rows, then c_k * (sum / total).
__global__ void __launch_bounds__(kThreads) zcount_terms_kernel(const uint64_t* __restrict__ z, size_t T, int W,
                                                               const uint64_t* __restrict__ packed,
                                                               const double* __restrict__ counts, size_t rows,
                                                               double* __restrict__ weighted) {
  __shared__ double red[kThreads / 32];
  for (size_t t = blockIdx.x; t < T; t += gridDim.x) {
    double acc = 0.0;
    for (size_t r = threadIdx.x; r < rows; r += kThreads) {
      unsigned odd = 0;
      for (int w = 0; w < W; ++w) odd ^= __popcll(z[t * W + w] & packed[r * W + w]) & 1u;
      acc += odd ? -counts[r] : counts[r];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) s += red[w];
      weighted[t] = s;
    }
    __syncthreads();
  }
}

__global__ void zcount_total_kernel(const double* __restrict__ c, const double* __restrict__ weighted, size_t T,
                                    const double* __restrict__ counts, size_t rows, double* __restrict__ out) {
  // single thread: sums in the reference's order (total over rows, then terms)
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double total = 0.0;
  for (size_t r = 0; r < rows; ++r) total += counts[r];
  double re = 0.0, im = 0.0;
  for (size_t t = 0; t < T; ++t) {
    const double f = weighted[t] / total;
    re += c[2 * t] * f;
    im += c[2 * t + 1] * f;
  }
  out[0] = re;
  out[1] = im;
}

}  // namespace

extern "C" {

int wg_group_commuting(int device, size_t words, size_t n_terms, const uint64_t* x, const uint64_t* z, int mode_full,
                       size_t* order_out, size_t* sizes_out, size_t* n_groups, wg_stream_t stream) {
  return wg::guarded([&] {
    *n_groups = 0;
    if (n_terms == 0) return;
    if (n_terms >= 0xffffffffull) wg::throw_invalid("group_commuting supports fewer than 2^32-1 terms");
    if (words > 4) wg::throw_invalid("group_commuting on the device supports at most 256 qubits");
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    const size_t T = n_terms;
    const int W = static_cast<int>(words);
    const int K = 1 + 2 * W;
    wg::Scratch keys(8 * K * T, s), idx(4 * T, s);
    order_keys_kernel<<<wg::grid_for(T, kThreads, device, 4), kThreads, 0, s>>>(x, z, T, W, keys.as<uint64_t>(),
                                                                                idx.as<uint32_t>());
    wg::check_launch("launch order keys");
    wg::radix_sort_keys(device, T, K, keys, idx, s);
    keys.release();
    const uint32_t* order = idx.as<uint32_t>();
    const size_t Wa = W > 0 ? W : 1;
    wg::Scratch ox(8 * Wa * T, s), oz(8 * Wa * T, s);
    if (W > 0) {
      gather_terms_kernel<<<wg::grid_for(T, kThreads, device, 4), kThreads, 0, s>>>(x, z, order, T, W,
                                                                                   ox.as<uint64_t>(), oz.as<uint64_t>());
      wg::check_launch("launch gather terms");
    } else {
      wg::check_cuda(cudaMemsetAsync(ox.get(), 0, 8 * T, s), "clear masks");
      wg::check_cuda(cudaMemsetAsync(oz.get(), 0, 8 * T, s), "clear masks");
    }
    wg::Scratch bx(8 * Wa * T, s), bz(8 * Wa * T, s), first(4 * T, s), last(4 * T, s), next(4 * T, s),
        gid(4 * T, s), ng(4, s);
    const bool full = mode_full != 0;
    const uint32_t T32 = static_cast<uint32_t>(T);
    switch (W) {
      case 0:
      case 1: launch_greedy<1>(full, ox.as<uint64_t>(), oz.as<uint64_t>(), T32, bx.as<uint64_t>(), bz.as<uint64_t>(),
                               first.as<uint32_t>(), last.as<uint32_t>(), next.as<uint32_t>(), gid.as<uint32_t>(),
                               ng.as<uint32_t>(), s); break;
      case 2: launch_greedy<2>(full, ox.as<uint64_t>(), oz.as<uint64_t>(), T32, bx.as<uint64_t>(), bz.as<uint64_t>(),
                               first.as<uint32_t>(), last.as<uint32_t>(), next.as<uint32_t>(), gid.as<uint32_t>(),
                               ng.as<uint32_t>(), s); break;
      case 3: launch_greedy<3>(full, ox.as<uint64_t>(), oz.as<uint64_t>(), T32, bx.as<uint64_t>(), bz.as<uint64_t>(),
                               first.as<uint32_t>(), last.as<uint32_t>(), next.as<uint32_t>(), gid.as<uint32_t>(),
                               ng.as<uint32_t>(), s); break;
      default: launch_greedy<4>(full, ox.as<uint64_t>(), oz.as<uint64_t>(), T32, bx.as<uint64_t>(), bz.as<uint64_t>(),
                                first.as<uint32_t>(), last.as<uint32_t>(), next.as<uint32_t>(), gid.as<uint32_t>(),
                                ng.as<uint32_t>(), s); break;
    }
    uint32_t G = 0;
    wg::check_cuda(cudaMemcpyAsync(&G, ng.get(), 4, cudaMemcpyDeviceToHost, s), "read group count");
    wg::check_cuda(cudaStreamSynchronize(s), "group greedy");
    // Stable partition of processing positions by group id.
    wg::Scratch gkeys(8 * T, s), pos(4 * T, s);
    widen_ids_kernel<<<wg::grid_for(T, kThreads, device, 4), kThreads, 0, s>>>(gid.as<uint32_t>(), T,
                                                                             gkeys.as<uint64_t>(), pos.as<uint32_t>());
    wg::check_launch("launch group id widen");
    wg::radix_sort_keys(device, T, 1, gkeys, pos, s);
    wg::Scratch flags(4 * T, s), fpos(4 * T, s), out_order(8 * T, s), starts(8 * (size_t(G) + 1), s);
    const unsigned gr = wg::grid_for(T, kThreads, device, 4);
    group_head_kernel<<<gr, kThreads, 0, s>>>(gkeys.as<uint64_t>(), T, flags.as<uint32_t>());
    wg::check_launch("launch group heads");
    wgs::exclusive_scan<uint32_t>(flags.as<uint32_t>(), fpos.as<uint32_t>(), T, nullptr, s);
    group_out_kernel<<<gr, kThreads, 0, s>>>(order, pos.as<uint32_t>(), flags.as<uint32_t>(), fpos.as<uint32_t>(), T,
                                             out_order.as<uint64_t>(), starts.as<uint64_t>());
    wg::check_launch("launch group output");
    std::vector<uint64_t> hs(static_cast<size_t>(G) + 1);
    static_assert(sizeof(size_t) == sizeof(uint64_t), "size_t must be 64-bit");
    wg::check_cuda(cudaMemcpyAsync(order_out, out_order.get(), 8 * T, cudaMemcpyDeviceToHost, s), "read groups");
    wg::check_cuda(cudaMemcpyAsync(hs.data(), starts.get(), 8 * G, cudaMemcpyDeviceToHost, s), "read groups");
    wg::check_cuda(cudaStreamSynchronize(s), "read groups");
    hs[G] = T;
    for (uint32_t k = 0; k < G; ++k) sizes_out[k] = hs[k + 1] - hs[k];
    *n_groups = G;
  });
}

int wg_expectation_z_counts(int device, size_t words, size_t n_terms, const uint64_t* x, const uint64_t* z,
                            const double* coeffs, size_t rows, const uint64_t* packed, const double* counts,
                            double* result_host, wg_stream_t stream) {
  return wg::guarded([&] {
    result_host[0] = result_host[1] = 0.0;
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    if (n_terms > 0 && words > 0) {
      wg::Scratch o(8, s);
      wg::check_cuda(cudaMemsetAsync(o.get(), 0, 8, s), "clear");
      or_reduce_kernel<<<wg::grid_for(n_terms * words, kThreads, device, 4), kThreads, 0, s>>>(
          x, n_terms * words, o.as<unsigned long long>());
      wg::check_launch("launch diagonal check");
      unsigned long long h = 0;
      wg::check_cuda(cudaMemcpyAsync(&h, o.get(), 8, cudaMemcpyDeviceToHost, s), "read diagonal check");
      wg::check_cuda(cudaStreamSynchronize(s), "read diagonal check");
      if (h != 0) wg::throw_invalid("expectation_z_counts requires diagonal Pauli terms");
    }
    if (n_terms == 0) return;
    wg::Scratch weighted(8 * n_terms, s), res(16, s);
    const unsigned grid = static_cast<unsigned>(std::min<size_t>(n_terms, 65535));
    WG_TIMED("zcount_terms_kernel", s,
      zcount_terms_kernel<<<grid, kThreads, 0, s>>>(z, n_terms, static_cast<int>(words), packed, counts, rows,
                                                    weighted.as<double>()));
    wg::check_launch("launch z-count terms");
    zcount_total_kernel<<<1, 32, 0, s>>>(coeffs, weighted.as<double>(), n_terms, counts, rows, res.as<double>());
    wg::check_launch("launch z-count total");
    wg::check_cuda(cudaMemcpyAsync(result_host, res.get(), 16, cudaMemcpyDeviceToHost, s), "read z-count result");
    wg::check_cuda(cudaStreamSynchronize(s), "read z-count result");
  });
}

}  // extern "C"
