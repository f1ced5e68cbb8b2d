// wg_scan.cuh -- device-wide exclusive prefix sums (reduce-then-scan).
//
// Used for radix-sort digit offsets, segment heads and survivor compaction.
// Chunks of 4096 items per 256-thread block are staged through shared memory
// so global loads and stores stay coalesced; block totals are scanned
// recursively.
#pragma once

#include <cuda_runtime.h>

#include "wg_common.cuh"

namespace wgs {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanChunk = kScanThreads * kScanItems;  // 4096

__device__ __forceinline__ int pad_idx(int i) { return i + (i >> 5); }

template <typename T>
__device__ T block_exclusive_scan(T v, T* warp_sums, T* block_total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += n;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T ws = lane < (kScanThreads / 32) ? warp_sums[lane] : T(0);
    T wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T n = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += n;
    }
    if (lane < (kScanThreads / 32)) warp_sums[lane] = wi - ws;
    if (lane == (kScanThreads / 32) - 1) *block_total = wi;
  }
  __syncthreads();
  return incl - v + warp_sums[warp];
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) chunk_sum_kernel(const T* __restrict__ in, size_t n,
                                                                 T* __restrict__ sums) {
  const size_t base = static_cast<size_t>(blockIdx.x) * kScanChunk;
  T acc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const size_t i = base + static_cast<size_t>(k) * kScanThreads + threadIdx.x;
    if (i < n) acc += in[i];
  }
  __shared__ T ws[kScanThreads / 32];
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) ws[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    T s = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) s += ws[w];
    sums[blockIdx.x] = s;
  }
}

// out[i] = offsets[block] + exclusive prefix of in within the chunk.  The
// last block also writes the grand total when `total` is non-null.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) chunk_scan_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                                  size_t n, const T* __restrict__ offsets,
                                                                  T* __restrict__ total) {
  __shared__ T s[kScanChunk + kScanChunk / 32];
  __shared__ T warp_sums[kScanThreads / 32];
  __shared__ T block_total;
  const size_t base = static_cast<size_t>(blockIdx.x) * kScanChunk;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int li = k * kScanThreads + threadIdx.x;
    const size_t i = base + li;
    s[pad_idx(li)] = i < n ? in[i] : T(0);
  }
  __syncthreads();
  T local[kScanItems];
  T sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    local[k] = s[pad_idx(threadIdx.x * kScanItems + k)];
    sum += local[k];
  }
  const T excl = block_exclusive_scan<T>(sum, warp_sums, &block_total);
  const T off = offsets ? offsets[blockIdx.x] : T(0);
  T run = excl + off;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s[pad_idx(threadIdx.x * kScanItems + k)] = run;
    run += local[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int li = k * kScanThreads + threadIdx.x;
    const size_t i = base + li;
    if (i < n) out[i] = s[pad_idx(li)];
  }
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = off + block_total;
}

// Exclusive scan of n items (in == out allowed).  Writes the grand total to
// the device scalar `total` when non-null.
template <typename T>
void exclusive_scan(const T* in, T* out, size_t n, T* total, cudaStream_t s) {
  if (n == 0) {
    if (total) wg::check_cuda(cudaMemsetAsync(total, 0, sizeof(T), s), "clear scan total");
    return;
  }
  const size_t blocks = (n + kScanChunk - 1) / kScanChunk;
  if (blocks > 0x7fffffffu) wg::throw_invalid("scan length exceeds the launch grid");
  if (blocks == 1) {
    chunk_scan_kernel<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total);
    wg::check_launch("launch scan");
    return;
  }
  wg::Scratch sums(blocks * sizeof(T), s);
  chunk_sum_kernel<T><<<static_cast<unsigned>(blocks), kScanThreads, 0, s>>>(in, n, sums.as<T>());
  wg::check_launch("launch scan reduce");
  exclusive_scan<T>(sums.as<T>(), sums.as<T>(), blocks, nullptr, s);
  chunk_scan_kernel<T><<<static_cast<unsigned>(blocks), kScanThreads, 0, s>>>(in, out, n, sums.as<T>(), total);
  wg::check_launch("launch scan");
}

// Elements of workspace that exclusive_scan_ws needs for n items: the block
// sums of every level of the recursion.
inline size_t scan_workspace(size_t n) {
  if (n <= static_cast<size_t>(kScanChunk)) return 0;
  const size_t blocks = (n + kScanChunk - 1) / kScanChunk;
  return blocks + scan_workspace(blocks);
}

// exclusive_scan with its block sums in a caller's workspace of
// scan_workspace(n) elements: no allocation, so a sequence of launches that
// uses it can be captured in a CUDA graph and replayed.
template <typename T>
void exclusive_scan_ws(const T* in, T* out, size_t n, T* total, T* ws, cudaStream_t s) {
  if (n == 0) {
    if (total) wg::check_cuda(cudaMemsetAsync(total, 0, sizeof(T), s), "clear scan total");
    return;
  }
  const size_t blocks = (n + kScanChunk - 1) / kScanChunk;
  if (blocks > 0x7fffffffu) wg::throw_invalid("scan length exceeds the launch grid");
  if (blocks == 1) {
    chunk_scan_kernel<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total);
    wg::check_launch("launch scan");
    return;
  }
  chunk_sum_kernel<T><<<static_cast<unsigned>(blocks), kScanThreads, 0, s>>>(in, n, ws);
  wg::check_launch("launch scan reduce");
  exclusive_scan_ws<T>(ws, ws, blocks, nullptr, ws + blocks, s);
  chunk_scan_kernel<T><<<static_cast<unsigned>(blocks), kScanThreads, 0, s>>>(in, out, n, ws, total);
  wg::check_launch("launch scan");
}

}  // namespace wgs
