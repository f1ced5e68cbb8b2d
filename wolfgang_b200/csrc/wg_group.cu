// wg_group.cu -- greedy commuting groups and the Z-count expectation.
//
// group_commuting (reference src/grouping.cpp:197-290):
//   order = terms sorted by (weight desc, canonical key, index)   (:36-62)
//   qwc : a term joins the first group whose OR-basis has no conflict
//         ((tx & gz) ^ (tz & gx)) == 0 in every word               (:64-84)
//   full: a term joins the first group all of whose members commute with it
//                                                                  (:96-126)
//   otherwise it opens a new group.  Groups list members in placement order.
// The first-fit is sequential over terms; here it runs in chunks: a bound pass
// over the whole GPU finds, for every term of a chunk, the first group that
// accepts it at the chunk's start, and one warp then places the chunk's terms
// in order starting from those bounds (see group_bound_kernel), so the result
// equals the sequential first-fit.

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "wg_common.cuh"
#include "wg_scan.cuh"

namespace {

constexpr int kThreads = 256;

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

// First-fit over ordered terms (ox/oz in processing order), in chunks of
// kChunk terms.  Group state only grows (a qwc basis gains bits, a full-mode
// group gains members), so a term's set of accepting groups only shrinks as
// terms are placed: the first group that accepts a term at the start of its
// chunk is a lower bound on the group it joins.  group_bound_kernel finds
// that bound for every term of a chunk at once (a warp per term, 32 groups per
// ballot); group_resolve_kernel then places the chunk's terms one by one from
// their bounds, checking groups from the bound upward against the current
// state, which is the sequential first-fit's answer.  In full mode the bound
// group itself was checked against every member present at the chunk's start,
// so only the members it gained during the chunk are checked again.
// qwc state: one basis row per group, rows[g] = [x words | z words] (2W
// words, moved as 16-byte pieces).  full state: first[g] / last[g] /
// next[pos] member lists in processing order; the bound pass also records
// which of the 32 groups from the bound accepted the term at the chunk's start
// (lbm), so that those need checking only against the chunk's own members.
// Chunk lengths, measured on random 128-qubit terms (each qubit non-identity
// with probability 0.05): qwc 1,024 (512: 88 ms, 1,024: 81 ms, 2,048: 122 ms
// for 262,144 terms); full mode 96 (64: 88 ms, 96: 79 ms, 128: 81 ms, 256:
// 114 ms, 512: 213 ms for 32,768 terms), where every failed bound costs
// member-list walks and shorter chunks keep the bounds closer.
constexpr int kChunk = 1024;     // terms per chunk (qwc); also the staging capacity
constexpr int kChunkFull = 96;   // terms per chunk in full mode
constexpr int kBoundThreads = 256;
constexpr int kResolveThreads = 256;

template <int W>
__device__ __forceinline__ void load_row(const uint64_t* p, uint64_t (&r)[2 * W]) {
  const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const ulonglong2 v = q[j];
    r[2 * j] = v.x;
    r[2 * j + 1] = v.y;
  }
}

template <int W>
__device__ __forceinline__ void store_row(uint64_t* p, const uint64_t (&r)[2 * W]) {
  ulonglong2* q = reinterpret_cast<ulonglong2*>(p);
#pragma unroll
  for (int j = 0; j < W; ++j) q[j] = make_ulonglong2(r[2 * j], r[2 * j + 1]);
}

// qwc: no qubit on which the term and the basis hold different non-identity
// Paulis.  Rows are [x words | z words].
template <int W>
__device__ __forceinline__ bool row_accepts(const uint64_t (&t)[2 * W], const uint64_t (&b)[2 * W]) {
  uint64_t d = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) d |= (t[w] & b[W + w]) ^ (t[W + w] & b[w]);
  return d == 0;
}

// Every member from position m on (following next) commutes with the term.
template <int W>
__device__ __forceinline__ bool members_commute(const uint64_t (&t)[2 * W], const uint64_t* __restrict__ ox,
                                                const uint64_t* __restrict__ oz, const uint32_t* next, uint32_t m) {
  for (; m != UINT_MAX; m = next[m]) {
    uint64_t acc = 0;
#pragma unroll
    for (int w = 0; w < W; ++w)
      acc ^= (t[w] & oz[static_cast<size_t>(m) * W + w]) ^ (t[W + w] & ox[static_cast<size_t>(m) * W + w]);
    if (__popcll(acc) & 1u) return false;
  }
  return true;
}

// The term anticommutes with the staged row (2W words in shared memory).
template <int W>
__device__ __forceinline__ bool anticommutes(const uint64_t (&t)[2 * W], const uint64_t* row) {
  uint64_t r[2 * W];
  load_row<W>(row, r);
  uint64_t acc = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) acc ^= (t[w] & r[W + w]) ^ (t[W + w] & r[w]);
  return (__popcll(acc) & 1u) != 0;
}

// Full mode: the bound of each term of a chunk is searched by kBoundSplit
// warps, warp s taking every kBoundSplit-th round of 32 groups from round s.
// A warp records the first accepting group of its rounds with atomicMin on
// lb[i] (set to UINT_MAX beforehand) and stops once its next round starts at
// or above the smallest group recorded so far, so lb[i] ends as the first
// accepting group overall.  Member lists make a round of checks long; the
// split keeps a chunk of few terms from leaving most of the GPU idle.
constexpr int kBoundSplit = 8;

template <int W>
__global__ void __launch_bounds__(kBoundThreads) group_search_full_kernel(
    const uint64_t* __restrict__ ox, const uint64_t* __restrict__ oz, uint32_t c0, uint32_t c1,
    const uint32_t* __restrict__ first, const uint32_t* __restrict__ next, const uint32_t* __restrict__ n_groups,
    uint32_t* lb) {
  const uint32_t G0 = *n_groups;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t units = (c1 - c0) * kBoundSplit;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units; u += nw) {
    const uint32_t i = c0 + u / kBoundSplit, sub = u % kBoundSplit;
    uint64_t t[2 * W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      t[w] = ox[static_cast<size_t>(i) * W + w];
      t[W + w] = oz[static_cast<size_t>(i) * W + w];
    }
    for (uint32_t g0 = sub * 32; g0 < G0; g0 += 32 * kBoundSplit) {
      // the smallest accepting group any warp has recorded, read once per warp
      uint32_t best = 0;
      if (lane == 0) best = *static_cast<volatile uint32_t*>(&lb[i]);
      best = __shfl_sync(0xffffffffu, best, 0);
      if (g0 >= best) break;
      const uint32_t g = g0 + lane;
      const bool ok = g < G0 && members_commute<W>(t, ox, oz, next, first[g]);
      const unsigned b = __ballot_sync(0xffffffffu, ok);
      if (b) {
        if (lane == 0) atomicMin(&lb[i], g0 + __ffs(b) - 1);
        break;
      }
    }
  }
}

template <int W, bool FULL>
__global__ void __launch_bounds__(kBoundThreads) group_bound_kernel(const uint64_t* __restrict__ ox,
                                                                   const uint64_t* __restrict__ oz, uint32_t c0,
                                                                   uint32_t c1, const uint64_t* __restrict__ rows,
                                                                   const uint32_t* __restrict__ first,
                                                                   const uint32_t* __restrict__ next,
                                                                   const uint32_t* __restrict__ n_groups,
                                                                   uint32_t* __restrict__ lb,
                                                                   uint32_t* __restrict__ lbm) {
  const uint32_t G0 = *n_groups;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = c0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < c1; i += nw) {
    uint64_t t[2 * W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      t[w] = ox[static_cast<size_t>(i) * W + w];
      t[W + w] = oz[static_cast<size_t>(i) * W + w];
    }
    uint32_t found = G0;
    if (FULL) {
      // found by group_search_full_kernel (UINT_MAX: no group accepts)
      found = min(lb[i], G0);
    } else {
      for (uint32_t g0 = 0; g0 < G0; g0 += 32) {
        const uint32_t g = g0 + lane;
        bool ok = false;
        if (g < G0) {
          uint64_t r[2 * W];
          load_row<W>(rows + static_cast<size_t>(g) * (2 * W), r);
          ok = row_accepts<W>(t, r);
        }
        const unsigned b = __ballot_sync(0xffffffffu, ok);
        if (b) {
          found = g0 + __ffs(b) - 1;
          break;
        }
      }
    }
    __syncwarp();
    if (lane == 0) lb[i] = found;
    if (FULL) {
      // which of the 32 groups from the bound accept the term now
      const uint32_t g = found + lane;
      const bool ok = g < G0 && members_commute<W>(t, ox, oz, next, first[g]);
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (lane == 0) lbm[i] = m;
    }
  }
}

// qwc placement of a chunk's staged term rows by one warp.  Lane j owns the
// groups g with g % 32 == j: any 32 consecutive groups hold one group of each
// lane, so a round over [g0, g0 + 32) has lane j check g0 + ((j - g0) & 31),
// and a basis row is only ever read and written by its owner (no cross-lane
// ordering is needed).  One warp reduction per round gives the smallest
// accepting group; its owner ORs the term into the row.  The fast loop runs
// the first round of each term (most terms end there) and leaves at the first
// term it cannot place; that term's later rounds (or its new group) are
// handled outside it, and the fast loop resumes.  Keeping the rare path out of
// the per-term loop keeps the loop free of nested warp-synchronous control
// flow.  B holds the basis rows: shared memory (SMEM) or global memory.
template <int W, bool SMEM>
__device__ __forceinline__ uint32_t place_qwc(const uint64_t* st, const uint32_t* slb, uint32_t* sgid, uint32_t n,
                                              uint32_t G, uint64_t* B) {
  const uint32_t lane = threadIdx.x & 31;
  auto row_at = [&](uint32_t g) { return SMEM ? B + g * (2 * W) : B + static_cast<size_t>(g) * (2 * W); };
  uint32_t k = 0;
  while (k < n) {
    uint64_t t[2 * W], r[2 * W];
    uint32_t l = 0;
    for (; k < n; ++k) {
      load_row<W>(st + k * (2 * W), t);
      l = slb[k];
      const uint32_t g = l + ((lane - l) & 31u);
      bool ok = false;
      if (g < G) {
        load_row<W>(row_at(g), r);
        ok = row_accepts<W>(t, r);
      }
      const uint32_t best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
      if (best == UINT_MAX) break;
      if (best % 32 == lane) {
#pragma unroll
        for (int e = 0; e < 2 * W; ++e) r[e] |= t[e];
        store_row<W>(row_at(best), r);
      }
      if (lane == 0) sgid[k] = best;
    }
    if (k >= n) break;
    // term k: the rounds after the first, then a new group if none accepts
    uint32_t best = UINT_MAX;
    for (uint32_t g0 = l + 32; best == UINT_MAX && g0 < G; g0 += 32) {
      const uint32_t g = g0 + ((lane - g0) & 31u);
      bool ok = false;
      if (g < G) {
        load_row<W>(row_at(g), r);
        ok = row_accepts<W>(t, r);
      }
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    const bool fresh = best == UINT_MAX;
    if (fresh) best = G;
    if (best % 32 == lane) {
#pragma unroll
      for (int e = 0; e < 2 * W; ++e) r[e] = fresh ? t[e] : (r[e] | t[e]);
      store_row<W>(row_at(best), r);
    }
    if (fresh) ++G;
    if (lane == 0) sgid[k] = best;
    ++k;
  }
  return G;
}

// Full-mode placement of a chunk's staged term rows by one warp.  A term's
// bound group l accepted it at the chunk's start, so the fast loop checks it
// only against the chunk's members placed in l so far (lane-parallel over the
// chunk's earlier terms, one vote).  A term that fails, or had no bound, goes
// through the groups in first-fit order outside the fast loop: the window
// groups that accepted it at the chunk's start (lbm), again against the
// chunk's members only; the older groups beyond the window, by a walk of their
// whole member list; the groups opened during the chunk, whose members are all
// chunk members.  sgid[k] is written by lane k % 32, the lane that reads it in
// the fast loop; the slow path starts with a warp barrier so that every lane
// sees all group ids and list links written so far.
template <int W>
__device__ __forceinline__ uint32_t place_full(const uint64_t* __restrict__ ox, const uint64_t* __restrict__ oz,
                                               const uint64_t* st, const uint32_t* slb, const uint32_t* smask,
                                               uint32_t* sgid, uint32_t n, uint32_t c0, uint32_t G0, uint32_t* first,
                                               uint32_t* last, uint32_t* next) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t G = G0;
  // no member placed in group g among the chunk's first k terms anticommutes with t
  auto chunk_members_commute = [&](const uint64_t (&t)[2 * W], uint32_t g, uint32_t k) {
    for (uint32_t q = 0; q < k; ++q)
      if (sgid[q] == g && anticommutes<W>(t, st + q * (2 * W))) return false;
    return true;
  };
  auto place = [&](uint32_t k, uint32_t best, bool fresh) {
    if ((k & 31u) == lane) sgid[k] = best;
    if (lane == 0) {
      const uint32_t i = c0 + k;
      next[i] = UINT_MAX;
      if (fresh) first[best] = i;
      else next[last[best]] = i;
      last[best] = i;
    }
  };
  uint32_t k = 0;
  while (k < n) {
    uint64_t t[2 * W];
    uint32_t l = 0;
    for (; k < n; ++k) {
      load_row<W>(st + k * (2 * W), t);
      l = slb[k];
      if (l >= G0) break;
      bool bad = false;
      for (uint32_t q = lane; q < k; q += 32)
        if (sgid[q] == l && anticommutes<W>(t, st + q * (2 * W))) bad = true;
      if (__any_sync(0xffffffffu, bad)) break;
      place(k, l, false);
    }
    if (k >= n) break;
    __syncwarp();
    const uint32_t m = smask[k];
    uint32_t best = UINT_MAX;
    {
      const uint32_t g = l + lane;
      const bool ok = l < G0 && lane > 0 && g < G0 && ((m >> lane) & 1u) && chunk_members_commute(t, g, k);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    for (uint32_t g0 = l + 32; best == UINT_MAX && g0 < G0; g0 += 32) {
      const uint32_t g = g0 + lane;
      const bool ok = g < G0 && members_commute<W>(t, ox, oz, next, first[g]);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    for (uint32_t g0 = G0; best == UINT_MAX && g0 < G; g0 += 32) {
      const uint32_t g = g0 + lane;
      const bool ok = g < G && chunk_members_commute(t, g, k);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    const bool fresh = best == UINT_MAX;
    if (fresh) best = G;
    place(k, best, fresh);
    if (fresh) ++G;
    __syncwarp();
    ++k;
  }
  return G;
}

// One CTA: its threads stage the chunk's term rows and bounds (and, in qwc
// mode, the basis rows when every group of the chunk fits) in shared memory;
// warp 0 places the terms in order; the threads then write the basis rows
// back and the chunk's group ids out.
template <int W, bool FULL>
__global__ void __launch_bounds__(kResolveThreads) group_resolve_kernel(
    const uint64_t* __restrict__ ox, const uint64_t* __restrict__ oz, uint32_t c0, uint32_t c1, uint32_t cap, uint64_t* __restrict__ rows, uint32_t* __restrict__ first, uint32_t* __restrict__ last,
    uint32_t* __restrict__ next, const uint32_t* __restrict__ lb, const uint32_t* __restrict__ lbm,
    uint32_t* __restrict__ group_of, uint32_t* __restrict__ n_groups) {
  extern __shared__ __align__(16) unsigned char rraw[];
  __shared__ uint32_t s_G;
  const uint32_t n = c1 - c0;
  uint64_t* st = reinterpret_cast<uint64_t*>(rraw);         // [kChunk][2W] term rows
  uint64_t* sb = st + kChunk * (2 * W);                       // [cap][2W] basis rows
  uint32_t* slb = reinterpret_cast<uint32_t*>(sb + static_cast<size_t>(cap) * (2 * W));
  uint32_t* sgid = slb + kChunk;
  uint32_t* smask = sgid + kChunk;
  const uint32_t G0 = *n_groups;
  const bool in_smem = !FULL && static_cast<uint64_t>(G0) + n <= cap;
  for (uint32_t k = threadIdx.x; k < n * W; k += blockDim.x) {
    const uint32_t kk = k / W, w = k - kk * W;
    st[kk * (2 * W) + w] = ox[static_cast<size_t>(c0) * W + k];
    st[kk * (2 * W) + W + w] = oz[static_cast<size_t>(c0) * W + k];
  }
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    slb[k] = lb[c0 + k];
    if (FULL) smask[k] = lbm[c0 + k];
  }
  if (in_smem) {
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(rows);
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(sb);
    for (uint32_t k = threadIdx.x; k < G0 * W; k += blockDim.x) dst[k] = src[k];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t G = G0;
    if (!FULL) {
      G = in_smem ? place_qwc<W, true>(st, slb, sgid, n, G0, sb) : place_qwc<W, false>(st, slb, sgid, n, G0, rows);
    } else {
      G = place_full<W>(ox, oz, st, slb, smask, sgid, n, c0, G0, first, last, next);
    }
    if (threadIdx.x == 0) {
      *n_groups = G;
      s_G = G;
    }
  }
  __syncthreads();
  if (in_smem) {
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(sb);
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(rows);
    for (uint32_t k = threadIdx.x; k < s_G * W; k += blockDim.x) dst[k] = src[k];
  }
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) group_of[c0 + k] = sgid[k];
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

// Chunk lengths the autotuner chooses among (the measured defaults above are
// candidates 2 and 1); every chunk length gives the same groups.
constexpr uint32_t kQwcChunks[] = {256, 512, 1024};
constexpr uint32_t kFullChunks[] = {64, 96, 128, 192};
static_assert(kQwcChunks[2] == kChunk && kFullChunks[1] == kChunkFull, "defaults are candidates");

template <int W>
void run_greedy(int device, bool full, const uint64_t* ox, const uint64_t* oz, uint32_t T, uint64_t* rows,
                uint32_t* first, uint32_t* last, uint32_t* next, uint32_t* lb, uint32_t* lbm, uint32_t* gid,
                uint32_t* ng, cudaStream_t s, uint32_t chunk) {
  const auto& props = wg::device_props(device);
  auto* kb = full ? group_bound_kernel<W, true> : group_bound_kernel<W, false>;
  auto* kr = full ? group_resolve_kernel<W, true> : group_resolve_kernel<W, false>;
  // term rows, bounds, bound masks and group ids of a chunk, then as many basis rows as fit
  // beside the kernel's static shared memory
  cudaFuncAttributes fa{};
  wg::check_cuda(cudaFuncGetAttributes(&fa, kr), "query group resolve attributes");
  const size_t stage = static_cast<size_t>(kChunk) * (16 * W + 12);
  const size_t smem_max = static_cast<size_t>(props.max_smem_optin) - fa.sharedSizeBytes;
  const uint32_t cap = full || smem_max <= stage ? 0u : static_cast<uint32_t>((smem_max - stage) / (16 * W));
  const size_t smem = stage + static_cast<size_t>(cap) * 16 * W;
  wg::check_cuda(cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                 "set group resolve shared memory");
  wg::check_cuda(cudaMemsetAsync(ng, 0, 4, s), "clear group count");
  const unsigned max_blocks = static_cast<unsigned>(props.sm_count) * 8;
  if (chunk == 0 || chunk > static_cast<uint32_t>(kChunk)) chunk = full ? kChunkFull : kChunk;  // staging holds kChunk
  for (uint32_t c0 = 0; c0 < T; c0 += chunk) {
    const uint32_t c1 = T - c0 > chunk ? c0 + chunk : T;
    const unsigned blocks = std::min<unsigned>(max_blocks, (c1 - c0 + kBoundThreads / 32 - 1) / (kBoundThreads / 32));
    if (full) {
      wg::check_cuda(cudaMemsetAsync(lb + c0, 0xff, 4 * static_cast<size_t>(c1 - c0), s), "clear bounds");
      const unsigned sblocks = std::min<unsigned>(
          max_blocks, ((c1 - c0) * kBoundSplit + kBoundThreads / 32 - 1) / (kBoundThreads / 32));
      WG_TIMED("group_search_full_kernel", s,
        group_search_full_kernel<W><<<sblocks, kBoundThreads, 0, s>>>(ox, oz, c0, c1, first, next, ng, lb));
      wg::check_launch("launch group bound search");
    }
    WG_TIMED("group_bound_kernel", s,
      kb<<<blocks, kBoundThreads, 0, s>>>(ox, oz, c0, c1, rows, first, next, ng, lb, lbm));
    wg::check_launch("launch group bounds");
    WG_TIMED("group_resolve_kernel", s,
      kr<<<1, kResolveThreads, smem, s>>>(ox, oz, c0, c1, cap, rows, first, last, next, lb, lbm, gid, ng));
    wg::check_launch("launch group resolve");
  }
}

// ------------------------------------------------ any number of mask words
// More than 4 mask words (over 256 qubits): the same chunked first-fit as
// above, with each row read word by word from memory instead of held in
// registers.  Term rows are interleaved once as trows[i] = [x words | z words]
// (processing order); a chunk's term rows are staged in shared memory, the
// qwc basis rows and the full-mode member lists stay in global memory.  The
// chunk is shortened when its staged rows would not fit in shared memory.

__device__ __forceinline__ bool row_accepts_n(const uint64_t* t, const uint64_t* b, int W) {
  uint64_t d = 0;
  for (int w = 0; w < W; ++w) d |= (t[w] & b[W + w]) ^ (t[W + w] & b[w]);
  return d == 0;
}

// parity of the symplectic product of two [x | z] rows
__device__ __forceinline__ bool anticommutes_n(const uint64_t* t, const uint64_t* row, int W) {
  uint64_t acc = 0;
  for (int w = 0; w < W; ++w) acc ^= (t[w] & row[W + w]) ^ (t[W + w] & row[w]);
  return (__popcll(acc) & 1u) != 0;
}

__device__ __forceinline__ bool members_commute_n(const uint64_t* t, const uint64_t* __restrict__ trows,
                                                  const uint32_t* next, uint32_t m, int W) {
  for (; m != UINT_MAX; m = next[m])
    if (anticommutes_n(t, trows + static_cast<size_t>(m) * (2 * W), W)) return false;
  return true;
}

__global__ void interleave_rows_kernel(const uint64_t* __restrict__ ox, const uint64_t* __restrict__ oz, size_t T,
                                       int W, uint64_t* __restrict__ trows) {
  const size_t n = T * static_cast<size_t>(W);
  for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < n;
       k += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t i = k / W, w = k - i * W;
    trows[i * (2 * W) + w] = ox[k];
    trows[i * (2 * W) + W + w] = oz[k];
  }
}

// group_search_full_kernel for any width
__global__ void __launch_bounds__(kBoundThreads) group_search_full_n_kernel(
    const uint64_t* __restrict__ trows, int W, uint32_t c0, uint32_t c1, const uint32_t* __restrict__ first,
    const uint32_t* __restrict__ next, const uint32_t* __restrict__ n_groups, uint32_t* lb) {
  const uint32_t G0 = *n_groups;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t units = (c1 - c0) * kBoundSplit;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units; u += nw) {
    const uint32_t i = c0 + u / kBoundSplit, sub = u % kBoundSplit;
    const uint64_t* t = trows + static_cast<size_t>(i) * (2 * W);
    for (uint32_t g0 = sub * 32; g0 < G0; g0 += 32 * kBoundSplit) {
      uint32_t best = 0;
      if (lane == 0) best = *static_cast<volatile uint32_t*>(&lb[i]);
      best = __shfl_sync(0xffffffffu, best, 0);
      if (g0 >= best) break;
      const uint32_t g = g0 + lane;
      const bool ok = g < G0 && members_commute_n(t, trows, next, first[g], W);
      const unsigned b = __ballot_sync(0xffffffffu, ok);
      if (b) {
        if (lane == 0) atomicMin(&lb[i], g0 + __ffs(b) - 1);
        break;
      }
    }
  }
}

// group_bound_kernel for any width
__global__ void __launch_bounds__(kBoundThreads) group_bound_n_kernel(
    const uint64_t* __restrict__ trows, int W, uint32_t c0, uint32_t c1, const uint64_t* __restrict__ rows,
    const uint32_t* __restrict__ first, const uint32_t* __restrict__ next, const uint32_t* __restrict__ n_groups,
    uint32_t* __restrict__ lb, uint32_t* __restrict__ lbm, int full) {
  const uint32_t G0 = *n_groups;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = c0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < c1; i += nw) {
    const uint64_t* t = trows + static_cast<size_t>(i) * (2 * W);
    uint32_t found = G0;
    if (full) {
      found = min(lb[i], G0);
    } else {
      for (uint32_t g0 = 0; g0 < G0; g0 += 32) {
        const uint32_t g = g0 + lane;
        const bool ok = g < G0 && row_accepts_n(t, rows + static_cast<size_t>(g) * (2 * W), W);
        const unsigned b = __ballot_sync(0xffffffffu, ok);
        if (b) {
          found = g0 + __ffs(b) - 1;
          break;
        }
      }
    }
    __syncwarp();
    if (lane == 0) lb[i] = found;
    if (full) {
      const uint32_t g = found + lane;
      const bool ok = g < G0 && members_commute_n(t, trows, next, first[g], W);
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (lane == 0) lbm[i] = m;
    }
  }
}

// place_qwc for any width, basis rows in global memory (lane g % 32 owns row g)
__device__ uint32_t place_qwc_n(const uint64_t* st, const uint32_t* slb, uint32_t* sgid, uint32_t n, uint32_t G,
                                uint64_t* B, int W) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t rw = 2 * static_cast<size_t>(W);
  uint32_t k = 0;
  while (k < n) {
    uint32_t l = 0;
    for (; k < n; ++k) {
      const uint64_t* t = st + k * rw;
      l = slb[k];
      const uint32_t g = l + ((lane - l) & 31u);
      const bool ok = g < G && row_accepts_n(t, B + g * rw, W);
      const uint32_t best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
      if (best == UINT_MAX) break;
      if (best % 32 == lane)
        for (size_t e = 0; e < rw; ++e) B[best * rw + e] |= t[e];
      if (lane == 0) sgid[k] = best;
    }
    if (k >= n) break;
    const uint64_t* t = st + k * rw;
    uint32_t best = UINT_MAX;
    for (uint32_t g0 = l + 32; best == UINT_MAX && g0 < G; g0 += 32) {
      const uint32_t g = g0 + ((lane - g0) & 31u);
      const bool ok = g < G && row_accepts_n(t, B + g * rw, W);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    const bool fresh = best == UINT_MAX;
    if (fresh) best = G;
    if (best % 32 == lane)
      for (size_t e = 0; e < rw; ++e) B[best * rw + e] = fresh ? t[e] : (B[best * rw + e] | t[e]);
    if (fresh) ++G;
    if (lane == 0) sgid[k] = best;
    ++k;
  }
  return G;
}

// place_full for any width
__device__ uint32_t place_full_n(const uint64_t* __restrict__ trows, const uint64_t* st, const uint32_t* slb,
                                 const uint32_t* smask, uint32_t* sgid, uint32_t n, uint32_t c0, uint32_t G0,
                                 uint32_t* first, uint32_t* last, uint32_t* next, int W) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t rw = 2 * static_cast<size_t>(W);
  uint32_t G = G0;
  auto chunk_members_commute = [&](const uint64_t* t, uint32_t g, uint32_t k) {
    for (uint32_t q = 0; q < k; ++q)
      if (sgid[q] == g && anticommutes_n(t, st + q * rw, W)) return false;
    return true;
  };
  auto place = [&](uint32_t k, uint32_t best, bool fresh) {
    if ((k & 31u) == lane) sgid[k] = best;
    if (lane == 0) {
      const uint32_t i = c0 + k;
      next[i] = UINT_MAX;
      if (fresh) first[best] = i;
      else next[last[best]] = i;
      last[best] = i;
    }
  };
  uint32_t k = 0;
  while (k < n) {
    uint32_t l = 0;
    for (; k < n; ++k) {
      const uint64_t* t = st + k * rw;
      l = slb[k];
      if (l >= G0) break;
      bool bad = false;
      for (uint32_t q = lane; q < k; q += 32)
        if (sgid[q] == l && anticommutes_n(t, st + q * rw, W)) bad = true;
      if (__any_sync(0xffffffffu, bad)) break;
      place(k, l, false);
    }
    if (k >= n) break;
    __syncwarp();
    const uint64_t* t = st + k * rw;
    const uint32_t m = smask[k];
    uint32_t best = UINT_MAX;
    {
      const uint32_t g = l + lane;
      const bool ok = l < G0 && lane > 0 && g < G0 && ((m >> lane) & 1u) && chunk_members_commute(t, g, k);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    for (uint32_t g0 = l + 32; best == UINT_MAX && g0 < G0; g0 += 32) {
      const uint32_t g = g0 + lane;
      const bool ok = g < G0 && members_commute_n(t, trows, next, first[g], W);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    for (uint32_t g0 = G0; best == UINT_MAX && g0 < G; g0 += 32) {
      const uint32_t g = g0 + lane;
      const bool ok = g < G && chunk_members_commute(t, g, k);
      best = __reduce_min_sync(0xffffffffu, ok ? g : UINT_MAX);
    }
    const bool fresh = best == UINT_MAX;
    if (fresh) best = G;
    place(k, best, fresh);
    if (fresh) ++G;
    __syncwarp();
    ++k;
  }
  return G;
}

// group_resolve_kernel for any width: stages up to `cap_terms` term rows
__global__ void __launch_bounds__(kResolveThreads) group_resolve_n_kernel(
    const uint64_t* __restrict__ trows, int W, uint32_t c0, uint32_t c1, uint32_t cap_terms, uint64_t* rows,
    uint32_t* first, uint32_t* last, uint32_t* next, const uint32_t* __restrict__ lb,
    const uint32_t* __restrict__ lbm, uint32_t* __restrict__ group_of, uint32_t* __restrict__ n_groups, int full) {
  extern __shared__ __align__(16) unsigned char nraw[];
  const size_t rw = 2 * static_cast<size_t>(W);
  const uint32_t n = c1 - c0;
  uint64_t* st = reinterpret_cast<uint64_t*>(nraw);
  uint32_t* slb = reinterpret_cast<uint32_t*>(st + static_cast<size_t>(cap_terms) * rw);
  uint32_t* sgid = slb + cap_terms;
  uint32_t* smask = sgid + cap_terms;
  const uint32_t G0 = *n_groups;
  for (size_t k = threadIdx.x; k < n * rw; k += blockDim.x) st[k] = trows[static_cast<size_t>(c0) * rw + k];
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    slb[k] = lb[c0 + k];
    if (full) smask[k] = lbm[c0 + k];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const uint32_t G = full ? place_full_n(trows, st, slb, smask, sgid, n, c0, G0, first, last, next, W)
                            : place_qwc_n(st, slb, sgid, n, G0, rows, W);
    if (threadIdx.x == 0) *n_groups = G;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) group_of[c0 + k] = sgid[k];
}

void run_greedy_n(int device, bool full, int W, const uint64_t* trows, uint32_t T, uint64_t* rows, uint32_t* first,
                  uint32_t* last, uint32_t* next, uint32_t* lb, uint32_t* lbm, uint32_t* gid, uint32_t* ng,
                  cudaStream_t s) {
  const auto& props = wg::device_props(device);
  const size_t per_term = 16 * static_cast<size_t>(W) + 12;  // staged row, bound, group id, bound mask
  const size_t smem_max = static_cast<size_t>(props.max_smem_optin);
  const uint32_t want = full ? kChunkFull : kChunk;
  const uint32_t chunk = static_cast<uint32_t>(std::min<size_t>(want, smem_max / per_term));
  if (chunk == 0) wg::throw_invalid("group_commuting: a term row does not fit in shared memory");
  const size_t smem = static_cast<size_t>(chunk) * per_term;
  wg::check_cuda(cudaFuncSetAttribute(group_resolve_n_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)),
                 "set group resolve shared memory");
  wg::check_cuda(cudaMemsetAsync(ng, 0, 4, s), "clear group count");
  const unsigned max_blocks = static_cast<unsigned>(props.sm_count) * 8;
  for (uint32_t c0 = 0; c0 < T; c0 += chunk) {
    const uint32_t c1 = T - c0 > chunk ? c0 + chunk : T;
    const unsigned blocks = std::min<unsigned>(max_blocks, (c1 - c0 + kBoundThreads / 32 - 1) / (kBoundThreads / 32));
    if (full) {
      wg::check_cuda(cudaMemsetAsync(lb + c0, 0xff, 4 * static_cast<size_t>(c1 - c0), s), "clear bounds");
      const unsigned sblocks = std::min<unsigned>(
          max_blocks, ((c1 - c0) * kBoundSplit + kBoundThreads / 32 - 1) / (kBoundThreads / 32));
      WG_TIMED("group_search_full_n_kernel", s,
        group_search_full_n_kernel<<<sblocks, kBoundThreads, 0, s>>>(trows, W, c0, c1, first, next, ng, lb));
      wg::check_launch("launch group bound search");
    }
    WG_TIMED("group_bound_n_kernel", s,
      group_bound_n_kernel<<<blocks, kBoundThreads, 0, s>>>(trows, W, c0, c1, rows, first, next, ng, lb, lbm,
                                                            full ? 1 : 0));
    wg::check_launch("launch group bounds");
    WG_TIMED("group_resolve_n_kernel", s,
      group_resolve_n_kernel<<<1, kResolveThreads, smem, s>>>(trows, W, c0, c1, chunk, rows, first, last, next, lb,
                                                              lbm, gid, ng, full ? 1 : 0));
    wg::check_launch("launch group resolve");
  }
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
    wg::Scratch rows(16 * Wa * T, s), first(4 * T, s), last(4 * T, s), next(4 * T, s), lb(4 * T, s), lbm(4 * T, s),
        gid(4 * T, s), ng(4, s);
    const bool full = mode_full != 0;
    const uint32_t T32 = static_cast<uint32_t>(T);
    wg::Scratch trows(W > 4 ? 16 * Wa * T : 0, s);
    if (W > 4) {
      WG_TIMED("interleave_rows_kernel", s,
        interleave_rows_kernel<<<wg::grid_for(T * W, kThreads, device, 4), kThreads, 0, s>>>(
            ox.as<uint64_t>(), oz.as<uint64_t>(), T, W, trows.as<uint64_t>()));
      wg::check_launch("launch interleave rows");
    }
    auto greedy = [&](uint32_t chunk) {
      auto* r = rows.as<uint64_t>();
      auto* f = first.as<uint32_t>();
      auto* l = last.as<uint32_t>();
      auto* nx = next.as<uint32_t>();
      auto* b = lb.as<uint32_t>();
      auto* bm = lbm.as<uint32_t>();
      auto* gi = gid.as<uint32_t>();
      auto* n = ng.as<uint32_t>();
      const uint64_t* px = ox.as<uint64_t>();
      const uint64_t* pz = oz.as<uint64_t>();
      switch (W) {
        case 0:
        case 1: run_greedy<1>(device, full, px, pz, T32, r, f, l, nx, b, bm, gi, n, s, chunk); break;
        case 2: run_greedy<2>(device, full, px, pz, T32, r, f, l, nx, b, bm, gi, n, s, chunk); break;
        case 3: run_greedy<3>(device, full, px, pz, T32, r, f, l, nx, b, bm, gi, n, s, chunk); break;
        case 4: run_greedy<4>(device, full, px, pz, T32, r, f, l, nx, b, bm, gi, n, s, chunk); break;
        default: run_greedy_n(device, full, W, trows.as<uint64_t>(), T32, r, f, l, nx, b, bm, gi, n, s); break;
      }
    };
    if (W <= 4) {
      // chunk length: the autotuner's choice for (mode, words, log2 terms)
      const uint32_t* cands = full ? kFullChunks : kQwcChunks;
      bool done = false;
      const int choice = wg::tune_choose(
          full ? wg::kTuneGroupFull : wg::kTuneGroupQwc, W, wg::ceil_log2(T), 0, full ? 1 : 2, true, s,
          [&](int c) {
            greedy(cands[c]);
            return true;
          },
          &done);
      if (!done) greedy(cands[choice]);
    } else {
      greedy(0);
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
