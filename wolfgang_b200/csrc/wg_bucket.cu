// wg_bucket.cu -- bucketed sort-reduce for products and simplify (1 or 2 mask words).
//
// Same results as the LSD pipeline of wg_simplify.cu (equal keys summed in
// input-index order, glibc-exact cull, canonical key order) with far less data
// movement.  An item is only its 32-bit index (a product l*n_r + r, or an input
// term); its key and coefficient are recomputed from the packed operands, which
// stay in L2, whenever they are needed.
//
// Compressed keys.  The significant bits (the OR of all keys) are numbered by
// rank from the most significant end (word 0, bit 63 first).  A key compressed
// to its significant bits, rank r at bit 63 - r%64 of word r/64, orders like the
// key itself (the other bits are zero in every key).  Compression is linear
// over XOR, so a product's compressed key is the XOR of its factors'.
//
// Codes.  Items of one bucket share their first L ranks.  The 64-bit code of a
// compressed key relative to L is
//   dense     (when at most 64 ranks remain): bits L .. L+63 -- exact;
//   position  (otherwise): one byte per set bit of rank >= L, the first eight
//             of them, each 255 - (rank - L), padded with zero bytes.
// Both agree with the key order wherever codes differ (a < b implies
// code(a) <= code(b)), so a partition of items by code ranges is a partition
// by key ranges, and the common prefix of a code range gives the L of the
// bucket below it.  Equal position codes are told apart by the next eight set
// bits, then, rarely, by the full key.
//
//  coarse  sample codes (L = 0), sort, pick splitters; each item finds its
//          coarse bucket by binary search over the splitters in shared memory
//          and its index is scattered into that bucket's region;
//  fine    one CTA per coarse bucket: sample in-bucket codes, sort them in
//          shared memory, pick fine splitters (a heavily repeated code gets a
//          bucket of its own), count, then write (code relative to the fine
//          bucket's L, index) in fine order;
//  final   fine buckets in global order, at most kCap items each: shared-memory
//          merge sort by (code, index), tie runs reordered by (next code,
//          index) and if need be by (key, index); every item's coefficient is
//          formed, equal-key runs are summed left to right from shared memory
//          and culled, and the survivors (index, sum) are compacted at the
//          start of the bucket's record range with their count.  A bucket of
//          one key above kCap items has its indices radix-sorted in global
//          memory instead and is summed by one thread;
//  output  after a scan of the counts, one warp per fine bucket copies its
//          survivors to their ranks, each key rebuilt from its operands.
//
// Anything outside this path's limits (more than 255 significant bits, a
// coarse region or fine bucket over capacity, a tie of more than 16 different
// keys) makes the driver return false and the caller runs the LSD pipeline.

#include <cuda_runtime.h>

#include <climits>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "wg_common.cuh"
#include "wg_scan.cuh"

namespace {

using wgd::c128;

constexpr int kCoarseLog = 18;           // about 2^18 items per coarse bucket
constexpr int kCoarseMax = 2048;         // coarse buckets
constexpr int kCoarseSample = 128;       // samples per coarse bucket
constexpr int kFineAvg = 896;            // target items per fine bucket (default; settable at run time)
constexpr int kFineMax = 640;            // target fine buckets per coarse bucket
constexpr int kFineSlots = 832;          // fine bucket slots per coarse bucket (targets + isolated codes)
constexpr int kSample2 = 8192;           // in-bucket sample for fine splitters (about 28 per fine bucket)
constexpr int kRefineRounds = 4;         // rounds of extra splitters for fine buckets over capacity
constexpr int kRefineMax = 32;           // fine buckets split in one round
constexpr int kHeavyRun = 3;             // sample repeats that may isolate a code
constexpr int kK1Threads = 512;
constexpr int kK1Items = 16;
constexpr int kK2Threads = 512;
constexpr int kK3Threads = 256;
constexpr int kK3PerSM = 4;                     // final-kernel CTAs resident per SM
constexpr int kIPT = 8;                         // most records per thread in the final sort network
constexpr int kCap = kK3Threads * kIPT;         // 2048 items per fine bucket
constexpr int kPadded = kCap + kCap / 16;       // one spare slot per 16 (bank spread)
constexpr int kWords = kCap / 32;
constexpr int kMaxRuns = kCap / 2;              // tie runs per bucket (runs have >= 2 items)
constexpr int kDistinct = 16;                   // distinct keys in one tie of 16-digit codes
constexpr uint32_t kExactBit = 1u << 31;        // fine bucket codes are exact (equal code = equal key)
constexpr uint32_t kPureBit = 1u << 30;         // every key of the fine bucket is equal
constexpr uint32_t kCountMask = kPureBit - 1;
constexpr unsigned kFlagOverrun = 4u;           // an output rank beyond capacity (internal error)
constexpr unsigned kFlagCoarseFull = 8u;        // fallbacks: a coarse region over capacity,
constexpr unsigned kFlagFineFull = 16u;         //   a fine bucket over kCap items (not of one key),
constexpr unsigned kFlagDistinct = 32u;         //   a tie of more than kDistinct keys
constexpr unsigned kFallbackMask = kFlagCoarseFull | kFlagFineFull | kFlagDistinct;

struct Control {
  unsigned k2_ticket;
  unsigned k3_ticket;
  unsigned flags;
  unsigned inf_seen;
  unsigned long long max_bits;
  double thr;
  unsigned long long survivors;
  unsigned fine_total;
  unsigned max_fine;             // largest fine bucket
  unsigned long long tie_items;  // items in runs of equal 8-digit codes (traced runs)
  unsigned refined;              // fine buckets split again after counting
  unsigned long long phase[4];   // final-kernel cycles per phase (traced runs)
  unsigned long long fphase[5];  // fine-kernel cycles per phase (traced runs)
  unsigned long long digits[9];  // traced runs: fine buckets by the number of 8-bit code digits that vary
};

// ------------------------------------------------------------------ keys and codes

template <int KW>
__device__ __forceinline__ bool keq(const uint64_t (&a)[KW], const uint64_t (&b)[KW]) {
  bool e = true;
#pragma unroll
  for (int i = 0; i < KW; ++i) e = e && (a[i] == b[i]);
  return e;
}

template <int KW>
__device__ __forceinline__ bool kless(const uint64_t (&a)[KW], const uint64_t (&b)[KW]) {
#pragma unroll
  for (int i = 0; i < KW; ++i)
    if (a[i] != b[i]) return a[i] < b[i];
  return false;
}

// Bits L .. L+63 of a compressed key (zero past its end).
template <int KW>
__device__ __forceinline__ uint64_t window64(const uint64_t (&c)[KW], int L) {
  const int w = L >> 6, s = L & 63;
  uint64_t hi = 0, lo = 0;
#pragma unroll
  for (int i = 0; i < KW; ++i) {
    if (i == w) hi = c[i];
    if (i == w + 1) lo = c[i];
  }
  return s == 0 ? hi : (hi << s) | (lo >> (64 - s));
}

// Position digits skip .. skip+7 of the set bits of rank >= L.
template <int KW>
__device__ __forceinline__ uint64_t position_code(const uint64_t (&c)[KW], int L, int skip) {
  uint64_t code = 0;
  int nd = 0;
#pragma unroll
  for (int w = 0; w < KW; ++w) {
    const int r0 = 64 * w;
    uint64_t v = c[w];
    if (L >= r0 + 64) v = 0;
    else if (L > r0) v &= ~0ull >> (L - r0);
    while (v && nd < skip + 8) {
      const int b = __clzll(v);
      v &= ~(0x8000000000000000ull >> b);
      if (nd >= skip) code |= static_cast<uint64_t>(255 - (r0 + b - L)) << (56 - 8 * (nd - skip));
      ++nd;
    }
  }
  return code;
}

template <int KW>
__device__ __forceinline__ uint64_t code_of(const uint64_t (&c)[KW], int L, bool dense) {
  return dense ? window64<KW>(c, L) : position_code<KW>(c, L, 0);
}

__device__ __forceinline__ bool dense_at(int total, int L) { return total - L <= 64; }

// Ranks shared by every key whose code (relative to L) lies in [lo, hi].
__device__ __forceinline__ int child_prefix(int L, bool dense, int total, uint64_t lo, uint64_t hi) {
  const uint64_t d = lo ^ hi;
  if (dense) return min(total, L + (d ? __clzll(d) : 64));
  const int m = d ? (__clzll(d) >> 3) : 8;
  int Lc = L;
  for (int q = 0; q < m; ++q) {
    const int digit = static_cast<int>((lo >> (56 - 8 * q)) & 0xffu);
    if (digit == 0) return total;  // no further set bits: the keys are equal
    Lc = L + (255 - digit) + 1;
  }
  return min(Lc, total);
}

// Code range [lo, hi] of bucket j under ns sorted splitters (bucket j holds
// codes c with split[j-1] <= c < split[j]); false when it is empty.
__device__ __forceinline__ bool bucket_range(const uint64_t* split, int ns, int j, uint64_t& lo, uint64_t& hi) {
  lo = j > 0 ? split[j - 1] : 0ull;
  if (j < ns) {
    if (split[j] == 0ull) return false;
    hi = split[j] - 1;
  } else {
    hi = ~0ull;
  }
  return lo <= hi;
}

// Number of sorted splitters a[0..n) whose top 12 bits are below h, for every
// h in 0 .. 4096: the splitters sharing a code's top 12 bits are
// a[tbl[h] .. tbl[h+1]).  Built by the block.
constexpr int kTopBits = 12;
__device__ __forceinline__ void build_top_table(const uint64_t* a, int n, uint16_t* tbl) {
  for (int h = threadIdx.x; h <= (1 << kTopBits); h += blockDim.x) {
    const uint64_t v = static_cast<uint64_t>(h) << (64 - kTopBits);
    int lo = 0, hi = n;
    if (h == (1 << kTopBits)) {
      lo = n;
    } else {
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
      }
    }
    tbl[h] = static_cast<uint16_t>(lo);
  }
}

__device__ __forceinline__ int upper_bound_u64(const uint64_t* a, int n, uint64_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (v < a[mid]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// First position in the sorted a[0..n) whose value is not below v.
__device__ __forceinline__ int lower_bound_u64(const uint64_t* a, int n, uint64_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// upper_bound_u64 through the top-12-bit table: only the splitters that share
// v's top bits are searched.
__device__ __forceinline__ int upper_bound_top(const uint64_t* a, const uint16_t* tbl, uint64_t v) {
  const int h = static_cast<int>(v >> (64 - kTopBits));
  int lo = tbl[h], hi = tbl[h + 1];
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (v < a[mid]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// ------------------------------------------------------------------ item sources

// Exact quotient p / d for p, d < 2^32: m = ceil(2^64 / d), and the error of
// p*m / 2^64 stays below 2^-32 <= 1/d, under the gap to the next integer.
struct FastDiv {
  uint32_t d;
  uint64_t m;
  __device__ __forceinline__ uint32_t div(uint32_t p) const {
    return d == 1 ? p : static_cast<uint32_t>(__umul64hi(static_cast<uint64_t>(p), m));
  }
};

// Operand records: [t][KW + 2] words, the key (x0, z0, x1, z1 in significance
// order) then the coefficient's re and im bits; KW + 2 is even, so every
// record starts on 16 bytes and moves as 128-bit loads.
template <int KW>
__device__ __forceinline__ void load_key(const uint64_t* rec, uint32_t t, uint64_t (&k)[KW]) {
  const ulonglong2* r = reinterpret_cast<const ulonglong2*>(rec + static_cast<size_t>(t) * (KW + 2));
#pragma unroll
  for (int i = 0; i < KW / 2; ++i) {
    const ulonglong2 v = __ldg(r + i);
    k[2 * i] = v.x;
    k[2 * i + 1] = v.y;
  }
}

template <int KW>
__device__ __forceinline__ c128 load_coeff(const uint64_t* rec, uint32_t t) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(rec + static_cast<size_t>(t) * (KW + 2) + KW));
  return {v.x, v.y};
}

// Compressed keys [t][KW] (KW even: 16-byte rows).
template <int KW>
__device__ __forceinline__ void load_ckey(const uint64_t* c2, uint32_t t, uint64_t (&k)[KW]) {
  const ulonglong2* r = reinterpret_cast<const ulonglong2*>(c2 + static_cast<size_t>(t) * KW);
#pragma unroll
  for (int i = 0; i < KW / 2; ++i) {
    const ulonglong2 v = __ldg(r + i);
    k[2 * i] = v.x;
    k[2 * i + 1] = v.y;
  }
}

// Products p = a*nb + b of two packed operands (rhs acts first).
template <int KW>
struct ProdSrc {
  const uint64_t* arec;  // [na][KW + 2]
  const uint64_t* brec;  // [nb][KW + 2]
  const uint64_t* ac2;   // [na][KW] compressed keys
  const uint64_t* bc2;   // [nb][KW]
  FastDiv nb;

  __device__ __forceinline__ void ckey(uint32_t p, uint64_t (&c)[KW]) const {
    const uint32_t a = nb.div(p), b = p - a * nb.d;
    uint64_t ca[KW], cb[KW];
    load_ckey<KW>(ac2, a, ca);
    load_ckey<KW>(bc2, b, cb);
#pragma unroll
    for (int i = 0; i < KW; ++i) c[i] = ca[i] ^ cb[i];
  }
  __device__ __forceinline__ void key(uint32_t p, uint64_t (&k)[KW]) const {
    const uint32_t a = nb.div(p), b = p - a * nb.d;
    uint64_t ka[KW], kb[KW];
    load_key<KW>(arec, a, ka);
    load_key<KW>(brec, b, kb);
#pragma unroll
    for (int i = 0; i < KW; ++i) k[i] = ka[i] ^ kb[i];
  }
  // Key and coefficient of the product: masks XOR'd, phase exponent
  // e = sum_w [popc(ox&oz) - popc(ax&az) - popc(bx&bz) + 2 popc(ax&bz)] mod 4,
  // coefficient (ca * cb) * i^e.
  __device__ __forceinline__ c128 key_coeff(uint32_t p, uint64_t (&k)[KW]) const {
    const uint32_t a = nb.div(p), b = p - a * nb.d;
    uint64_t ka[KW], kb[KW];
    load_key<KW>(arec, a, ka);
    load_key<KW>(brec, b, kb);
    const c128 ca = load_coeff<KW>(arec, a);
    const c128 cb = load_coeff<KW>(brec, b);
    unsigned e = 0, ya = 0, yb = 0;
#pragma unroll
    for (int i = 0; i < KW; i += 2) {
      k[i] = ka[i] ^ kb[i];
      k[i + 1] = ka[i + 1] ^ kb[i + 1];
      e += __popcll(k[i] & k[i + 1]) + 2u * __popcll(ka[i] & kb[i + 1]);
      ya += __popcll(ka[i] & ka[i + 1]);
      yb += __popcll(kb[i] & kb[i + 1]);
    }
    e += 8u - (ya & 3u) - (yb & 3u);
    return wgd::rotate(wgd::cmul(ca, cb), e);
  }
};

// Input terms of simplify.
template <int KW>
struct TermSrc {
  const uint64_t* trec;  // [n][KW + 2]
  const uint64_t* tc2;   // [n][KW] compressed keys

  __device__ __forceinline__ void ckey(uint32_t p, uint64_t (&k)[KW]) const { load_ckey<KW>(tc2, p, k); }
  __device__ __forceinline__ void key(uint32_t p, uint64_t (&k)[KW]) const { load_key<KW>(trec, p, k); }
  __device__ __forceinline__ c128 key_coeff(uint32_t p, uint64_t (&k)[KW]) const {
    load_key<KW>(trec, p, k);
    return load_coeff<KW>(trec, p);
  }
};

// ------------------------------------------------------------------ packing

// Operand records [t][2W + 2] (key words in significance order, then the
// coefficient) and the OR of every key word into sig.
__global__ void bucket_pack_kernel(const uint64_t* __restrict__ x, const uint64_t* __restrict__ z,
                                   const double* __restrict__ c, size_t T, int W, uint64_t* __restrict__ rec,
                                   unsigned long long* __restrict__ sig) {
  uint64_t acc[4] = {0, 0, 0, 0};
  const int R = 2 * W + 2;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < T;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    for (int w = 0; w < W; ++w) {
      const uint64_t xv = x[t * W + w], zv = z[t * W + w];
      rec[t * R + 2 * w] = xv;
      rec[t * R + 2 * w + 1] = zv;
      acc[2 * w] |= xv;
      acc[2 * w + 1] |= zv;
    }
    rec[t * R + 2 * W] = static_cast<uint64_t>(__double_as_longlong(c[2 * t]));
    rec[t * R + 2 * W + 1] = static_cast<uint64_t>(__double_as_longlong(c[2 * t + 1]));
  }
  for (int i = 0; i < 2 * W; ++i) {
    uint64_t v = acc[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicOr(sig + i, static_cast<unsigned long long>(v));
  }
}

struct SigWords {
  uint64_t w[4];
};

// Compressed keys [t][KW] of the records' keys under the significant bits.
__global__ void bucket_compress_kernel(const uint64_t* __restrict__ rec, size_t T, int KW, SigWords sig,
                                       uint64_t* __restrict__ out) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < T;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint64_t c[4] = {0, 0, 0, 0};
    int base = 0;
    for (int w = 0; w < KW; ++w) {
      uint64_t m = rec[t * (KW + 2) + w] & sig.w[w];
      while (m) {
        const int b = 63 - __clzll(m);
        m ^= uint64_t{1} << b;
        const int r = base + __popcll(sig.w[w] & ~((uint64_t{2} << b) - 1));
        c[r >> 6] |= 0x8000000000000000ull >> (r & 63);
      }
      base += __popcll(sig.w[w]);
    }
    for (int w = 0; w < KW; ++w) out[t * KW + w] = c[w];
  }
}

// ------------------------------------------------------------------ coarse splitters

// splitmix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t v) {
  v += 0x9e3779b97f4a7c15ull;
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
  return v ^ (v >> 31);
}

template <int KW, class Src>
__global__ void bucket_sample_kernel(Src src, uint32_t n, uint32_t S, bool dense, uint64_t* __restrict__ codes,
                                     uint32_t* __restrict__ idx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S; i += gridDim.x * blockDim.x) {
    const uint32_t p = S >= n ? i : static_cast<uint32_t>(__umul64hi(mix64(i), static_cast<uint64_t>(n)));
    uint64_t c[KW];
    src.ckey(p, c);
    codes[i] = code_of<KW>(c, 0, dense);
    idx[i] = i;
  }
}

__global__ void bucket_pick_kernel(const uint64_t* __restrict__ sorted, uint32_t S, int parts,
                                   uint64_t* __restrict__ split) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < parts - 1; j += gridDim.x * blockDim.x)
    split[j] = sorted[(static_cast<uint64_t>(j) + 1) * S / parts];
}

// ------------------------------------------------------------------ coarse scatter

struct CoarseParams {
  const uint64_t* split;  // [B1-1]
  int B1;
  uint32_t capc;          // region capacity per coarse bucket
  unsigned* fill;         // [B1] items per coarse bucket (may exceed capc: overflow)
  uint32_t* idx_out;      // [B1][capc]
  bool dense;
  bool want_max;
  unsigned long long* max_bits;
};

// Tiles of 8192 items: shared-memory histogram ranks, one global reservation
// per (tile, bucket), then the index writes.
template <int KW, class Src>
__global__ void __launch_bounds__(kK1Threads, 2) bucket_coarse_kernel(Src src, uint32_t n, CoarseParams P) {
  __shared__ uint64_t ss[kCoarseMax - 1];
  __shared__ unsigned hist[kCoarseMax];
  __shared__ unsigned base[kCoarseMax];
  __shared__ uint16_t top[(1 << kTopBits) + 1];
  const int ns = P.B1 - 1;
  for (int i = threadIdx.x; i < ns; i += blockDim.x) ss[i] = P.split[i];
  for (int i = threadIdx.x; i < P.B1; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  build_top_table(ss, ns, top);
  __syncthreads();
  double mx = 0.0;
  const uint64_t tile = static_cast<uint64_t>(blockDim.x) * kK1Items;
  for (uint64_t t0 = blockIdx.x * tile; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * tile) {
    uint32_t br[kK1Items];  // bucket << 16 | rank in tile
#pragma unroll
    for (int r = 0; r < kK1Items; ++r) {
      const uint64_t p = t0 + static_cast<uint64_t>(r) * blockDim.x + threadIdx.x;
      const bool valid = p < n;
      int b = 0;
      if (valid) {
        if (P.want_max) {
          uint64_t k[KW];
          const c128 c = src.key_coeff(static_cast<uint32_t>(p), k);
          const double a = wgd::hypot_ref(c.re, c.im);
          if (mx < a) mx = a;  // std::max: a NaN never replaces the running max
        }
        uint64_t c[KW];
        src.ckey(static_cast<uint32_t>(p), c);
        b = upper_bound_top(ss, top, code_of<KW>(c, 0, P.dense));
      }
      const unsigned rk = valid ? atomicAdd(&hist[b], 1u) : 0u;
      br[r] = (static_cast<uint32_t>(b) << 16) | rk;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P.B1; i += blockDim.x) {
      const unsigned c = hist[i];
      base[i] = c ? atomicAdd(P.fill + i, c) : 0u;
      hist[i] = 0;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kK1Items; ++r) {
      const uint64_t p = t0 + static_cast<uint64_t>(r) * blockDim.x + threadIdx.x;
      if (p < n) {
        const unsigned b = br[r] >> 16;
        const unsigned pos = base[b] + (br[r] & 0xffffu);
        if (pos < P.capc) P.idx_out[static_cast<size_t>(b) * P.capc + pos] = static_cast<uint32_t>(p);
      }
    }
    __syncthreads();
  }
  if (P.want_max) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, mx, o);
      if (mx < other) mx = other;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(P.max_bits, static_cast<unsigned long long>(__double_as_longlong(mx)));
  }
}

// ------------------------------------------------------------------ plan

__device__ __forceinline__ unsigned fine_target(unsigned n, unsigned favg) {
  const unsigned f = (n + favg - 1) / favg;
  return f < 1 ? 1u : (f > kFineMax ? static_cast<unsigned>(kFineMax) : f);
}

// Fine bucket slots of a coarse bucket: the target count, a quarter more for
// codes isolated on their own, and a few spare.
__device__ __forceinline__ unsigned fine_slots(unsigned n, unsigned favg) {
  const unsigned t = fine_target(n, favg);
  return t + t / 4 + 8;
}

// Exclusive scan of one value per thread over the block (blockDim.x a multiple
// of 32, at most 1024); the block total is returned through *total.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* warp_tmp, unsigned* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  unsigned incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tmp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const unsigned w = lane < nw ? warp_tmp[lane] : 0u;
    unsigned wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) warp_tmp[lane] = wi - w;
    if (lane == 31) warp_tmp[32] = wi;
  }
  __syncthreads();
  const unsigned r = warp_tmp[warp] + incl - v;
  *total = warp_tmp[32];
  __syncthreads();
  return r;
}

// One block of 1024 threads: coarse bucket sizes -> fine slot numbering, the
// common prefix of every coarse bucket, and the cull threshold.
__global__ void __launch_bounds__(1024) bucket_plan_kernel(const unsigned* __restrict__ fill, int B1, uint32_t capc,
                                                           const uint64_t* __restrict__ split, int total, bool dense0,
                                                           int thr_mode, double atol, double rtol, double thr_fixed,
                                                           unsigned favg, Control* ctl, uint32_t* __restrict__ fine_base,
                                                           int* __restrict__ Lj, uint32_t* __restrict__ order) {
  __shared__ unsigned warp_tmp[33];
  __shared__ uint64_t by_size[kCoarseMax];
  unsigned carry = 0;
  for (int j0 = 0; j0 < B1; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    unsigned slots = 0;
    if (j < B1) {
      const unsigned c = fill[j];
      if (c > capc) atomicOr(&ctl->flags, kFlagCoarseFull);
      slots = fine_slots(min(c, capc), favg);
      uint64_t lo, hi;
      const int L = bucket_range(split, B1 - 1, j, lo, hi) ? child_prefix(0, dense0, total, lo, hi) : total;
      Lj[j] = L | (dense_at(total, L) ? 0x10000 : 0);
    }
    unsigned tot;
    const unsigned ex = block_exclusive_scan(slots, warp_tmp, &tot);
    if (j < B1) fine_base[j] = carry + ex;
    carry += tot;
  }
  // The fine pass takes its coarse buckets largest first (a persistent CTA
  // per ticket): the last tickets are the shortest jobs, which shortens the
  // pass's tail.  B1 is a power of two.
  for (int j = threadIdx.x; j < B1; j += blockDim.x)
    by_size[j] = (static_cast<uint64_t>(~min(fill[j], capc)) << 32) | static_cast<uint32_t>(j);
  __syncthreads();
  for (int size = 2; size <= B1; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < B1 / 2; i += blockDim.x) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const uint64_t x = by_size[lo], y = by_size[hi];
        if (((lo & size) == 0) ? (y < x) : (x < y)) {
          by_size[lo] = y;
          by_size[hi] = x;
        }
      }
      __syncthreads();
    }
  }
  for (int j = threadIdx.x; j < B1; j += blockDim.x) order[j] = static_cast<uint32_t>(by_size[j]);
  if (threadIdx.x == 0) {
    fine_base[B1] = carry;
    ctl->fine_total = carry;
    double thr = thr_fixed;
    if (thr_mode == 1) {
      const double mx = __longlong_as_double(static_cast<long long>(ctl->max_bits));
      thr = wgd::add(atol, wgd::mul(rtol, mx));
    } else if (thr_mode == 2) {
      thr = atol;
    }
    ctl->thr = thr;
  }
}

// ------------------------------------------------------------------ fine partition

struct FineParams {
  const unsigned* fill;
  uint32_t capc;
  int B1;
  int total;
  const uint32_t* fine_base;  // [B1+1]
  const int* Lj;              // prefix | dense << 16
  const uint32_t* idx_in;     // [B1][capc]
  uint16_t* fid_tmp;          // [B1][capc] fine bucket of each item
  uint32_t rstride;           // record region per coarse bucket (multiple of 32); 0: one-pass layout
  uint64_t* rec_code;         // records in fine-bucket order (see bucket_fine_kernel)
  uint32_t* rec_idx;
  uint32_t* fine_start;       // [G]
  uint32_t* fine_count;       // [G] count | kExactBit | kPureBit
  uint16_t* fine_L;           // [G] prefix of the bucket's codes
  Control* ctl;
  unsigned favg;              // target items per fine bucket
  int trace;                  // record per-phase cycles
  const uint32_t* order;      // [B1] coarse buckets, largest first (ticket -> bucket)
};

// Exclusive block scans (blockDim.x a multiple of 32, at most 1024; tmp holds
// 32 ints): the maximum over lower threads (INT_MIN for none) and the minimum
// over higher threads (INT_MAX for none).
__device__ int block_prefix_max_excl(int v, int* tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x = max(x, y);
  }
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nw ? tmp[lane] : INT_MIN;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w = max(w, y);
    }
    int ex = __shfl_up_sync(0xffffffffu, w, 1);
    if (lane == 0) ex = INT_MIN;
    if (lane < nw) tmp[lane] = ex;
  }
  __syncthreads();
  int in_warp = __shfl_up_sync(0xffffffffu, x, 1);
  if (lane == 0) in_warp = INT_MIN;
  const int r = max(tmp[warp], in_warp);
  __syncthreads();
  return r;
}

__device__ int block_suffix_min_excl(int v, int* tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_down_sync(0xffffffffu, x, o);
    if (lane + o < 32) x = min(x, y);
  }
  if (lane == 0) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nw ? tmp[lane] : INT_MAX;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_down_sync(0xffffffffu, w, o);
      if (lane + o < 32) w = min(w, y);
    }
    int ex = __shfl_down_sync(0xffffffffu, w, 1);
    if (lane == 31) ex = INT_MAX;
    if (lane < nw) tmp[lane] = ex;
  }
  __syncthreads();
  int in_warp = __shfl_down_sync(0xffffffffu, x, 1);
  if (lane == 31) in_warp = INT_MAX;
  const int r = min(tmp[warp], in_warp);
  __syncthreads();
  return r;
}

constexpr int kPickChunk = kSample2 / kK2Threads;  // sorted samples per thread in the splitter pick
static_assert(kPickChunk * kK2Threads == kSample2 && kPickChunk <= 31, "splitter pick chunks");

// Prefix (and dense flag) of every fine bucket's codes under ns splitters;
// slots past the last bucket take the full length.
__device__ __forceinline__ void fine_prefixes(const uint64_t* fs, int ns, int slots, int Lp, bool densep, int total,
                                              int* fL) {
  for (int f = threadIdx.x; f < slots; f += blockDim.x) {
    uint64_t lo, hi;
    const int L = f <= ns && bucket_range(fs, ns, f, lo, hi) ? child_prefix(Lp, densep, total, lo, hi) : total;
    fL[f] = L | (dense_at(total, L) ? 0x10000 : 0);
  }
}

// A splitter v with lo < v <= hi for the fine bucket of codes [lo, hi] (lo <
// hi): the median of the bucket's samples; the next sampled code above lo when
// that median is lo itself, or lo + 1 when there is none; the middle of the
// range when no sample falls in it.
__device__ uint64_t refine_splitter(const uint64_t* samp, int S2, uint64_t lo, uint64_t hi) {
  const int a = lower_bound_u64(samp, S2, lo);
  const int b = upper_bound_u64(samp, S2, hi);
  if (a >= b) return lo + (hi - lo) / 2 + 1;
  const uint64_t m = samp[a + (b - a) / 2];
  if (m > lo) return m;
  const int c = a + upper_bound_u64(samp + a, b - a, lo);
  return c < b ? samp[c] : lo + 1;
}

constexpr int kSplitBit = 0x40000000;  // fL flag during refinement: the bucket was split

constexpr size_t kK2Smem = sizeof(uint64_t) * (kSample2 + kFineSlots) + sizeof(int) * kFineSlots +
                           sizeof(unsigned) * kFineSlots + sizeof(uint16_t) * ((1 << kTopBits) + 8);

// Ascending bitonic sort of n (a power of two) words in shared memory.
__device__ void smem_bitonic_u64(uint64_t* a, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < n / 2; i += blockDim.x) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const uint64_t x = a[lo], y = a[hi];
        const bool up = (lo & size) == 0;
        if (up ? (y < x) : (x < y)) {
          a[lo] = y;
          a[hi] = x;
        }
      }
      __syncthreads();
    }
  }
}

template <int KW, class Src>
__global__ void __launch_bounds__(kK2Threads) bucket_fine_kernel(Src src, FineParams P) {
  extern __shared__ __align__(16) unsigned char k2raw[];
  uint64_t* samp = reinterpret_cast<uint64_t*>(k2raw);
  uint64_t* fs = samp + kSample2;
  int* fL = reinterpret_cast<int*>(fs + kFineSlots);
  unsigned* cnt = reinterpret_cast<unsigned*>(fL + kFineSlots);
  uint16_t* ftop = reinterpret_cast<uint16_t*>(cnt + kFineSlots);  // top-bit table of the fine splitters
  __shared__ unsigned s_job;
  __shared__ int s_ns;
  __shared__ unsigned warp_tmp[33];
  __shared__ int s_scan[32];
  __shared__ long long s_tp[6];
  __shared__ unsigned s_nfix;
  __shared__ int s_fixf[kRefineMax];
  __shared__ uint64_t s_fixv[kRefineMax];
  __shared__ int s_over;  // one-pass layout: a fine bucket got more than kCap items
  const int total = P.total;
  while (true) {
    if (P.trace && threadIdx.x == 0) s_tp[0] = clock64();
    if (threadIdx.x == 0) s_job = atomicAdd(&P.ctl->k2_ticket, 1u);
    __syncthreads();
    const int ticket = static_cast<int>(s_job);
    __syncthreads();
    if (ticket >= P.B1) break;
    const int j = static_cast<int>(P.order[ticket]);
    const uint32_t n = min(P.fill[j], P.capc);
    const size_t base = static_cast<size_t>(j) * P.capc;
    // One-pass layout (rstride 0): fine slot f of this coarse bucket owns
    // records [(fine_base[j] + f) * kCap, + kCap), and pass 1 writes every item
    // there as it counts it; a coarse bucket with a fine bucket over kCap
    // items falls back to the two passes, packing its fine buckets 32-aligned
    // from the start of its region (slots * kCap records: room enough).
    // Otherwise each coarse bucket owns rstride records, packed the same way.
    const bool one_pass = P.rstride == 0;
    const size_t rbase = one_pass ? static_cast<size_t>(P.fine_base[j]) * kCap : static_cast<size_t>(j) * P.rstride;
    const uint32_t g0 = P.fine_base[j];
    const int slots = static_cast<int>(P.fine_base[j + 1] - g0);
    const int target = static_cast<int>(fine_target(n, P.favg));
    const int Lp = P.Lj[j] & 0xffff;
    const bool densep = (P.Lj[j] >> 16) & 1;
    // random sample of codes relative to the coarse prefix, sorted
    const int S2 = static_cast<int>(n < static_cast<uint32_t>(kSample2) ? n : static_cast<uint32_t>(kSample2));
    int SP = 1;
    while (SP < S2) SP <<= 1;
    for (int t = threadIdx.x; t < SP; t += blockDim.x) {
      uint64_t code = ~0ull;
      if (t < S2) {
        const uint32_t pos = S2 == static_cast<int>(n)
                                 ? static_cast<uint32_t>(t)
                                 : static_cast<uint32_t>(__umul64hi(mix64((static_cast<uint64_t>(j) << 32) | t), n));
        uint64_t c[KW];
        src.ckey(P.idx_in[base + pos], c);
        code = code_of<KW>(c, Lp, densep);
      }
      samp[t] = code;
    }
    __syncthreads();
    smem_bitonic_u64(samp, SP);
    if (P.trace && threadIdx.x == 0) s_tp[1] = clock64();
    // Splitters.  Runs of equal codes in the sorted sample are never cut.  A
    // bucket boundary goes at the first run that starts in each window of
    // `share` samples; a code whose sample run stands for a quarter of kCap
    // items or more (a heavily repeated key) gets a bucket of its own,
    // [c, c + 1).  Every thread takes kPickChunk consecutive samples; scans
    // find the run starts around each chunk and the output positions.
    {
      const int share = max(1, S2 / target);
      const int t = threadIdx.x;
      uint32_t rs = 0;
      int first_rs = INT_MAX, last_rs = -1;
#pragma unroll
      for (int k = 0; k < kPickChunk; ++k) {
        const int i = t * kPickChunk + k;
        if (i < S2 && (i == 0 || samp[i] != samp[i - 1])) {
          rs |= 1u << k;
          first_rs = min(first_rs, i);
          last_rs = i;
        }
      }
      const int prev_in = block_prefix_max_excl(last_rs, s_scan);
      const int next_in = min(block_suffix_min_excl(first_rs, s_scan), S2);
      // splitters this thread emits: pass 0 counts them, pass 1 writes them
      unsigned cnt = 0, off = 0, total = 0;
      for (int pass = 0; pass < 2; ++pass) {
        int prev = prev_in;
        unsigned o = off;
#pragma unroll
        for (int k = 0; k < kPickChunk; ++k) {
          if (!((rs >> k) & 1u)) continue;
          const int i = t * kPickChunk + k;
          const uint32_t later = rs & ~((2u << k) - 1u);
          const int r = (later ? t * kPickChunk + __ffs(later) - 1 : next_in) - i;
          const uint64_t v = samp[i];
          const bool heavy =
              r >= kHeavyRun && static_cast<uint64_t>(r) * n >= static_cast<uint64_t>(kCap / 4) * S2 && v != ~0ull;
          const bool regular = i > 0 && (i / share) != (prev / share);
          if (pass == 0) {
            cnt += heavy ? (i > 0 ? 2u : 1u) : (regular ? 1u : 0u);
          } else {
            if ((heavy && i > 0) || (!heavy && regular)) fs[o++] = v;
            if (heavy) fs[o++] = v + 1;
          }
          prev = i;
        }
        if (pass == 0) {
          off = block_exclusive_scan(cnt, warp_tmp, &total);
          if (total > static_cast<unsigned>(slots - 1)) break;  // uniform: the greedy pick below instead
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        if (total <= static_cast<unsigned>(slots - 1)) {
          s_ns = static_cast<int>(total);
        } else {
          // greedy, one thread: a bucket closes after the run that brings it
          // to its share; heavy runs isolated while slots remain
          int ns = 0, acc = 0, i = 0;
          while (i < S2 && ns < slots - 1) {
            const uint64_t v = samp[i];
            int r = 1;
            while (i + r < S2 && samp[i + r] == v) ++r;
            const bool heavy =
                r >= kHeavyRun && static_cast<uint64_t>(r) * n >= static_cast<uint64_t>(kCap / 4) * S2;
            if (heavy && v != ~0ull && ns + 2 <= slots - 1) {
              if (acc > 0 && (ns == 0 || fs[ns - 1] < v)) fs[ns++] = v;
              fs[ns++] = v + 1;
              acc = 0;
            } else {
              acc += r;
              if (acc >= share && i + r < S2) {
                fs[ns++] = samp[i + r];
                acc = 0;
              }
            }
            i += r;
          }
          s_ns = ns;
        }
        if (P.trace) s_tp[2] = clock64();
      }
    }
    __syncthreads();
    fine_prefixes(fs, s_ns, slots, Lp, densep, total, fL);
    for (int f = threadIdx.x; f < slots; f += blockDim.x) cnt[f] = 0;
    build_top_table(fs, s_ns, ftop);
    __syncthreads();
    // pass 1: fine bucket of every item; in the one-pass layout also its
    // record (code relative to the fine prefix, index) at its fine slot
    for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x) {
      const uint32_t t = t0 + threadIdx.x;
      if (t < n) {
        const uint32_t p = P.idx_in[base + t];
        uint64_t c[KW];
        src.ckey(p, c);
        const int f = upper_bound_top(fs, ftop, code_of<KW>(c, Lp, densep));
        if (!one_pass) P.fid_tmp[base + t] = static_cast<uint16_t>(f);
        const unsigned slot = atomicAdd(&cnt[f], 1u);
        if (one_pass && slot < static_cast<unsigned>(kCap)) {
          const int Lf = fL[f];
          const size_t r = rbase + static_cast<size_t>(f) * kCap + slot;
          P.rec_code[r] = code_of<KW>(c, Lf & 0xffff, (Lf >> 16) & 1);
          P.rec_idx[r] = p;
        }
      }
    }
    if (threadIdx.x == 0) s_over = 0;
    __syncthreads();
    if (one_pass) {
      for (int f = threadIdx.x; f < slots; f += blockDim.x)
        if (cnt[f] > static_cast<unsigned>(kCap)) s_over = 1;
    }
    __syncthreads();
    const bool placed = one_pass && s_over == 0;
    if (one_pass && !placed) {
      // the packed fallback needs every item's fine bucket: count again,
      // keeping them (the one pass did not store them)
      for (int f = threadIdx.x; f < slots; f += blockDim.x) cnt[f] = 0;
      __syncthreads();
      for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        if (t < n) {
          uint64_t c[KW];
          src.ckey(P.idx_in[base + t], c);
          const int f = upper_bound_top(fs, ftop, code_of<KW>(c, Lp, densep));
          P.fid_tmp[base + t] = static_cast<uint16_t>(f);
          atomicAdd(&cnt[f], 1u);
        }
      }
      __syncthreads();
    }
    // Refinement.  The sample puts about 2.5 times the mean into the largest of
    // a million fine buckets; one over kCap items whose range holds more than
    // one code gets one more splitter from its own samples (refine_splitter),
    // up to kRefineMax buckets a round.  Only the split buckets' items are
    // searched again; every other item's bucket id moves up by the number of
    // splitters inserted below it.  A bucket still over capacity after
    // kRefineRounds rounds, or with no room left for a splitter, is flagged by
    // the final kernel, as before.
    for (int round = 0; round < kRefineRounds; ++round) {
      const int ns = s_ns;
      if (threadIdx.x == 0) s_nfix = 0;
      __syncthreads();
      for (int f = threadIdx.x; f <= ns; f += blockDim.x) {
        uint64_t lo, hi;
        if (cnt[f] > static_cast<unsigned>(kCap) && bucket_range(fs, ns, f, lo, hi) && lo < hi) {
          const unsigned q = atomicAdd(&s_nfix, 1u);
          if (q < static_cast<unsigned>(kRefineMax)) s_fixf[q] = f;
        }
      }
      __syncthreads();
      if (s_nfix == 0) break;
      __syncthreads();
      if (threadIdx.x == 0) {
        // the split buckets in ascending order, as many as there are free slots
        const int m = min(min(static_cast<int>(s_nfix), kRefineMax), slots - 1 - ns);
        for (int q = 1; q < m; ++q) {
          const int v = s_fixf[q];
          int r = q;
          for (; r > 0 && s_fixf[r - 1] > v; --r) s_fixf[r] = s_fixf[r - 1];
          s_fixf[r] = v;
        }
        for (int q = 0; q < m; ++q) {
          uint64_t lo, hi;
          bucket_range(fs, ns, s_fixf[q], lo, hi);
          s_fixv[q] = refine_splitter(samp, S2, lo, hi);
        }
        // splitters rewritten in place from the back: bucket b's new splitter
        // goes just before old splitter b; fL[b] takes the shift of bucket b's
        // id and whether it was split
        if (m > 0) {
          int w = ns + m - 1, q = m - 1;
          for (int b = ns; b >= 0; --b) {
            if (b < ns) fs[w--] = fs[b];
            const bool sp = q >= 0 && s_fixf[q] == b;
            if (sp) fs[w--] = s_fixv[q--];
            fL[b] = (q + 1) | (sp ? kSplitBit : 0);
          }
          s_ns = ns + m;
          atomicAdd(&P.ctl->refined, static_cast<unsigned>(m));
        }
        s_nfix = static_cast<unsigned>(m);
      }
      __syncthreads();
      if (s_nfix == 0) break;
      build_top_table(fs, s_ns, ftop);
      for (int f = threadIdx.x; f < slots; f += blockDim.x) cnt[f] = 0;
      __syncthreads();
      for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        if (t < n) {
          const int f = P.fid_tmp[base + t];
          const int sh = fL[f];
          int nf = f + (sh & ~kSplitBit);
          if (sh & kSplitBit) {
            uint64_t c[KW];
            src.ckey(P.idx_in[base + t], c);
            nf = upper_bound_top(fs, ftop, code_of<KW>(c, Lp, densep));
          }
          if (nf != f) P.fid_tmp[base + t] = static_cast<uint16_t>(nf);
          atomicAdd(&cnt[nf], 1u);
        }
      }
      __syncthreads();
      fine_prefixes(fs, s_ns, slots, Lp, densep, total, fL);
      __syncthreads();
    }
    if (P.trace && threadIdx.x == 0) s_tp[3] = clock64();
    if (placed) {
      // every record is in place: fine bucket f starts at its slot
      for (int f = threadIdx.x; f < slots; f += blockDim.x) {
        const bool exact = (fL[f] >> 16) & 1;
        const bool pure = exact && (fL[f] & 0xffff) == total;  // every key of the bucket is equal
        P.fine_start[g0 + f] = static_cast<uint32_t>(rbase + static_cast<size_t>(f) * kCap);
        P.fine_count[g0 + f] = cnt[f] | (exact ? kExactBit : 0u) | (pure ? kPureBit : 0u);
        P.fine_L[g0 + f] = static_cast<uint16_t>(fL[f] & 0xffff);
      }
      __syncthreads();
      if (P.trace && threadIdx.x == 0) s_tp[4] = clock64();
    } else {
      // fine bucket offsets, each bucket starting on a multiple of 32 records
      // (slots <= kFineSlots: a few rounds of the block scan)
      unsigned carry = 0;
      for (int f0 = 0; f0 < slots; f0 += blockDim.x) {
        const int f = f0 + threadIdx.x;
        const unsigned c = f < slots ? cnt[f] : 0u;
        unsigned tot;
        const unsigned ex = block_exclusive_scan((c + 31u) & ~31u, warp_tmp, &tot);
        if (f < slots) {
          const unsigned off = carry + ex;
          const bool exact = (fL[f] >> 16) & 1;
          const bool pure = exact && (fL[f] & 0xffff) == total;  // every key of the bucket is equal
          P.fine_start[g0 + f] = static_cast<uint32_t>(rbase + off);
          P.fine_count[g0 + f] = c | (exact ? kExactBit : 0u) | (pure ? kPureBit : 0u);
          P.fine_L[g0 + f] = static_cast<uint16_t>(fL[f] & 0xffff);
          cnt[f] = off;
        }
        carry += tot;
      }
      __syncthreads();
      if (P.trace && threadIdx.x == 0) s_tp[4] = clock64();
      // pass 2: (code relative to the fine prefix, index) into fine-bucket order
      for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        const bool valid = t < n;
        const int f = valid ? P.fid_tmp[base + t] : 0;
        const unsigned pos = valid ? atomicAdd(&cnt[f], 1u) : 0u;
        if (valid) {
          const uint32_t p = P.idx_in[base + t];
          uint64_t c[KW];
          src.ckey(p, c);
          const int Lf = fL[f];
          P.rec_code[rbase + pos] = code_of<KW>(c, Lf & 0xffff, (Lf >> 16) & 1);
          P.rec_idx[rbase + pos] = p;
        }
      }
      __syncthreads();
    }
    if (P.trace && threadIdx.x == 0) {
      s_tp[5] = clock64();
      for (int q = 0; q < 5; ++q) atomicAdd(&P.ctl->fphase[q], static_cast<unsigned long long>(s_tp[q + 1] - s_tp[q]));
    }
  }
}

// ------------------------------------------------------------------ final

struct FinalParams {
  const uint32_t* fine_start;
  const uint32_t* fine_count;
  const uint16_t* fine_L;
  uint64_t* rec_code;     // codes in; real parts of the survivors' sums out
  uint32_t* rec_idx;      // indices in; survivors' indices out (bucket start + rank)
  double* rec_im;         // imaginary parts of the survivors' sums
  uint32_t* counts;       // [G] survivors per fine bucket
  Control* ctl;
  int trace;              // record per-phase cycles
};

struct FinalSmem {
  uint64_t code[kPadded];   // codes; once sorted and tied, the real parts of coefficients and sums
  double im[kPadded];       // imaginary parts of coefficients and sums
  uint32_t idx[kPadded];
  uint32_t head[kWords];
  uint32_t keep[kWords];
  uint32_t wpre[kWords];    // survivors before each keep word
  uint32_t runs[kMaxRuns];  // start << 16 | end of tie runs
  unsigned n_runs;
  unsigned job;
  long long tp[5];          // phase clocks of traced runs
};

__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

__device__ __forceinline__ bool rec_less(uint64_t ca, uint32_t ia, uint64_t cb, uint32_t ib) {
  return ca < cb || (ca == cb && ia < ib);
}

__device__ __forceinline__ bool bit_at(const uint32_t* m, int i) { return (m[i >> 5] >> (i & 31)) & 1u; }

// First set bit after position i, or n.
__device__ __forceinline__ int next_set(const uint32_t* m, int i, int n) {
  const int p = i + 1;
  if (p >= n) return n;
  int w = p >> 5;
  uint32_t v = m[w] & (~0u << (p & 31));
  const int nw = (n + 31) >> 5;
  while (!v) {
    if (++w >= nw) return n;
    v = m[w];
  }
  return min(n, (w << 5) + __ffs(v) - 1);
}

// Insertion sort of sorted positions [i, e) by (code, idx); the run is short,
// or already ordered (then each insertion stops at once).
__device__ void insertion_sort(FinalSmem& S, int i, int e) {
  for (int q = i + 1; q < e; ++q) {
    const uint64_t cq = S.code[pidx(q)];
    const uint32_t xq = S.idx[pidx(q)];
    int r = q;
    while (r > i && rec_less(cq, xq, S.code[pidx(r - 1)], S.idx[pidx(r - 1)])) {
      S.code[pidx(r)] = S.code[pidx(r - 1)];
      S.idx[pidx(r)] = S.idx[pidx(r - 1)];
      --r;
    }
    S.code[pidx(r)] = cq;
    S.idx[pidx(r)] = xq;
  }
}

// Compare-exchange of two sort keys: k0 takes the smaller when up, the larger
// otherwise.
__device__ __forceinline__ void cas(uint64_t& k0, uint64_t& k1, bool up) {
  const bool sw = up == (k1 < k0);
  const uint64_t t = k0;
  k0 = sw ? k1 : k0;
  k1 = sw ? t : k1;
}

constexpr int kSlotBits = 12;  // slot field of a sort key: positions up to kCap - 1 < 2^12 - 1
constexpr uint64_t kSlotMask = (uint64_t{1} << kSlotBits) - 1;
static_assert(kCap < (1 << kSlotBits), "a real sort key must stay below the sentinel");

// Bitonic sort of the first n records by (code, idx).  The network orders one
// 64-bit key per record: the code with its low kSlotBits bits replaced by the
// record's position before the sort (keys are distinct, and below the ~0
// padding).  Records whose codes agree above those bits come out in position
// order; the caller puts them in (code, idx) order, run by run.  The network
// is padded to N = kK3Threads * IPT; thread t holds sorted positions t*IPT ..
// t*IPT+IPT-1 in registers.  A stage with partner distance j < IPT runs in
// registers, IPT <= j < 32*IPT by warp shuffles, and j >= 32*IPT through shared
// memory (the im area, unused until the sums) in a slot-major layout (item k of
// thread t at k*kK3Threads + t), free of bank conflicts.
template <int IPT>
__device__ void bitonic_block_sort(FinalSmem& S, int n) {
  constexpr int N = kK3Threads * IPT;
  const int t = threadIdx.x;
  uint64_t* ex = reinterpret_cast<uint64_t*>(S.im);
  uint64_t key[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = t * IPT + k;
    key[k] = i < n ? (S.code[pidx(i)] & ~kSlotMask) | static_cast<uint64_t>(i) : ~0ull;
  }
  for (int size = 2; size <= N; size <<= 1) {
    for (int j = size >> 1; j >= IPT; j >>= 1) {
      const int m = j / IPT;  // partner thread t ^ m
      const bool keep_min = ((t & m) == 0) == ((t * IPT & size) == 0);
      if (m < 32) {
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          const uint64_t o = __shfl_xor_sync(0xffffffffu, key[k], m);
          if ((o < key[k]) == keep_min) key[k] = o;
        }
      } else {
#pragma unroll
        for (int k = 0; k < IPT; ++k) ex[k * kK3Threads + t] = key[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          const uint64_t o = ex[k * kK3Threads + (t ^ m)];
          if ((o < key[k]) == keep_min) key[k] = o;
        }
        __syncthreads();
      }
    }
#pragma unroll
    for (int jj = IPT / 2; jj > 0; jj >>= 1) {
      if (jj < size) {
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          if ((k & jj) == 0) cas(key[k], key[k | jj], ((t * IPT + k) & size) == 0);
        }
      }
    }
  }
  // records to their sorted positions: the slots go through shared memory
  // (the exchange area) so that only one position's record is live at a time
  uint16_t* slot = reinterpret_cast<uint16_t*>(ex);
#pragma unroll
  for (int k = 0; k < IPT; ++k) slot[t * IPT + k] = static_cast<uint16_t>(key[k] & kSlotMask);
  __syncthreads();
  uint64_t c[IPT];
  uint32_t x[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int sl = min(static_cast<int>(slot[t * IPT + k]), n - 1);
    c[k] = S.code[pidx(sl)];
    x[k] = S.idx[pidx(sl)];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    if (t * IPT + k < n) {
      S.code[pidx(t * IPT + k)] = c[k];
      S.idx[pidx(t * IPT + k)] = x[k];
    }
  }
  __syncthreads();
}

// Sorts the first n (<= kCap) records by (code, idx) with the narrowest
// bitonic network that holds them.
__device__ __forceinline__ void block_sort(FinalSmem& S, int n) {
  if (n <= kK3Threads) bitonic_block_sort<1>(S, n);
  else if (n <= 2 * kK3Threads) bitonic_block_sort<2>(S, n);
  else if (n <= 4 * kK3Threads) bitonic_block_sort<4>(S, n);
  else bitonic_block_sort<8>(S, n);
}

// Positions [i, e) hold one tie of 16-digit codes: keys with more than 16 set
// bits after the prefix may still differ.  Reordered by (key, index) -- the
// distinct keys (at most kDistinct) are sorted, then each key's items are
// emitted in index order -- with a segment head where the key changes.  The
// code slots of the range are free by now and carry the indices on the way.
template <int KW, class Src>
__device__ void resolve_mixed(const Src& src, FinalSmem& S, int i, int e, unsigned* flags) {
  uint64_t D[kDistinct][KW];
  int nd = 0;
  for (int m = i; m < e; ++m) {
    uint64_t k[KW];
    src.key(S.idx[pidx(m)], k);
    bool seen = false;
    for (int d = 0; d < nd && !seen; ++d) {
      bool eq = true;
      for (int w = 0; w < KW; ++w) eq = eq && D[d][w] == k[w];
      seen = eq;
    }
    if (seen) continue;
    if (nd == kDistinct) {
      atomicOr(flags, kFlagDistinct);
      return;
    }
    for (int w = 0; w < KW; ++w) D[nd][w] = k[w];
    ++nd;
  }
  if (nd == 1) return;
  for (int q = 1; q < nd; ++q) {
    uint64_t kq[KW];
    for (int w = 0; w < KW; ++w) kq[w] = D[q][w];
    int r = q;
    while (r > 0) {
      uint64_t kp[KW];
      for (int w = 0; w < KW; ++w) kp[w] = D[r - 1][w];
      if (!kless<KW>(kq, kp)) break;
      for (int w = 0; w < KW; ++w) D[r][w] = kp[w];
      --r;
    }
    for (int w = 0; w < KW; ++w) D[r][w] = kq[w];
  }
  int o = i;
  for (int d = 0; d < nd; ++d) {
    if (d > 0) atomicOr(&S.head[o >> 5], 1u << (o & 31));
    uint64_t kd[KW];
    for (int w = 0; w < KW; ++w) kd[w] = D[d][w];
    for (int m = i; m < e; ++m) {
      const uint32_t id = S.idx[pidx(m)];
      uint64_t k[KW];
      src.key(id, k);
      if (keq<KW>(k, kd)) S.code[pidx(o++)] = id;
    }
  }
  for (int m = i; m < e; ++m) S.idx[pidx(m)] = static_cast<uint32_t>(S.code[pidx(m)]);
}

// A run [i, e) of equal 8-digit position codes: the items take their next
// eight digits as code and are reordered by (code, index); a head goes where
// that code changes, and ties of all 16 digits with a 16th digit (the key may
// have more set bits) are checked key by key.
template <int KW, class Src>
__device__ void resolve_tie(const Src& src, FinalSmem& S, int i, int e, int L, unsigned* flags) {
  for (int m = i; m < e; ++m) {
    uint64_t c[KW];
    src.ckey(S.idx[pidx(m)], c);
    S.code[pidx(m)] = position_code<KW>(c, L, 8);
  }
  insertion_sort(S, i, e);
  int s = i;
  while (s < e) {
    const uint64_t cs = S.code[pidx(s)];
    int t = s + 1;
    while (t < e && S.code[pidx(t)] == cs) ++t;
    if (s > i) atomicOr(&S.head[s >> 5], 1u << (s & 31));
    if (t - s > 1 && (cs & 0xffu) != 0) resolve_mixed<KW>(src, S, s, t, flags);
    s = t;
  }
}

static_assert(kK3Threads == 256, "radix_sort_u32 maps one thread per digit");
static_assert(sizeof(unsigned) * (256 + (kK3Threads / 32) * 256 + 2) <= sizeof(uint64_t) * kPadded,
              "radix_sort_u32 scratch must fit in the code area");

// Stable LSD radix sort (8-bit digits) of n indices in global memory by one
// block, ping-ponging between a and tmp; digits on which all indices agree are
// skipped.  Returns the array that holds the sorted indices.  Scratch lives in
// the (unused) code area of the shared-memory tile.
__device__ const uint32_t* radix_sort_u32(FinalSmem& S, uint32_t* a, uint32_t* tmp, int n) {
  unsigned* hist = reinterpret_cast<unsigned*>(S.code);           // [256]
  unsigned* wcnt = hist + 256;                                      // [8][256]
  unsigned* red = wcnt + (kK3Threads / 32) * 256;                   // [2]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 2) red[tid] = tid == 0 ? 0u : ~0u;
  __syncthreads();
  unsigned o = 0, d = ~0u;
  for (int i = tid; i < n; i += kK3Threads) {
    o |= a[i];
    d &= a[i];
  }
  atomicOr(&red[0], o);
  atomicAnd(&red[1], d);
  __syncthreads();
  const unsigned vary = red[0] ^ red[1];
  uint32_t* src = a;
  uint32_t* dst = tmp;
  const uint32_t lt = (1u << lane) - 1u;
  for (int sh = 0; sh < 32; sh += 8) {
    if (((vary >> sh) & 0xffu) == 0) continue;
    hist[tid] = 0;
    __syncthreads();
    for (int i = tid; i < n; i += kK3Threads) atomicAdd(&hist[(src[i] >> sh) & 0xffu], 1u);
    __syncthreads();
    if (warp == 0) {
      // exclusive scan of 256 counts, 8 per lane
      unsigned v[8], t = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        v[q] = hist[lane * 8 + q];
        t += v[q];
      }
      unsigned incl = t;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
      }
      unsigned run = incl - t;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        hist[lane * 8 + q] = run;
        run += v[q];
      }
    }
    __syncthreads();
    for (int i0 = 0; i0 < n; i0 += kK3Threads) {
      const int i = i0 + tid;
      const bool valid = i < n;
      const uint32_t val = valid ? src[i] : 0u;
      const unsigned dg = valid ? (val >> sh) & 0xffu : 0x100u;
      for (int e = tid; e < (kK3Threads / 32) * 256; e += kK3Threads) wcnt[e] = 0;
      __syncthreads();
      const unsigned peers = __match_any_sync(0xffffffffu, dg);
      const unsigned rank = __popc(peers & lt);
      if (valid && rank == 0) wcnt[warp * 256 + dg] = __popc(peers);
      __syncthreads();
      {
        unsigned run = hist[tid];
        for (int w = 0; w < kK3Threads / 32; ++w) {
          const unsigned c = wcnt[w * 256 + tid];
          wcnt[w * 256 + tid] = run;
          run += c;
        }
        hist[tid] = run;
      }
      __syncthreads();
      if (valid) dst[wcnt[warp * 256 + dg] + rank] = val;
      __syncthreads();
    }
    uint32_t* t2 = src;
    src = dst;
    dst = t2;
  }
  __threadfence_block();
  __syncthreads();
  return src;
}

template <int KW, class Src>
__global__ void __launch_bounds__(kK3Threads, kK3PerSM) bucket_final_kernel(Src src, FinalParams P) {
  extern __shared__ __align__(16) unsigned char k3raw[];
  FinalSmem& S = *reinterpret_cast<FinalSmem*>(k3raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned G = P.ctl->fine_total;
  const double thr = P.ctl->thr;
  bool inf = false;
  while (true) {
    if (P.trace && tid == 0) S.tp[0] = clock64();
    if (tid == 0) S.job = atomicAdd(&P.ctl->k3_ticket, 1u);
    __syncthreads();
    const unsigned g = S.job;
    __syncthreads();
    if (g >= G) break;
    const uint32_t start = P.fine_start[g];
    const uint32_t cw = P.fine_count[g];
    const int n = static_cast<int>(cw & kCountMask);
    const bool exact = (cw & kExactBit) != 0;
    bool pure = (cw & kPureBit) != 0;
    const bool fits = n <= kCap;
    if (!fits && !pure) {
      // an isolated code whose eight digits do not fix the key: one key if
      // every item's key equals the first
      uint64_t k0[KW], k[KW];
      src.key(P.rec_idx[start], k0);
      bool same = true;
      for (int i = tid; i < n && same; i += kK3Threads) {
        src.key(P.rec_idx[start + i], k);
        same = keq<KW>(k, k0);
      }
      pure = __syncthreads_and(same) != 0;
    }
    if (tid == 0 && n > 0) {
      if (!fits && !pure) atomicOr(&P.ctl->flags, kFlagFineFull);
      atomicMax(&P.ctl->max_fine, static_cast<unsigned>(n));
    }
    if (!fits && pure) {
      // one key, more items than shared memory holds: sort the indices in
      // global memory, then one thread sums them in index order
      uint32_t* a = P.rec_idx + start;
      uint32_t* tmp = reinterpret_cast<uint32_t*>(P.rec_code + start);
      const uint32_t* sorted = radix_sort_u32(S, a, tmp, n);
      if (tid == 0) {
        c128 acc{0.0, 0.0};
        for (int m = 0; m < n; ++m) {
          uint64_t k[KW];
          const c128 c = src.key_coeff(sorted[m], k);
          if (!(fabs(c.re) <= 0x1p1022 && fabs(c.im) <= 0x1p1022) && isinf(wgd::hypot_ref(c.re, c.im))) inf = true;
          acc = wgd::cadd(acc, c);
        }
        const bool kp = wgd::hypot_ref(acc.re, acc.im) > thr;
        const uint32_t first = sorted[0];
        P.rec_idx[start] = first;
        P.rec_code[start] = static_cast<uint64_t>(__double_as_longlong(acc.re));
        P.rec_im[start] = acc.im;
        P.counts[g] = kp ? 1u : 0u;
      }
      __syncthreads();
    }
    if (fits && n > 0) {
      for (int i = tid; i < n; i += kK3Threads) {
        S.code[pidx(i)] = P.rec_code[start + i];
        S.idx[pidx(i)] = P.rec_idx[start + i];
      }
      for (int w = tid; w < kWords; w += kK3Threads) {
        S.head[w] = 0;
        S.keep[w] = 0;
      }
      if (tid == 0) S.n_runs = 0;
      __syncthreads();
      if (P.trace) {
        // how many 8-bit digits of the bucket's codes vary (an LSD pass would sort one each)
        const uint64_t c0 = S.code[pidx(0)];
        uint64_t v = 0;
        for (int i = tid; i < n; i += kK3Threads) v |= S.code[pidx(i)] ^ c0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
        uint64_t* red = reinterpret_cast<uint64_t*>(S.im);
        if (lane == 0) red[warp] = v;
        __syncthreads();
        if (tid == 0) {
          uint64_t all = 0;
          for (int w = 0; w < kK3Threads / 32; ++w) all |= red[w];
          int d = 0;
          for (int b = 0; b < 64; b += 8) d += ((all >> b) & 0xffu) != 0;
          atomicAdd(&P.ctl->digits[d], 1ull);
          S.tp[1] = clock64();
        }
        __syncthreads();
      }
      block_sort(S, n);
      // runs of codes equal above the slot bits, each put in (code, idx) order
      // by the thread at its first position
      for (int i = tid; i + 1 < n; i += kK3Threads) {
        const uint64_t hi = S.code[pidx(i)] >> kSlotBits;
        if ((S.code[pidx(i + 1)] >> kSlotBits) != hi || (i > 0 && (S.code[pidx(i - 1)] >> kSlotBits) == hi)) continue;
        int e = i + 2;
        while (e < n && (S.code[pidx(e)] >> kSlotBits) == hi) ++e;
        insertion_sort(S, i, e);
      }
      __syncthreads();
      if (P.trace && tid == 0) S.tp[2] = clock64();
      // segment heads where the code changes, and (inexact codes) runs of
      // equal position code, listed by the thread at the run's first position
      // and resolved once every thread is done reading codes
      for (int i0 = warp * 32; i0 < n; i0 += kK3Threads) {
        const int i = i0 + lane;
        const uint64_t ci = i < n ? S.code[pidx(i)] : 0;
        const bool h = i < n && (i == 0 || S.code[pidx(i - 1)] != ci);
        const uint32_t b = __ballot_sync(0xffffffffu, h);
        if (lane == 0) S.head[i0 >> 5] = b;
        // a code with an empty eighth digit holds every set bit: one key
        if (!exact && h && i + 1 < n && (ci & 0xffu) != 0 && S.code[pidx(i + 1)] == ci) {
          int e = i + 2;
          while (e < n && S.code[pidx(e)] == ci) ++e;
          const unsigned q = atomicAdd(&S.n_runs, 1u);
          S.runs[q] = (static_cast<uint32_t>(i) << 16) | static_cast<uint32_t>(e);
          if (P.trace) atomicAdd(&P.ctl->tie_items, static_cast<unsigned long long>(e - i));
        }
      }
      if (!exact) {
        __syncthreads();
        const int L = P.fine_L[g];
        const int nr = static_cast<int>(S.n_runs);
        for (int q = tid; q < nr; q += kK3Threads)
          resolve_tie<KW>(src, S, static_cast<int>(S.runs[q] >> 16), static_cast<int>(S.runs[q] & 0xffffu), L,
                          &P.ctl->flags);
      }
      __syncthreads();
      if (P.trace && tid == 0) S.tp[3] = clock64();
      // every item's coefficient, two items per thread in flight; the code
      // slots take the real parts
      for (int i0 = tid; i0 < n; i0 += 2 * kK3Threads) {
        c128 cv[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int i = i0 + u * kK3Threads;
          if (i < n) {
            uint64_t k[KW];
            cv[u] = src.key_coeff(S.idx[pidx(i)], k);
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int i = i0 + u * kK3Threads;
          if (i < n) {
            const c128 c = cv[u];
            if (!(fabs(c.re) <= 0x1p1022 && fabs(c.im) <= 0x1p1022) && isinf(wgd::hypot_ref(c.re, c.im))) inf = true;
            S.code[pidx(i)] = static_cast<uint64_t>(__double_as_longlong(c.re));
            S.im[pidx(i)] = c.im;
          }
        }
      }
      __syncthreads();
      // segment sums, left to right from zero, and the cull; a head's slot
      // takes its segment's sum
      for (int i0 = warp * 32; i0 < n; i0 += kK3Threads) {
        const int i = i0 + lane;
        bool kp = false;
        if (i < n && bit_at(S.head, i)) {
          const int e = next_set(S.head, i, n);
          c128 acc{0.0, 0.0};
          for (int m = i; m < e; ++m)
            acc = wgd::cadd(acc, c128{__longlong_as_double(static_cast<long long>(S.code[pidx(m)])), S.im[pidx(m)]});
          // without NaNs the rounded |s| is never below max(|re|, |im|), which
          // decides most sums without the full hypot
          const bool plain = !isnan(acc.re) && !isnan(acc.im);
          kp = (plain && (fabs(acc.re) > thr || fabs(acc.im) > thr)) || wgd::hypot_ref(acc.re, acc.im) > thr;
          S.code[pidx(i)] = static_cast<uint64_t>(__double_as_longlong(acc.re));
          S.im[pidx(i)] = acc.im;
        }
        const uint32_t b = __ballot_sync(0xffffffffu, kp);
        if (lane == 0) S.keep[i0 >> 5] = b;
      }
      __syncthreads();
      // survivors before each keep word (at most kWords = 64: two per lane)
      const int nw = (n + 31) >> 5;
      if (warp == 0) {
        const int w0 = 2 * lane;
        const unsigned v0 = w0 < nw ? __popc(S.keep[w0]) : 0u, v1 = w0 + 1 < nw ? __popc(S.keep[w0 + 1]) : 0u;
        unsigned incl = v0 + v1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        const unsigned ex = incl - v0 - v1;
        if (w0 < nw) S.wpre[w0] = ex;
        if (w0 + 1 < nw) S.wpre[w0 + 1] = ex + v0;
        if (lane == 31) P.counts[g] = incl;
      }
      __syncthreads();
      // survivors compacted at the start of the bucket's records: index, sum
      for (int i = tid; i < n; i += kK3Threads) {
        const uint32_t kw = S.keep[i >> 5];
        if (!((kw >> (i & 31)) & 1u)) continue;
        const uint32_t r = start + S.wpre[i >> 5] + __popc(kw & ((1u << (i & 31)) - 1u));
        P.rec_idx[r] = S.idx[pidx(i)];
        P.rec_code[r] = S.code[pidx(i)];
        P.rec_im[r] = S.im[pidx(i)];
      }
      if (P.trace && tid == 0) {
        S.tp[4] = clock64();
        for (int q = 0; q < 4; ++q) atomicAdd(&P.ctl->phase[q], static_cast<unsigned long long>(S.tp[q + 1] - S.tp[q]));
      }
    }
    __syncthreads();
  }
  if (inf) atomicOr(&P.ctl->inf_seen, 1u);
}

// ------------------------------------------------------------------ output

struct OutputParams {
  const uint32_t* fine_start;
  const uint32_t* rec_idx;     // survivors' indices at the start of each bucket
  const uint64_t* rec_re;      // their sums
  const double* rec_im;
  const uint32_t* offsets;     // [G] exclusive prefix of the survivor counts
  const uint32_t* counts;
  const Control* ctl;
  uint64_t* out_x;
  uint64_t* out_z;
  double* out_c;
  size_t out_cap;
  unsigned* flags;
};

// One warp per fine bucket: its survivors go to consecutive ranks from the
// bucket's offset, each key rebuilt from its operands.  A lane moves kU
// survivors at a time, their loads issued before any store.
template <int KW, class Src>
__global__ void __launch_bounds__(256) bucket_output_kernel(Src src, OutputParams P) {
  constexpr int kU = 6;  // survivors per lane in flight (config 2: 4: 7.95 ms, 5: 7.19, 6: 7.03, 7: 7.14, 8: 8.44)
  const int lane = threadIdx.x & 31;
  const unsigned G = P.ctl->fine_total;
  const unsigned warps = gridDim.x * (blockDim.x >> 5);
  for (unsigned g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < G; g += warps) {
    const uint32_t cnt = P.counts[g];
    if (cnt == 0) continue;
    const uint32_t start = P.fine_start[g];
    const size_t base = P.offsets[g];
    if (base + cnt > P.out_cap) {
      if (lane == 0) atomicOr(P.flags, kFlagOverrun);
      continue;
    }
    for (uint32_t i0 = lane; i0 < cnt; i0 += 32 * kU) {
      uint32_t id[kU];
      uint64_t re[kU];
      double im[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const uint32_t i = i0 + 32 * u;
        if (i < cnt) {
          id[u] = P.rec_idx[start + i];
          re[u] = P.rec_re[start + i];
          im[u] = P.rec_im[start + i];
        }
      }
      uint64_t k[kU][KW];
#pragma unroll
      for (int u = 0; u < kU; ++u)
        if (i0 + 32 * u < cnt) src.key(id[u], k[u]);
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const uint32_t i = i0 + 32 * u;
        if (i < cnt) {
          const size_t o = base + i;
          if (KW == 4) {
            reinterpret_cast<ulonglong2*>(P.out_x)[o] = make_ulonglong2(k[u][0], k[u][2]);
            reinterpret_cast<ulonglong2*>(P.out_z)[o] = make_ulonglong2(k[u][1], k[u][3]);
          } else {
#pragma unroll
            for (int w = 0; w < KW / 2; ++w) {
              P.out_x[o * (KW / 2) + w] = k[u][2 * w];
              P.out_z[o * (KW / 2) + w] = k[u][2 * w + 1];
            }
          }
          reinterpret_cast<double2*>(P.out_c)[o] =
              make_double2(__longlong_as_double(static_cast<long long>(re[u])), im[u]);
        }
      }
    }
  }
}

// ------------------------------------------------------------------ host side

std::atomic<int> g_sort_algorithm{WG_SORT_AUTO};
std::atomic<unsigned> g_fine_target{0};  // target items per fine bucket; 0: kFineAvg
std::atomic<bool> g_one_pass_fine{true};  // fine pass in one-pass layout where it fits (see run_bucket)
thread_local unsigned t_fine_choice = 0;   // the autotuner's target for the running call; 0: none

// Fine-bucket targets the autotuner chooses among (kFineAvg is candidate 2).
constexpr unsigned kFineCandidates[] = {640, 768, 896, 1024, 1280};
static_assert(kFineCandidates[2] == kFineAvg, "the default target is the fallback candidate");

struct FineChoice {
  explicit FineChoice(unsigned t) { t_fine_choice = t; }
  ~FineChoice() { t_fine_choice = 0; }
};

// A bucketed call with the fine-bucket target chosen by the autotuner when
// no process-wide target is set (wg_set_bucket_fine_target).  call(ox, oz,
// oc, U) runs the whole sort-reduce and returns false when the bucketed path
// cannot serve the inputs.  During a search every candidate's run allocates
// its own outputs; the latest successful run's are kept, the others freed.
template <class Call>
bool bucket_tuned(int W, size_t items, uint64_t** ox, uint64_t** oz, double** oc, size_t* U, cudaStream_t s,
                  Call&& call) {
  if (g_fine_target.load(std::memory_order_relaxed) != 0) return call(ox, oz, oc, U);
  uint64_t *kx = nullptr, *kz = nullptr;
  double* kc = nullptr;
  size_t ku = 0;
  bool have = false;
  auto run = [&](int c) -> bool {
    FineChoice fc(kFineCandidates[c]);
    uint64_t *x = nullptr, *z = nullptr;
    double* cc = nullptr;
    size_t u = 0;
    if (!call(&x, &z, &cc, &u)) return false;
    if (have) {
      wg::pool_free(kx, s);
      wg::pool_free(kz, s);
      wg::pool_free(kc, s);
    }
    kx = x;
    kz = z;
    kc = cc;
    ku = u;
    have = true;
    return true;
  };
  bool done = false;
  int choice;
  try {
    choice = wg::tune_choose(wg::kTuneBucket, W, wg::ceil_log2(items), 0, 2, true, s, run, &done);
  } catch (...) {
    if (have) {
      wg::pool_free(kx, s);
      wg::pool_free(kz, s);
      wg::pool_free(kc, s);
    }
    throw;
  }
  if (done) {
    *ox = kx;
    *oz = kz;
    *oc = kc;
    *U = ku;
    return true;
  }
  if (have) {  // a search whose candidates all failed but one earlier run
    wg::pool_free(kx, s);
    wg::pool_free(kz, s);
    wg::pool_free(kc, s);
  }
  FineChoice fc(kFineCandidates[choice >= 0 && choice < 5 ? choice : 2]);
  return call(ox, oz, oc, U);
}
thread_local int t_last_sort = 0;

struct ThrSpec {
  int mode;  // 0 fixed, 1 atol + rtol * max|c|, 2 atol (an infinite |c| empties the result)
  double atol, rtol, fixed;
};

struct Outs {
  uint64_t** x;
  uint64_t** z;
  double** c;
  size_t* n;
};

// Host-side stage times of one traced call (WG_BUCKET_TRACE set).
struct Stamps {
  bool on = std::getenv("WG_BUCKET_TRACE") != nullptr;
  int k = 0;
  const char* name[16];
  std::chrono::steady_clock::time_point t[16];
  void operator()(const char* what) {
    if (on && k < 16) {
      name[k] = what;
      t[k++] = std::chrono::steady_clock::now();
    }
  }
  ~Stamps() {
    if (!on || k < 2) return;
    std::fprintf(stderr, "bucket host stages (ms):");
    for (int i = 1; i < k; ++i)
      std::fprintf(stderr, " %s %.2f", name[i], std::chrono::duration<double, std::milli>(t[i] - t[i - 1]).count());
    std::fprintf(stderr, "\n");
  }
};

template <class K>
void set_smem(K kernel, size_t bytes) {
  wg::check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
                 "set bucket kernel shared memory");
  // the occupancy the grids are sized for assumes the largest shared-memory
  // configuration: ask for it, whatever ran before on the SM
  wg::check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      static_cast<int>(cudaSharedmemCarveoutMaxShared)),
                 "set bucket kernel shared-memory carveout");
}

template <int KW, class Src>
bool run_bucket(int device, const Src& src, uint32_t n, int total, const ThrSpec& thr, const Outs& out,
                cudaStream_t s) {
  Stamps stamp;
  stamp("start");
  const int W = KW / 2;
  const bool dense0 = total <= 64;
  int B1 = 2;
  while (B1 < kCoarseMax && (static_cast<uint64_t>(B1) << kCoarseLog) < n) B1 <<= 1;
  const uint64_t avg = (static_cast<uint64_t>(n) + B1 - 1) / B1;
  const uint64_t capc64 = 2 * avg + 8192;
  const unsigned set_avg = g_fine_target.load(std::memory_order_relaxed);
  const unsigned favg = t_fine_choice ? t_fine_choice : set_avg ? set_avg : static_cast<unsigned>(kFineAvg);
  if (capc64 > static_cast<uint64_t>(kFineMax) * favg) return false;  // fine buckets would overflow
  const uint32_t capc = static_cast<uint32_t>(capc64);
  const size_t region = static_cast<size_t>(B1) * capc;
  // fine slots: sum over coarse buckets of t + t/4 + 8 with t <= n_j/favg + 1
  const size_t Gmax = (static_cast<size_t>(n) / favg + B1) * 5 / 4 + static_cast<size_t>(B1) * 9 + 1;
  // records of the fine partition: rstride slots per coarse bucket, every fine
  // bucket starting on a multiple of 32
  const uint64_t rstride64 = ((static_cast<uint64_t>(capc) + 31) & ~uint64_t{31}) + 32ull * kFineSlots;
  if (static_cast<uint64_t>(B1) * rstride64 >= 0xffffffffull) return false;
  const auto& props = wg::device_props(device);
  // One-pass layout (kCap records per fine slot, the fine pass writes each
  // item as it counts it) where its 20 bytes per record fit in a quarter of
  // the device's memory and record indices stay 32-bit; else rstride records
  // per coarse bucket and two passes.
  const uint64_t one_records = static_cast<uint64_t>(Gmax) * kCap;
  const bool one_pass = g_one_pass_fine.load(std::memory_order_relaxed) && one_records < 0xffffffffull &&
                        one_records * 20 <= props.total_mem / 4;
  const uint32_t rstride = one_pass ? 0u : static_cast<uint32_t>(rstride64);
  const size_t records = one_pass ? static_cast<size_t>(one_records) : static_cast<size_t>(B1) * rstride64;
  const bool trace = stamp.on;

  // every intermediate lives in the device workspace
  using WS = wg::Workspace;
  const size_t ws_bytes = WS::rounded(sizeof(Control)) + WS::rounded(8 * B1) + WS::rounded(4 * B1) +
                          WS::rounded(4 * region) + WS::rounded(4 * (B1 + 1)) + 2 * WS::rounded(4 * B1) +
                          WS::rounded(8 * records) + WS::rounded(4 * records) + 2 * WS::rounded(4 * Gmax) +
                          WS::rounded(2 * Gmax) + WS::rounded(2 * region) + WS::rounded(8 * records) +
                          2 * WS::rounded(4 * Gmax) + WS::rounded(4);
  WS ws(device, ws_bytes, s);
  Control* dctl = ws.take_as<Control>(1);
  wg::check_cuda(cudaMemsetAsync(dctl, 0, sizeof(Control), s), "clear bucket control");

  // coarse splitters from a sorted sample of codes
  const uint32_t S1 = static_cast<uint32_t>(std::min<uint64_t>(n, static_cast<uint64_t>(kCoarseSample) * B1));
  uint64_t* split = ws.take_as<uint64_t>(B1);
  {
    wg::Scratch skeys(sizeof(uint64_t) * S1, s), sidx(sizeof(uint32_t) * S1, s);
    WG_TIMED("bucket_sample_kernel", s,
      bucket_sample_kernel<KW><<<wg::grid_for(S1, 256, device, 4), 256, 0, s>>>(src, n, S1, dense0,
                                                                                 skeys.as<uint64_t>(),
                                                                                 sidx.as<uint32_t>()));
    wg::check_launch("launch bucket sample");
    wg::radix_sort_keys(device, S1, 1, skeys, sidx, s);
    WG_TIMED("bucket_pick_kernel", s,
      bucket_pick_kernel<<<(B1 + 255) / 256, 256, 0, s>>>(skeys.as<uint64_t>(), S1, B1, split));
    wg::check_launch("launch bucket splitters");
  }
  stamp("sample");

  // coarse scatter
  unsigned* fill = ws.take_as<unsigned>(B1);
  uint32_t* idx1 = ws.take_as<uint32_t>(region);
  wg::check_cuda(cudaMemsetAsync(fill, 0, sizeof(unsigned) * B1, s), "clear coarse fill");
  {
    const CoarseParams cp{split, B1, capc, fill, idx1, dense0, thr.mode == 1, &dctl->max_bits};
    const unsigned grid = wg::grid_for(n, kK1Threads * kK1Items, device, 2);
    WG_TIMED("bucket_coarse_kernel", s, bucket_coarse_kernel<KW><<<grid, kK1Threads, 0, s>>>(src, n, cp));
    wg::check_launch("launch coarse scatter");
  }
  uint32_t* fine_base = ws.take_as<uint32_t>(B1 + 1);
  int* Lj = ws.take_as<int>(B1);
  uint32_t* order = ws.take_as<uint32_t>(B1);
  WG_TIMED("bucket_plan_kernel", s,
    bucket_plan_kernel<<<1, 1024, 0, s>>>(fill, B1, capc, split, total, dense0, thr.mode, thr.atol, thr.rtol,
                                          thr.fixed, favg, dctl, fine_base, Lj, order));
  wg::check_launch("launch bucket plan");
  stamp("coarse");

  // fine partition
  uint64_t* rec_code = ws.take_as<uint64_t>(records);
  uint32_t* rec_idx = ws.take_as<uint32_t>(records);
  uint32_t* fine_start = ws.take_as<uint32_t>(Gmax);
  uint32_t* fine_count = ws.take_as<uint32_t>(Gmax);
  uint16_t* fine_L = ws.take_as<uint16_t>(Gmax);
  {
    uint16_t* fid_tmp = ws.take_as<uint16_t>(region);
    const FineParams fp{fill, capc, B1, total, fine_base, Lj, idx1, fid_tmp, rstride, rec_code, rec_idx,
                        fine_start, fine_count, fine_L, dctl, favg, trace ? 1 : 0, order};
    auto* k2 = bucket_fine_kernel<KW, Src>;
    set_smem(k2, kK2Smem);
    int per_sm = 0;
    wg::check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2, kK2Threads, kK2Smem),
                   "query fine occupancy");
    const unsigned grid = static_cast<unsigned>(std::min<int>(B1, props.sm_count * std::max(1, per_sm)));
    WG_TIMED("bucket_fine_kernel", s, k2<<<grid, kK2Threads, kK2Smem, s>>>(src, fp));
    wg::check_launch("launch fine partition");
  }
  stamp("fine");

  // final: sort, reduce and cull each fine bucket; survivors per bucket
  double* rec_im = ws.take_as<double>(records);
  uint32_t* counts = ws.take_as<uint32_t>(Gmax);
  uint32_t* offsets = ws.take_as<uint32_t>(Gmax);
  uint32_t* survivors = ws.take_as<uint32_t>(1);
  wg::check_cuda(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * Gmax, s), "clear survivor counts");
  {
    const FinalParams fp{fine_start, fine_count, fine_L, rec_code, rec_idx, rec_im, counts, dctl, trace ? 1 : 0};
    auto* k3 = bucket_final_kernel<KW, Src>;
    set_smem(k3, sizeof(FinalSmem));
    int per_sm = 0;
    wg::check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k3, kK3Threads, sizeof(FinalSmem)),
                   "query final occupancy");
    const unsigned grid = static_cast<unsigned>(props.sm_count * std::max(1, per_sm));
    if (trace) std::fprintf(stderr, "bucket final: %d CTAs per SM, %zu bytes of shared memory each\n", per_sm, sizeof(FinalSmem));
    WG_TIMED("bucket_final_kernel", s, k3<<<grid, kK3Threads, sizeof(FinalSmem), s>>>(src, fp));
    wg::check_launch("launch bucket final");
  }
  wgs::exclusive_scan<uint32_t>(counts, offsets, Gmax, survivors, s);
  stamp("final");
  Control h{};
  uint32_t U32 = 0;
  wg::check_cuda(cudaMemcpyAsync(&h, dctl, sizeof(Control), cudaMemcpyDeviceToHost, s), "read bucket control");
  wg::check_cuda(cudaMemcpyAsync(&U32, survivors, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                 "read survivor count");
  wg::check_cuda(cudaStreamSynchronize(s), "synchronize bucket sort");
  stamp("sync");
  if (trace) {
    std::fprintf(stderr,
                 "bucket: n=%u coarse=%d fine=%u max_fine=%u refined=%u flags=0x%x survivors=%u tie_items=%llu\n", n,
                 B1, h.fine_total, h.max_fine, h.refined, h.flags, U32, h.tie_items);
    std::fprintf(stderr, "bucket final phases (Gcycles, all CTAs): load %.2f sort %.2f ties %.2f sums %.2f\n",
                 h.phase[0] * 1e-9, h.phase[1] * 1e-9, h.phase[2] * 1e-9, h.phase[3] * 1e-9);
    std::fprintf(stderr, "bucket final: fine buckets by varying code digits:");
    for (int d = 0; d <= 8; ++d) std::fprintf(stderr, " %d:%llu", d, h.digits[d]);
    std::fprintf(stderr, "\n");
    std::fprintf(stderr,
                 "bucket fine phases (Gcycles, all CTAs): sample %.2f splitters %.2f count %.2f scan %.2f place %.2f\n",
                 h.fphase[0] * 1e-9, h.fphase[1] * 1e-9, h.fphase[2] * 1e-9, h.fphase[3] * 1e-9, h.fphase[4] * 1e-9);
  }
  if (h.flags & kFallbackMask) return false;
  size_t U = U32;
  if (thr.mode == 2 && h.inf_seen) U = 0;  // atol + 0 * inf is NaN: nothing survives
  *out.n = U;
  *out.x = *out.z = nullptr;
  *out.c = nullptr;
  if (U == 0) return true;
  // output: each survivor at its rank
  wg::Scratch ox(sizeof(uint64_t) * W * U, s), oz(sizeof(uint64_t) * W * U, s), oc(sizeof(double) * 2 * U, s);
  stamp("alloc");
  {
    const OutputParams op{fine_start, rec_idx, rec_code, rec_im, offsets, counts, dctl,
                          ox.as<uint64_t>(), oz.as<uint64_t>(), oc.as<double>(), U, &dctl->flags};
    const unsigned grid = static_cast<unsigned>(props.sm_count * 8);
    WG_TIMED("bucket_output_kernel", s, bucket_output_kernel<KW><<<grid, 256, 0, s>>>(src, op));
    wg::check_launch("launch bucket output");
  }
  unsigned flags = 0;
  wg::check_cuda(cudaMemcpyAsync(&flags, &dctl->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "read flags");
  wg::check_cuda(cudaStreamSynchronize(s), "synchronize bucket outputs");
  stamp("output");
  if (flags & kFlagOverrun) throw wg::Error(WG_ERR_CUDA, "bucketed simplify: output rank beyond the survivor count");
  *out.x = static_cast<uint64_t*>(ox.detach());
  *out.z = static_cast<uint64_t*>(oz.detach());
  *out.c = static_cast<double*>(oc.detach());
  return true;
}

// Packs terms to operand records and ORs their key words into sig (device).
void pack(const uint64_t* x, const uint64_t* z, const double* c, size_t T, int W, wg::Scratch& rec,
          unsigned long long* sig, int device, cudaStream_t s) {
  rec.reset(sizeof(uint64_t) * (2 * W + 2) * std::max<size_t>(T, 1), s);
  WG_TIMED("bucket_pack_kernel", s,
    bucket_pack_kernel<<<wg::grid_for(T, 256, device, 4), 256, 0, s>>>(x, z, c, T, W, rec.as<uint64_t>(), sig));
  wg::check_launch("launch bucket pack");
}

void compress(const wg::Scratch& rec, size_t T, int KW, const SigWords& sig, wg::Scratch& out, int device,
              cudaStream_t s) {
  out.reset(sizeof(uint64_t) * KW * std::max<size_t>(T, 1), s);
  WG_TIMED("bucket_compress_kernel", s,
    bucket_compress_kernel<<<wg::grid_for(T, 256, device, 4), 256, 0, s>>>(rec.as<uint64_t>(), T, KW, sig,
                                                                            out.as<uint64_t>()));
  wg::check_launch("launch bucket compress");
}

// Significant bits of the packed keys (host copy) and their count.
// Under WG_SORT_AUTO, keys that vary in few 8-bit digits go to the LSD
// pipeline, which streams the items once per varying digit: measured on the
// B200, the bucketed path's time per item is that of about 5.5 LSD passes at
// two mask words (config 2: 73 ms bucketed, 329 ms for its 25 LSD passes)
// and it does not shrink with the key width, while narrow keys need few
// passes (a 20-qubit operator: 6).  kLsdDigits is the largest varying-digit
// count that the LSD pipeline takes, by mask words.
constexpr int kLsdDigits[3] = {0, 8, 5};

int varying_digits(const SigWords& sw, int KW) {
  int d = 0;
  for (int w = 0; w < KW; ++w)
    for (int b = 0; b < 64; b += 8) d += ((sw.w[w] >> b) & 0xffu) != 0;
  return d;
}

bool lsd_for_narrow_keys(const SigWords& sw, int KW) {
  return wg::sort_algorithm() == WG_SORT_AUTO && varying_digits(sw, KW) <= kLsdDigits[KW / 2];
}

int read_sig(const wg::Scratch& sig, int KW, SigWords& out, cudaStream_t s) {
  unsigned long long h[4] = {0, 0, 0, 0};
  wg::check_cuda(cudaMemcpyAsync(h, sig.get(), sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, s),
                 "read significant bits");
  wg::check_cuda(cudaStreamSynchronize(s), "read significant bits");
  int total = 0;
  for (int w = 0; w < 4; ++w) {
    out.w[w] = w < KW ? h[w] : 0ull;
    total += __builtin_popcountll(out.w[w]);
  }
  return total;
}

}  // namespace

namespace wg {

// One bucketed sort-reduce with the fine-bucket target of the calling
// thread's current choice (see bucket_tuned).
bool bucket_products_once(int device, int W, const uint64_t* lx, const uint64_t* lz, const double* lc, size_t n_l,
                          const uint64_t* rx, const uint64_t* rz, const double* rc, size_t n_r, int thr_mode,
                          double atol, double rtol, double thr_fixed, uint64_t** ox, uint64_t** oz, double** oc,
                          size_t* U, cudaStream_t s);
bool bucket_simplify_once(int device, int W, const uint64_t* x, const uint64_t* z, const double* c, size_t n,
                          int thr_mode, double atol, double rtol, uint64_t** ox, uint64_t** oz, double** oc,
                          size_t* U, cudaStream_t s);

int sort_algorithm() { return g_sort_algorithm.load(std::memory_order_relaxed); }
void note_sort(int algo) { t_last_sort = algo; }

bool bucket_products(int device, int W, const uint64_t* lx, const uint64_t* lz, const double* lc, size_t n_l,
                     const uint64_t* rx, const uint64_t* rz, const double* rc, size_t n_r, int thr_mode, double atol,
                     double rtol, double thr_fixed, uint64_t** ox, uint64_t** oz, double** oc, size_t* U,
                     cudaStream_t s) {
  if (W < 1 || W > 2 || n_l == 0 || n_r == 0 || n_l > 0xffffffffull || n_r > 0xffffffffull) return false;
  const size_t P = n_l * n_r;
  if (P > 0xffffffffull) return false;
  return bucket_tuned(W, P, ox, oz, oc, U, s, [&](uint64_t** x, uint64_t** z, double** c, size_t* u) {
    return bucket_products_once(device, W, lx, lz, lc, n_l, rx, rz, rc, n_r, thr_mode, atol, rtol, thr_fixed, x, z,
                                c, u, s);
  });
}

bool bucket_simplify(int device, int W, const uint64_t* x, const uint64_t* z, const double* c, size_t n,
                     int thr_mode, double atol, double rtol, uint64_t** ox, uint64_t** oz, double** oc, size_t* U,
                     cudaStream_t s) {
  if (W < 1 || W > 2 || n == 0 || n > 0xffffffffull) return false;
  return bucket_tuned(W, n, ox, oz, oc, U, s, [&](uint64_t** px, uint64_t** pz, double** pc, size_t* u) {
    return bucket_simplify_once(device, W, x, z, c, n, thr_mode, atol, rtol, px, pz, pc, u, s);
  });
}

bool bucket_products_once(int device, int W, const uint64_t* lx, const uint64_t* lz, const double* lc, size_t n_l,
                          const uint64_t* rx, const uint64_t* rz, const double* rc, size_t n_r, int thr_mode,
                          double atol, double rtol, double thr_fixed, uint64_t** ox, uint64_t** oz, double** oc,
                          size_t* U, cudaStream_t s) {
  const size_t P = n_l * n_r;
  const int KW = 2 * W;
  Scratch sig(sizeof(unsigned long long) * 4, s);
  check_cuda(cudaMemsetAsync(sig.get(), 0, sizeof(unsigned long long) * 4, s), "clear significant bits");
  Scratch ak, bk, ac2, bc2;
  pack(lx, lz, lc, n_l, W, ak, sig.as<unsigned long long>(), device, s);
  pack(rx, rz, rc, n_r, W, bk, sig.as<unsigned long long>(), device, s);
  SigWords sw{};
  const int total = read_sig(sig, KW, sw, s);
  if (total < 1 || total > 255 || lsd_for_narrow_keys(sw, KW)) return false;
  compress(ak, n_l, KW, sw, ac2, device, s);
  compress(bk, n_r, KW, sw, bc2, device, s);
  const ThrSpec thr{thr_mode, atol, rtol, thr_fixed};
  const Outs out{ox, oz, oc, U};
  const FastDiv fd{static_cast<uint32_t>(n_r), n_r > 1 ? ~0ull / n_r + 1 : 0ull};
  if (W == 1) {
    const ProdSrc<2> src{ak.as<uint64_t>(), bk.as<uint64_t>(), ac2.as<uint64_t>(), bc2.as<uint64_t>(), fd};
    return run_bucket<2>(device, src, static_cast<uint32_t>(P), total, thr, out, s);
  }
  const ProdSrc<4> src{ak.as<uint64_t>(), bk.as<uint64_t>(), ac2.as<uint64_t>(), bc2.as<uint64_t>(), fd};
  return run_bucket<4>(device, src, static_cast<uint32_t>(P), total, thr, out, s);
}

bool bucket_simplify_once(int device, int W, const uint64_t* x, const uint64_t* z, const double* c, size_t n,
                          int thr_mode, double atol, double rtol, uint64_t** ox, uint64_t** oz, double** oc,
                          size_t* U, cudaStream_t s) {
  const int KW = 2 * W;
  Scratch sig(sizeof(unsigned long long) * 4, s);
  check_cuda(cudaMemsetAsync(sig.get(), 0, sizeof(unsigned long long) * 4, s), "clear significant bits");
  Scratch tk, tc2;
  pack(x, z, c, n, W, tk, sig.as<unsigned long long>(), device, s);
  SigWords sw{};
  const int total = read_sig(sig, KW, sw, s);
  if (total < 1 || total > 255 || lsd_for_narrow_keys(sw, KW)) return false;
  compress(tk, n, KW, sw, tc2, device, s);
  const ThrSpec thr{thr_mode, atol, rtol, 0.0};
  const Outs out{ox, oz, oc, U};
  if (W == 1) {
    const TermSrc<2> src{tk.as<uint64_t>(), tc2.as<uint64_t>()};
    return run_bucket<2>(device, src, static_cast<uint32_t>(n), total, thr, out, s);
  }
  const TermSrc<4> src{tk.as<uint64_t>(), tc2.as<uint64_t>()};
  return run_bucket<4>(device, src, static_cast<uint32_t>(n), total, thr, out, s);
}

}  // namespace wg

extern "C" {

int wg_set_sort_algorithm(int algo) {
  return wg::guarded([&] {
    if (algo != WG_SORT_AUTO && algo != WG_SORT_LSD && algo != WG_SORT_BUCKET)
      wg::throw_invalid("sort algorithm must be WG_SORT_AUTO, WG_SORT_LSD or WG_SORT_BUCKET");
    g_sort_algorithm.store(algo, std::memory_order_relaxed);
  });
}

int wg_last_sort_algorithm(void) { return t_last_sort; }

int wg_set_bucket_fine_target(unsigned items) {
  return wg::guarded([&] {
    if (items != 0 && (items < 32 || items > static_cast<unsigned>(kCap)))
      wg::throw_invalid("fine bucket target must be 0 (default) or between 32 and 2048 items");
    g_fine_target.store(items, std::memory_order_relaxed);
  });
}

int wg_set_bucket_one_pass(int on) {
  return wg::guarded([&] {
    if (on != 0 && on != 1) wg::throw_invalid("one-pass setting must be 0 or 1");
    g_one_pass_fine.store(on != 0, std::memory_order_relaxed);
  });
}

}  // extern "C"
