// wg_expect.cu -- x-grouped statevector expectation, its adjoint, and the
// batched persistent form.
//
// Convention (reference src/expectation.cpp:121-150):
//   P|b> = i^y (-1)^{popc(z&b)} |b^x>,  y = popc(x&z),
//   e_k = <psi|P_k|psi> = sum_b conj(psi[b^x]) i^y (-1)^{popc(z&b)} psi[b]  (real),
//   E = sum_k c_k e_k.
// Terms sharing an x-mask form a group.  For x != 0 the pair (b, b^x) with one
// chosen bit of x clear in b gives t = conj(psi[b^x]) psi[b] and, since
// (-1)^{popc(z&(b^x))} = (-1)^{popc(z&b)} (-1)^y,
//   e_k = {2R, -2I, -2R, 2I}[y mod 4],  R = sum s_k(b) Re t,  I = sum s_k(b) Im t,
// over half the basis; one pass over the pairs serves every term of the group.
// For x == 0, e_k = sum_b s_k(b) |psi_b|^2.
//
// Forward schedule.  The qubit index splits into a tile (low t bits, 2^t
// amplitudes, t <= 19) and the tile number.  Groups whose x agree above the
// tile bits form a class; every group of a class pairs tile T1 with the same
// tile T1 ^ (x >> t).  Work items run class by class and tile pair by tile
// pair, so the groups of a class read a tile pair while it is in L2.  A group
// is cut into sub-groups of at most 16 terms; an item is (sub-group, tile
// pair, chunk of 2^16 pairs).  Each thread walks its pairs in Gray-code order,
// so one bit of b flips per step and the sign vector of all the sub-group's
// terms updates with one XOR (bit-sliced: bit kk of plane q says whether z_kk
// has bit q).
//
// Adjoint: (H psi)[j] = sum_g F_g(j^x_g) psi[j^x_g],
//   F_g(b) = sum_{k in g} c_k i^{y_k} (-1)^{popc(z_k&b)},
// output-stationary: a thread owns 16 outputs, walked in Gray-code order.
// Terms are cut into pieces of at most 8; F over a piece is a lookup in a
// table of its 2^8 sign patterns, so a group costs one lookup per piece.
//
// Every partial sum is stored per chunk and reduced in a fixed order: results
// are deterministic run to run.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "wg_common.cuh"

namespace {

using wgd::c128;

constexpr int kThreads = 256;
constexpr int kTileBits = 19;            // amplitudes per tile: 2^19
constexpr int kSubTerms = 16;            // terms per forward sub-group
constexpr int kChunkLog = 16;            // pairs per forward item: 2^16
constexpr int kPiece = 8;                // terms per adjoint table
constexpr int kQuadTerms = 4 * kPiece;   // terms per adjoint quad (four tables)
constexpr int kAdjR = 16;                // outputs per thread in the adjoint
constexpr int kAdjTileLog = 12;          // outputs per adjoint item: 2^12
constexpr int kAdjQuadChunk = 2048;      // quads whose tile sign masks a CTA stages at a time
constexpr uint32_t kDiagFlag = 4;        // ty bit: the term's group has x == 0

enum SubKind : uint32_t { kDiag = 0, kLowX = 1, kHighX = 2 };

struct ClassDev {
  uint32_t units;    // tile pairs (or tiles) of the class
  uint32_t ipu;      // items per unit: the chunks of every sub-group
  uint32_t s0, s1;   // sub-group range
  int pivot_hi;      // lowest set bit of x >> t (kind kHighX)
  int pad;
};

struct SubDev {
  uint64_t x;
  uint64_t pbase;    // first partial of the sub-group's terms
  uint32_t t0, nk;   // terms [t0, t0 + nk) in sorted order
  uint32_t imag;     // bit kk: term kk reads Im t
  uint32_t chunks;   // chunks per unit
  uint32_t cpre;     // chunk offset of the sub-group within its class's unit
  uint32_t chlog;    // pairs per chunk: 2^chlog
  uint32_t nch;      // partials per term: units * chunks
  uint32_t kind;     // SubKind
  int pivot;         // lowest set bit of x (kind kLowX)
  int pad;
};

struct QuadDev {
  uint64_t x;
  uint32_t t0, nk;      // terms [t0, t0 + nk), at most 32
  uint32_t tbase[4];    // table offsets of the four pieces
  uint32_t plane[4];    // sign planes of bits 8..11 (Gray steps of the adjoint)
};

// Device-side description of one operator (kernel parameter, by value).
struct PlanDev {
  int n, t;
  uint32_t T, G, NC, S, Q;
  uint64_t items;            // forward items
  const uint64_t* cls_item;  // [NC+1] item prefix per class
  const ClassDev* cls;       // [NC]
  const SubDev* sub;         // [S]
  const uint32_t* zpl;       // [S][64] sign planes
  const QuadDev* quad;       // [Q]
  const uint64_t* tz;        // [T] sorted z-masks
  const uint32_t* ty;        // [T] y mod 4 | kDiagFlag
  const uint32_t* torig;     // [T] original index of sorted term
  const uint64_t* tpbase;    // [T] first partial of the term
  const uint32_t* tnch;      // [T] partials of the term
  const double* coeffs;      // [2T] original-order coefficients
  double* td;                // [2T] sorted c_k * i^y
  double* table;             // [2 * entries] adjoint tables
  double* partial;           // forward partial sums
  uint32_t* stid;            // [Q][256] adjoint: bit kk = parity(z_kk & l) for lane offset l
};

struct wg_plan_host {
  int device;
  PlanDev dev;
  size_t n_groups = 0;
  wg::Scratch blob, coeffs, td, table, partial, stid;
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
  const uint64_t* item_base;  // [np+1] forward items per pair
  const uint64_t* term_base;  // [np+1] flat term offsets
  const uint64_t* tile_base;  // [np+1] adjoint items (0 for pairs without H psi)
  const void* const* psis;    // [np]
  double* const* evals;       // [np] e_k outputs (original order)
  double* const* results;     // [np] E outputs or null
  double* const* hpsis;       // [np] H psi outputs or null
  unsigned long long* counters;  // [2] forward / adjoint work queues
  uint32_t np;
  uint64_t n_items, n_terms, n_tiles;
};

template <typename T>
__device__ __forceinline__ uint32_t upper_index(const T* base, uint32_t n, T v) {
  // last i in [0, n) with base[i] <= v (base[0] <= v assumed)
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (base[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------- forward

struct FwdShared {
  uint32_t zpl[64];
  uint64_t gmask[8];   // Gray level l: bit of b that flips
  uint32_t gpl[8];     // Gray level l: sign plane of that bit
  double red[kThreads / 32][kSubTerms];
  unsigned long long item;
};

template <typename Amp, int KIND, int NK>
__device__ __forceinline__ void forward_item(const PlanDev& P, const void* psi, const SubDev& sd, uint32_t u,
                                             uint32_t ch, const ClassDev& cd, FwdShared& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t CH = uint64_t{1} << sd.chlog;
  const int K = CH >= kThreads ? static_cast<int>(CH / kThreads) : 1;
  const bool active = static_cast<uint64_t>(tid) < CH;
  const int t = P.t;
  const uint64_t x = sd.x;
  // Gray-step tables: level l flips pair-index bit 8 + l, i.e. bit q(l) of b
  if (tid < 8) {
    const int j = 8 + tid;
    const int q = KIND == kLowX ? j + (j >= sd.pivot ? 1 : 0) : j;
    sh.gmask[tid] = q < 64 ? uint64_t{1} << q : 0;
    sh.gpl[tid] = q < 64 ? sh.zpl[q] : 0u;
  }
  __syncthreads();
  double accr[NK], acci[NK];
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) accr[kk] = acci[kk] = 0.0;
  double tre = 0.0, tim = 0.0;
  if (active) {
    const uint64_t h0 = static_cast<uint64_t>(ch) * CH + tid;
    uint64_t b;
    if (KIND == kDiag) b = (static_cast<uint64_t>(u) << t) | h0;
    else if (KIND == kHighX) b = (insert_zero(u, cd.pivot_hi) << t) | h0;
    else b = insert_zero((static_cast<uint64_t>(u) << (t - 1)) | h0, sd.pivot);
    uint32_t S = 0;
    for (uint32_t kk = 0; kk < sd.nk; ++kk) S |= static_cast<uint32_t>(__popcll(P.tz[sd.t0 + kk] & b) & 1) << kk;
    const uint64_t m0 = sh.gmask[0];
    const uint32_t p0 = sh.gpl[0];
    // one pair: t = conj(psi[b ^ x]) psi[b]; every term with odd sign parity
    // adds t to its masked sum (Re or Im is taken at the end)
    auto pair = [&](uint64_t bb, uint32_t SS) {
      const c128 a = load_amp<Amp>(psi, bb);
      double vre, vim = 0.0;
      if (KIND == kDiag) {
        vre = a.re * a.re + a.im * a.im;
      } else {
        const c128 w = load_amp<Amp>(psi, bb ^ x);
        vre = w.re * a.re + w.im * a.im;
        vim = w.re * a.im - w.im * a.re;
      }
      tre += vre;
      if (KIND != kDiag) tim += vim;
#pragma unroll
      for (int kk = 0; kk < NK; ++kk) {
        if ((SS >> kk) & 1u) {
          accr[kk] += vre;
          if (KIND != kDiag) acci[kk] += vim;
        }
      }
    };
    for (int k = 0; k < K; k += 2) {
      if (k > 0) {
        const int l = __ffs(k) - 1;  // >= 1
        b ^= sh.gmask[l];
        S ^= sh.gpl[l];
      }
      pair(b, S);
      if (k + 1 < K) {
        b ^= m0;
        S ^= p0;
        pair(b, S);
      }
    }
  }
  // per-term value: (sum of all) - 2 (sum over odd sign parity)
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    const bool im = KIND != kDiag && ((sd.imag >> kk) & 1u);
    const double v = im ? tim - 2.0 * acci[kk] : tre - 2.0 * accr[kk];
    const double w = warp_sum(v);
    if (lane == 0) sh.red[warp][kk] = w;
  }
  __syncthreads();
  if (tid < static_cast<int>(sd.nk)) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += sh.red[w][tid];
    P.partial[sd.pbase + static_cast<uint64_t>(tid) * sd.nch + static_cast<uint64_t>(u) * sd.chunks + ch] = s;
  }
}

template <typename Amp, int KIND>
__device__ __forceinline__ void forward_dispatch(const PlanDev& P, const void* psi, const SubDev& sd, uint32_t u,
                                                 uint32_t ch, const ClassDev& cd, FwdShared& sh) {
  switch ((sd.nk + 1) >> 1) {
    case 0:
    case 1: forward_item<Amp, KIND, 2>(P, psi, sd, u, ch, cd, sh); break;
    case 2: forward_item<Amp, KIND, 4>(P, psi, sd, u, ch, cd, sh); break;
    case 3: forward_item<Amp, KIND, 6>(P, psi, sd, u, ch, cd, sh); break;
    case 4: forward_item<Amp, KIND, 8>(P, psi, sd, u, ch, cd, sh); break;
    case 5: forward_item<Amp, KIND, 10>(P, psi, sd, u, ch, cd, sh); break;
    case 6: forward_item<Amp, KIND, 12>(P, psi, sd, u, ch, cd, sh); break;
    case 7: forward_item<Amp, KIND, 14>(P, psi, sd, u, ch, cd, sh); break;
    default: forward_item<Amp, KIND, 16>(P, psi, sd, u, ch, cd, sh); break;
  }
}

template <typename Amp>
__global__ void __launch_bounds__(kThreads) expect_forward_kernel(BatchDev B) {
  __shared__ FwdShared sh;
  while (true) {
    if (threadIdx.x == 0) sh.item = atomicAdd(B.counters, 1ull);
    __syncthreads();
    const uint64_t item = sh.item;
    if (item >= B.n_items) break;
    const uint32_t p = upper_index<uint64_t>(B.item_base, B.np + 1, item);
    const PlanDev& P = B.plans[p];
    const uint64_t r = item - B.item_base[p];
    const uint32_t c = upper_index<uint64_t>(P.cls_item, P.NC + 1, r);
    const ClassDev cd = P.cls[c];
    const uint64_t rc = r - P.cls_item[c];
    const uint32_t u = static_cast<uint32_t>(rc / cd.ipu);
    const uint32_t r2 = static_cast<uint32_t>(rc - static_cast<uint64_t>(u) * cd.ipu);
    // sub-group: last s in [s0, s1) with cpre <= r2
    uint32_t lo = cd.s0, hi = cd.s1;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (P.sub[mid].cpre <= r2) lo = mid;
      else hi = mid;
    }
    const SubDev sd = P.sub[lo];
    const uint32_t ch = r2 - sd.cpre;
    for (int q = threadIdx.x; q < 64; q += kThreads) sh.zpl[q] = q < P.n ? P.zpl[static_cast<uint64_t>(lo) * 64 + q] : 0u;
    __syncthreads();
    const void* psi = B.psis[p];
    if (sd.kind == kDiag) forward_dispatch<Amp, kDiag>(P, psi, sd, u, ch, cd, sh);
    else if (sd.kind == kLowX) forward_dispatch<Amp, kLowX>(P, psi, sd, u, ch, cd, sh);
    else forward_dispatch<Amp, kHighX>(P, psi, sd, u, ch, cd, sh);
    __syncthreads();
  }
}

// e_k from the chunk partials (summed in chunk order), scaled by the pairing
// factor and scattered to original term order; flat over every pair's terms.
__global__ void __launch_bounds__(kThreads) expect_finish_terms_kernel(BatchDev B) {
  for (uint64_t f = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; f < B.n_terms;
       f += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t p = upper_index<uint64_t>(B.term_base, B.np + 1, f);
    const PlanDev& P = B.plans[p];
    const uint32_t k = static_cast<uint32_t>(f - B.term_base[p]);
    const double* part = P.partial + P.tpbase[k];
    const uint32_t nch = P.tnch[k];
    double s = 0.0;
    for (uint32_t c = 0; c < nch; ++c) s += part[c];
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

// ------------------------------------------------------------- adjoint

// Output-stationary adjoint over all pairs' tiles (persistent work queue): a
// thread owns the outputs j = tile0 + tid + 256 gray(r), r < R.
template <typename Amp>
__global__ void __launch_bounds__(kThreads) expect_adjoint_kernel(BatchDev B) {
  __shared__ unsigned long long s_item;
  __shared__ uint32_t s_hi[kAdjQuadChunk];  // per quad of the chunk: parity(z & (hi ^ x)) masks
  const int tid = threadIdx.x;
  while (true) {
    if (tid == 0) s_item = atomicAdd(B.counters + 1, 1ull);
    __syncthreads();
    const uint64_t item = s_item;
    __syncthreads();
    if (item >= B.n_tiles) break;
    const uint32_t p = upper_index<uint64_t>(B.tile_base, B.np + 1, item);
    const PlanDev& P = B.plans[p];
    const void* psi = B.psis[p];
    double* hpsi = B.hpsis[p];
    const int tlog = P.n < kAdjTileLog ? P.n : kAdjTileLog;
    const uint64_t TS = uint64_t{1} << tlog;
    const int R = TS >= kThreads ? static_cast<int>(TS / kThreads) : 1;
    const bool active = static_cast<uint64_t>(tid) < TS;
    // b = j0 ^ x splits into the tile's bits and the lane's: j0 = hi + tid
    // with hi a multiple of TS (>= 256 or 0), so a term's sign parity(z & b)
    // is parity(z & (hi ^ x)) -- staged per quad by the CTA, once per tile --
    // XOR parity(z & tid), the plan's stid table.
    const uint64_t hi = (item - B.tile_base[p]) * TS;
    const uint64_t j0 = hi + tid;
    c128 acc[kAdjR];
#pragma unroll
    for (int r = 0; r < kAdjR; ++r) acc[r] = {0.0, 0.0};
    const double2* tab = reinterpret_cast<const double2*>(P.table);
    for (uint32_t q0 = 0; q0 < P.Q; q0 += kAdjQuadChunk) {
      const uint32_t qn = min(static_cast<uint32_t>(kAdjQuadChunk), P.Q - q0);
      __syncthreads();  // the previous chunk's masks are read
      for (uint32_t qq = tid; qq < qn; qq += kThreads) {
        const QuadDev* qd = P.quad + q0 + qq;
        const uint64_t hb = hi ^ qd->x;
        const uint32_t nk = qd->nk, t0 = qd->t0;
        uint32_t m = 0;
        for (uint32_t kk = 0; kk < nk; ++kk) m |= static_cast<uint32_t>(__popcll(P.tz[t0 + kk] & hb) & 1) << kk;
        s_hi[qq] = m;
      }
      __syncthreads();
      if (!active) continue;
      for (uint32_t qq = 0; qq < qn; ++qq) {
        const uint32_t qi = q0 + qq;
        const QuadDev* qd = P.quad + qi;  // read in place: its small arrays are indexed at run time
        const uint32_t nk = qd->nk;
        uint64_t b = j0 ^ qd->x;
        uint32_t S = s_hi[qq] ^ P.stid[static_cast<size_t>(qi) * kThreads + tid];
        const int np = static_cast<int>((nk + kPiece - 1) / kPiece);
        uint32_t pl[4], tb[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          pl[q] = qd->plane[q];
          tb[q] = qd->tbase[q];
        }
#pragma unroll
        for (int r = 0; r < kAdjR; ++r) {
          if (r < R) {
            if (r > 0) {
              // Gray step flips output bit 8 + ctz(r), and the same bit of b
              const int j = (r & 1) ? 0 : (r & 2) ? 1 : (r & 4) ? 2 : 3;
              b ^= uint64_t{1} << (8 + j);
              S ^= pl[j];
            }
            const double2 f0 = tab[tb[0] + (S & 0xffu)];
            double fre = f0.x, fim = f0.y;
#pragma unroll
            for (int pc = 1; pc < 4; ++pc) {
              if (pc < np) {
                const double2 f = tab[tb[pc] + ((S >> (kPiece * pc)) & 0xffu)];
                fre += f.x;
                fim += f.y;
              }
            }
            const c128 v = load_amp<Amp>(psi, b);
            acc[r].re += v.re * fre - v.im * fim;
            acc[r].im += v.re * fim + v.im * fre;
          }
        }
      }
    }
    if (!active) continue;
    uint64_t j = j0;
#pragma unroll
    for (int r = 0; r < kAdjR; ++r) {
      if (r < R) {
        if (r > 0) j ^= uint64_t{1} << (8 + ((r & 1) ? 0 : (r & 2) ? 1 : (r & 4) ? 2 : 3));
        reinterpret_cast<double2*>(hpsi)[j] = make_double2(acc[r].re, acc[r].im);
      }
    }
  }
}

// ------------------------------------------------------------- plan build

// stid[q][l] bit kk = parity(z_kk & l) over the terms of quad q, for the
// adjoint's lane offsets l < 256 (z-masks only: built once per plan).
__global__ void plan_stid_kernel(PlanDev P) {
  const uint32_t l = threadIdx.x;
  for (uint32_t q = blockIdx.x; q < P.Q; q += gridDim.x) {
    const QuadDev* qd = P.quad + q;
    const uint32_t nk = qd->nk, t0 = qd->t0;
    uint32_t m = 0;
    for (uint32_t kk = 0; kk < nk; ++kk) m |= static_cast<uint32_t>(__popcll(P.tz[t0 + kk] & l) & 1) << kk;
    P.stid[static_cast<size_t>(q) * kThreads + l] = m;
  }
}

// td[i] = c[torig[i]] * i^{y_i} (sorted order).
__global__ void plan_coeffs_kernel(PlanDev P) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.T; i += gridDim.x * blockDim.x) {
    const uint32_t o = P.torig[i];
    const c128 d = wgd::rotate(c128{P.coeffs[2 * o], P.coeffs[2 * o + 1]}, P.ty[i] & 3u);
    P.td[2 * i] = d.re;
    P.td[2 * i + 1] = d.im;
  }
}

// Adjoint tables: entry s of a piece = sum over its terms of td * (-1)^{bit kk of s},
// in term order; one block per quad.
__global__ void plan_tables_kernel(PlanDev P) {
  for (uint32_t qi = blockIdx.x; qi < P.Q; qi += gridDim.x) {
    const QuadDev qd = P.quad[qi];
    for (uint32_t pc = 0; pc * kPiece < qd.nk; ++pc) {
      const uint32_t t0 = qd.t0 + pc * kPiece;
      const uint32_t np = min(static_cast<uint32_t>(kPiece), qd.nk - pc * kPiece);
      for (uint32_t s = threadIdx.x; s < (1u << np); s += blockDim.x) {
        double re = 0.0, im = 0.0;
        for (uint32_t kk = 0; kk < np; ++kk) {
          const double dre = P.td[2 * (t0 + kk)], dim = P.td[2 * (t0 + kk) + 1];
          if ((s >> kk) & 1u) {
            re -= dre;
            im -= dim;
          } else {
            re += dre;
            im += dim;
          }
        }
        P.table[2 * (qd.tbase[pc] + s)] = re;
        P.table[2 * (qd.tbase[pc] + s) + 1] = im;
      }
    }
  }
}

void refresh_coeffs(const wg_plan_host& h, cudaStream_t s) {
  const PlanDev& P = h.dev;
  if (P.T == 0) return;
  plan_coeffs_kernel<<<wg::grid_for(P.T, kThreads, h.device, 4), kThreads, 0, s>>>(P);
  wg::check_launch("launch plan coefficients");
  if (P.Q) {
    plan_tables_kernel<<<std::min<uint32_t>(P.Q, 65535u), kThreads, 0, s>>>(P);
    wg::check_launch("launch adjoint tables");
  }
}

// Appends raw bytes to the host image of the plan, 16-byte aligned.
struct Blob {
  std::vector<unsigned char> bytes;
  template <typename T>
  size_t put(const std::vector<T>& v) {
    const size_t at = (bytes.size() + 15) & ~size_t{15};
    bytes.resize(at + sizeof(T) * v.size());
    if (!v.empty()) std::memcpy(bytes.data() + at, v.data(), sizeof(T) * v.size());
    return at;
  }
};

wg_plan_host* make_plan(int device, size_t n, size_t T, const uint64_t* x, const uint64_t* z, const double* c,
                        cudaStream_t s) {
  if (n > 63) wg::throw_invalid("expectation_statevector requires num_qubits <= 63");
  if (T > 0xffffffffull) wg::throw_invalid("expectation supports at most 2^32-1 terms");
  std::unique_ptr<wg_plan_host> p(new wg_plan_host());
  p->device = device;
  PlanDev& d = p->dev;
  std::memset(&d, 0, sizeof(d));
  d.n = static_cast<int>(n);
  d.T = static_cast<uint32_t>(T);
  d.t = std::min<int>(static_cast<int>(n), kTileBits);
  p->coeffs.reset(std::max<size_t>(16, 16 * T), s);
  if (T) wg::check_cuda(cudaMemcpyAsync(p->coeffs.get(), c, 16 * T, cudaMemcpyDeviceToDevice, s), "copy coefficients");
  d.coeffs = p->coeffs.as<double>();
  if (T == 0) {
    wg::check_cuda(cudaStreamSynchronize(s), "build plan");
    p->coeffs.rebind(nullptr);
    return p.release();
  }
  // masks to the host; the plan's tables are built there
  const int words = n == 0 ? 0 : 1;
  std::vector<uint64_t> hx(T, 0), hz(T, 0);
  if (words) {
    wg::check_cuda(cudaMemcpyAsync(hx.data(), x, 8 * T, cudaMemcpyDeviceToHost, s), "read x masks");
    wg::check_cuda(cudaMemcpyAsync(hz.data(), z, 8 * T, cudaMemcpyDeviceToHost, s), "read z masks");
  }
  wg::check_cuda(cudaStreamSynchronize(s), "read masks");
  if (words && n < 64) {
    uint64_t bits = 0;
    for (size_t i = 0; i < T; ++i) bits |= hx[i] | hz[i];
    // the kernels index psi[b ^ x]: masks must stay below 2^n
    if ((bits >> n) != 0) wg::throw_invalid("Pauli masks set bits at or above num_qubits");
  }
  // terms sorted by x (stable): groups
  std::vector<uint32_t> order(T);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return hx[a] < hx[b]; });
  const int t = d.t;
  std::vector<uint64_t> tz(T), tpbase(T);
  std::vector<uint32_t> ty(T), torig(T), tnch(T);
  std::vector<ClassDev> cls;
  std::vector<uint64_t> cls_item{0};
  std::vector<SubDev> sub;
  std::vector<uint32_t> zpl;
  std::vector<QuadDev> quad;
  uint32_t table_entries = 0;
  uint64_t pbase = 0;
  size_t groups = 0;
  for (size_t i = 0; i < T; ++i) {
    const uint32_t o = order[i];
    tz[i] = hz[o];
    ty[i] = static_cast<uint32_t>(__builtin_popcountll(hx[o] & hz[o]) & 3) | (hx[o] == 0 ? kDiagFlag : 0u);
    torig[i] = o;
  }
  size_t g0 = 0;
  while (g0 < T) {
    // one class: groups with equal x >> t
    const uint64_t xhi = t < 64 ? (hx[order[g0]] >> t) : 0;
    ClassDev cd{};
    cd.s0 = static_cast<uint32_t>(sub.size());
    cd.pivot_hi = xhi ? __builtin_ctzll(xhi) : 0;
    const int rest = static_cast<int>(n) - t;  // tile-number bits
    cd.units = xhi ? (rest > 0 ? 1u << (rest - 1) : 1u) : (1u << rest);
    size_t gi = g0;
    uint32_t cpre = 0;
    std::vector<size_t> class_subs;
    while (gi < T && (t < 64 ? (hx[order[gi]] >> t) : 0) == xhi) {
      const uint64_t gx = hx[order[gi]];
      size_t ge = gi;
      while (ge < T && hx[order[ge]] == gx) ++ge;
      ++groups;
      // forward sub-groups
      for (size_t s0 = gi; s0 < ge; s0 += kSubTerms) {
        SubDev sd{};
        sd.x = gx;
        sd.t0 = static_cast<uint32_t>(s0);
        sd.nk = static_cast<uint32_t>(std::min<size_t>(kSubTerms, ge - s0));
        sd.kind = gx == 0 ? kDiag : (xhi ? kHighX : kLowX);
        sd.pivot = gx ? __builtin_ctzll(gx) : 0;
        const int replog = sd.kind == kLowX ? t - 1 : t;
        sd.chlog = static_cast<uint32_t>(std::min(kChunkLog, replog));
        sd.chunks = 1u << (replog - static_cast<int>(sd.chlog));
        sd.nch = cd.units * sd.chunks;
        sd.cpre = cpre;
        cpre += sd.chunks;
        sd.pbase = pbase;
        pbase += static_cast<uint64_t>(sd.nk) * sd.nch;
        for (uint32_t kk = 0; kk < sd.nk; ++kk) {
          if (ty[s0 + kk] & 1u) sd.imag |= 1u << kk;
          tpbase[s0 + kk] = sd.pbase + static_cast<uint64_t>(kk) * sd.nch;
          tnch[s0 + kk] = sd.nch;
        }
        for (int q = 0; q < 64; ++q) {
          uint32_t m = 0;
          for (uint32_t kk = 0; kk < sd.nk; ++kk)
            if (q < static_cast<int>(n) && ((tz[s0 + kk] >> q) & 1u)) m |= 1u << kk;
          zpl.push_back(m);
        }
        sub.push_back(sd);
      }
      // adjoint quads
      for (size_t q0 = gi; q0 < ge; q0 += kQuadTerms) {
        QuadDev qd{};
        qd.x = gx;
        qd.t0 = static_cast<uint32_t>(q0);
        qd.nk = static_cast<uint32_t>(std::min<size_t>(kQuadTerms, ge - q0));
        for (uint32_t pc = 0; pc * kPiece < qd.nk; ++pc) {
          const uint32_t np = std::min<uint32_t>(kPiece, qd.nk - pc * kPiece);
          qd.tbase[pc] = table_entries;
          table_entries += 1u << np;
        }
        for (int j = 0; j < 4; ++j) {
          uint32_t m = 0;
          const int bit = 8 + j;
          for (uint32_t kk = 0; kk < qd.nk; ++kk)
            if (bit < static_cast<int>(n) && ((tz[q0 + kk] >> bit) & 1u)) m |= 1u << kk;
          qd.plane[j] = m;
        }
        quad.push_back(qd);
      }
      gi = ge;
    }
    cd.s1 = static_cast<uint32_t>(sub.size());
    cd.ipu = cpre;
    cls.push_back(cd);
    cls_item.push_back(cls_item.back() + static_cast<uint64_t>(cd.units) * cd.ipu);
    g0 = gi;
  }
  d.NC = static_cast<uint32_t>(cls.size());
  d.S = static_cast<uint32_t>(sub.size());
  d.Q = static_cast<uint32_t>(quad.size());
  d.G = static_cast<uint32_t>(groups);
  d.items = cls_item.back();
  p->n_groups = groups;
  Blob blob;
  const size_t o_ci = blob.put(cls_item), o_cls = blob.put(cls), o_sub = blob.put(sub), o_zpl = blob.put(zpl),
               o_quad = blob.put(quad), o_tz = blob.put(tz), o_ty = blob.put(ty), o_torig = blob.put(torig),
               o_tpb = blob.put(tpbase), o_tnch = blob.put(tnch);
  p->blob.reset(blob.bytes.size(), s);
  wg::check_cuda(cudaMemcpyAsync(p->blob.get(), blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice, s),
                 "upload plan");
  auto* base = static_cast<unsigned char*>(p->blob.get());
  d.cls_item = reinterpret_cast<const uint64_t*>(base + o_ci);
  d.cls = reinterpret_cast<const ClassDev*>(base + o_cls);
  d.sub = reinterpret_cast<const SubDev*>(base + o_sub);
  d.zpl = reinterpret_cast<const uint32_t*>(base + o_zpl);
  d.quad = reinterpret_cast<const QuadDev*>(base + o_quad);
  d.tz = reinterpret_cast<const uint64_t*>(base + o_tz);
  d.ty = reinterpret_cast<const uint32_t*>(base + o_ty);
  d.torig = reinterpret_cast<const uint32_t*>(base + o_torig);
  d.tpbase = reinterpret_cast<const uint64_t*>(base + o_tpb);
  d.tnch = reinterpret_cast<const uint32_t*>(base + o_tnch);
  p->td.reset(16 * T, s);
  p->table.reset(16 * std::max<size_t>(1, table_entries), s);
  p->partial.reset(8 * std::max<uint64_t>(1, pbase), s);
  p->stid.reset(4 * kThreads * std::max<size_t>(1, d.Q), s);
  d.td = p->td.as<double>();
  d.table = p->table.as<double>();
  d.partial = p->partial.as<double>();
  d.stid = p->stid.as<uint32_t>();
  if (d.Q) {
    plan_stid_kernel<<<std::min<uint32_t>(d.Q, 65535u), kThreads, 0, s>>>(d);
    wg::check_launch("launch adjoint lane signs");
  }
  refresh_coeffs(*p, s);
  // pageable source above: wait until the plan image is on the device
  wg::check_cuda(cudaStreamSynchronize(s), "build plan");
  // The plan outlives the caller's stream: release its buffers on the legacy
  // default stream.
  for (wg::Scratch* b : {&p->blob, &p->coeffs, &p->td, &p->table, &p->partial, &p->stid}) b->rebind(nullptr);
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
    item_base[i + 1] = item_base[i] + (P.T ? P.items : 0);
    term_base[i + 1] = term_base[i] + P.T;
    const int tlog = P.n < kAdjTileLog ? P.n : kAdjTileLog;
    const bool adj = specs[i].hpsi != nullptr && P.T != 0;
    tile_base[i + 1] = tile_base[i] + (adj ? (uint64_t{1} << (P.n - tlog)) : 0);
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
    refresh_coeffs(plan->h, stream);
  });
}

int wg_expect_plan_info(wg_expect_plan_t plan, size_t* n_groups, size_t* n_terms) {
  return wg::guarded([&] {
    if (!plan) wg::throw_invalid("expectation plan is null");
    *n_groups = plan->h.n_groups;
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
