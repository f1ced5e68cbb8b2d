// wg_commute.cu -- bit-packed all-pairs commutation matrix and its consumers.
//
// Semantics (reference src/detail/commutation.hpp:10-46, src/commute.cpp:27-93):
// terms l and r commute iff parity(sum_w popc((lx_w & rz_w) ^ (lz_w & rx_w))) == 0.
// Because parity is additive over XOR, all words fold into one 64-bit value
// before a single population count.
//
// Output: bits[row*pitch + c/32] bit (c%32) = 1 iff (row, c) commute.  The
// reference writes one byte per entry (src/cuda/commutation_cuda.cu:123-151);
// the bit matrix is 8x smaller, which is what bounds the kernel at large sizes.

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "wg_common.cuh"

namespace {

constexpr int kColsPerLane = 8;                    // rhs columns held in registers per lane
constexpr int kWarpCols = 32 * kColsPerLane;       // 256 columns = 8 output words per warp
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRowsPerWarpIter = 64;               // rows a warp sweeps per column tile

// ---------------------------------------------------------------------------
// algo 1: popcount / LOP3 with warp-ballot packing.
// CTA = one 256-column tile x (kWarps * kRowsPerWarpIter) rows.  Every lane
// keeps the masks of its 8 columns in registers; each row's masks are a
// broadcast load; the 8 ballots of a row give 8 consecutive output words,
// stored by lanes 0..7 as one 32-byte sector.
template <int W>
__global__ void __launch_bounds__(kThreads) commute_ballot_kernel(
    const uint64_t* __restrict__ lx, const uint64_t* __restrict__ lz, size_t n_l,
    const uint64_t* __restrict__ rx, const uint64_t* __restrict__ rz, size_t n_r,
    uint32_t* __restrict__ bits, size_t pitch) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const size_t col_tile = blockIdx.x;
  const size_t col0 = col_tile * kWarpCols;
  const size_t words_needed = (n_r + 31) / 32;

  uint64_t cx[kColsPerLane][W], cz[kColsPerLane][W];
  uint32_t valid = 0;  // bit k: column k of this lane exists
#pragma unroll
  for (int k = 0; k < kColsPerLane; ++k) {
    const size_t c = col0 + 32 * k + lane;
    const bool ok = c < n_r;
    valid |= ok ? (1u << k) : 0u;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      cx[k][w] = ok ? __ldg(rx + c * W + w) : 0;
      cz[k][w] = ok ? __ldg(rz + c * W + w) : 0;
    }
  }
  // Word k of this tile holds columns col0 + 32k + lane; mask off absent ones.
  uint32_t word_valid[kColsPerLane];
#pragma unroll
  for (int k = 0; k < kColsPerLane; ++k) word_valid[k] = __ballot_sync(0xffffffffu, (valid >> k) & 1u);

  const size_t row_begin = static_cast<size_t>(blockIdx.y) * (kWarps * kRowsPerWarpIter) + warp;
  const size_t row_end = min(n_l, static_cast<size_t>(blockIdx.y + 1) * (kWarps * kRowsPerWarpIter));
  for (size_t row = row_begin; row < row_end; row += kWarps) {
    uint64_t ax[W], az[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      ax[w] = __ldg(lx + row * W + w);
      az[w] = __ldg(lz + row * W + w);
    }
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < kColsPerLane; ++k) {
      uint64_t acc = 0;
#pragma unroll
      for (int w = 0; w < W; ++w) acc ^= (ax[w] & cz[k][w]) ^ (az[w] & cx[k][w]);
      const uint32_t folded = static_cast<uint32_t>(acc) ^ static_cast<uint32_t>(acc >> 32);
      const bool commute = (__popc(folded) & 1u) == 0;
      const uint32_t word = __ballot_sync(0xffffffffu, commute) & word_valid[k];
      if (lane == k) mine = word;
    }
    const size_t wi = col_tile * kColsPerLane + lane;
    if (lane < kColsPerLane && wi < words_needed) bits[row * pitch + wi] = mine;
  }
}

// Generic word count (W > 4): masks read per pair from global/L1.
__global__ void __launch_bounds__(kThreads) commute_generic_kernel(
    const uint64_t* __restrict__ lx, const uint64_t* __restrict__ lz, size_t n_l,
    const uint64_t* __restrict__ rx, const uint64_t* __restrict__ rz, size_t n_r, size_t W,
    uint32_t* __restrict__ bits, size_t pitch) {
  const int lane = threadIdx.x & 31;
  const size_t words_needed = (n_r + 31) / 32;
  const size_t total = n_l * words_needed;
  const size_t warp_global = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = (static_cast<size_t>(gridDim.x) * blockDim.x) >> 5;
  for (size_t item = warp_global; item < total; item += nwarps) {
    const size_t row = item / words_needed;
    const size_t wi = item - row * words_needed;
    const size_t c = wi * 32 + lane;
    bool commute = false;
    if (c < n_r) {
      uint64_t acc = 0;
      for (size_t w = 0; w < W; ++w)
        acc ^= (lx[row * W + w] & rz[c * W + w]) ^ (lz[row * W + w] & rx[c * W + w]);
      commute = (__popcll(acc) & 1u) == 0;
    }
    const uint32_t word = __ballot_sync(0xffffffffu, commute);
    if (lane == 0) bits[row * pitch + wi] = word;
  }
}

// n_qubits == 0: every pair commutes.
__global__ void fill_ones_kernel(uint32_t* bits, size_t rows, size_t cols, size_t pitch) {
  const size_t words_needed = (cols + 31) / 32;
  const size_t total = rows * words_needed;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t row = i / words_needed;
    const size_t wi = i - row * words_needed;
    const size_t rem = cols - wi * 32;
    bits[row * pitch + wi] = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
  }
}

// ---------------------------------------------------------------------------
// algo 2: bit-plane XOR.  For a block of 32*LW*32 rhs columns, plane (q,
// X|Z) is the bit-vector over the block of the rhs x/z bits on qubit q.  Row
// l's output word j is the complement of XOR over q in supp(l) of
// (lx_q ? Zplane_q[j] : 0) ^ (lz_q ? Xplane_q[j] : 0).  Per output word that
// is ~weight(l) shared-memory reads instead of 32 * (4W LOP3 + POPC), so for
// sparse terms the kernel is bound by issue, not by POPC.  Each lane owns LW
// consecutive output words of a row (read as one LW-word vector per plane):
// LW = 4 with 1,024 threads for large products of 1-2 mask words (planes take
// up to 128 KB of shared memory), LW = 2 with 256 threads otherwise.
constexpr int kMaxConfiguredDevices = 64;
constexpr int kRowList = 16;  // plane offsets listed per row; rows with more set bits loop over their masks

template <int LW>
__device__ __forceinline__ void xor_plane(uint32_t (&acc)[LW], const uint32_t* planes, int vec) {
  if constexpr (LW == 4) {
    const uint4 v = reinterpret_cast<const uint4*>(planes)[vec];
    acc[0] ^= v.x;
    acc[1] ^= v.y;
    acc[2] ^= v.z;
    acc[3] ^= v.w;
  } else {
    static_assert(LW == 2, "two or four output words per lane");
    const uint2 v = reinterpret_cast<const uint2*>(planes)[vec];
    acc[0] ^= v.x;
    acc[1] ^= v.y;
  }
}

template <int W, int LW, int THREADS>
__global__ void __launch_bounds__(THREADS) commute_plane_kernel(
    const uint64_t* __restrict__ lx, const uint64_t* __restrict__ lz, size_t n_l,
    const uint64_t* __restrict__ rx, const uint64_t* __restrict__ rz, size_t n_r,
    uint32_t* __restrict__ bits, size_t pitch, size_t rows_per_cta) {
  constexpr int kWordsCta = 32 * LW;  // output words per row per CTA
  constexpr int kWarpsCta = THREADS / 32;
  // planes[(q*2 + 0)*kWordsCta + j] = X bits of rhs block word j on qubit q; +1 = Z bits.
  // In LW-word vectors a plane is 32 vectors long, so plane p starts at vector 32p.
  extern __shared__ __align__(16) uint32_t planes[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const size_t col0 = static_cast<size_t>(blockIdx.x) * (32 * kWordsCta);
  const size_t words_needed = (n_r + 31) / 32;
  // Build: warp handles block words j = warp, warp + kWarpsCta, ...; lane t
  // loads column col0 + 32j + t once, then one ballot per (qubit, x|z) gives a
  // plane word.
  for (int j = warp; j < kWordsCta; j += kWarpsCta) {
    const size_t c = col0 + 32 * static_cast<size_t>(j) + lane;
    const bool ok = c < n_r;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const uint64_t vx = ok ? __ldg(rx + c * W + w) : 0;
      const uint64_t vz = ok ? __ldg(rz + c * W + w) : 0;
#pragma unroll 8
      for (int b = 0; b < 64; ++b) {
        const uint32_t px = __ballot_sync(0xffffffffu, (vx >> b) & 1u);
        const uint32_t pz = __ballot_sync(0xffffffffu, (vz >> b) & 1u);
        if (lane == (b & 31)) {
          const int q = w * 64 + b;
          planes[(q * 2 + 0) * kWordsCta + j] = px;
          planes[(q * 2 + 1) * kWordsCta + j] = pz;
        }
      }
    }
  }
  __syncthreads();
  // lane covers output words LW*lane .. LW*lane + LW - 1 of the block
  uint32_t valid[LW];
  bool write_ok[LW];
  size_t wi[LW];
#pragma unroll
  for (int h = 0; h < LW; ++h) {
    const int j = LW * lane + h;
    const size_t c_first = col0 + 32 * static_cast<size_t>(j);
    valid[h] = c_first >= n_r ? 0u : (n_r - c_first < 32 ? (1u << (n_r - c_first)) - 1u : 0xffffffffu);
    wi[h] = static_cast<size_t>(blockIdx.x) * kWordsCta + j;
    write_ok[h] = wi[h] < words_needed;
  }
  const size_t row0 = static_cast<size_t>(blockIdx.y) * rows_per_cta;
  const size_t row1 = min(n_l, row0 + rows_per_cta);
  // A warp takes 32 rows at a time: lane r loads row rbase + r (coalesced)
  // and lists the plane offsets its row selects (set X bits select rhs Z
  // planes, set Z bits rhs X planes); each row's list is then read by the
  // whole warp (a broadcast, two offsets per 32-bit read), so a lane's work
  // per set bit is one LW-word shared-memory load and LW XORs.  A row with
  // more than kRowList set bits has its masks broadcast by shuffles and walked
  // bit by bit instead.
  __shared__ uint16_t lists[kWarpsCta][32][kRowList];
  __shared__ uint8_t counts[kWarpsCta][32];
  for (size_t rbase = row0 + 32 * static_cast<size_t>(warp); rbase < row1; rbase += 32 * kWarpsCta) {
    const size_t my = rbase + lane;
    uint64_t mx[W], mz[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      mx[w] = my < row1 ? __ldg(lx + my * W + w) : 0;
      mz[w] = my < row1 ? __ldg(lz + my * W + w) : 0;
    }
    {
      int cnt = 0;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        for (uint64_t m = mx[w]; m; m &= m - 1) {
          if (cnt < kRowList) lists[warp][lane][cnt] = static_cast<uint16_t>(((w * 64 + __ffsll(m) - 1) * 2 + 1) * 32);
          ++cnt;
        }
        for (uint64_t m = mz[w]; m; m &= m - 1) {
          if (cnt < kRowList) lists[warp][lane][cnt] = static_cast<uint16_t>(((w * 64 + __ffsll(m) - 1) * 2) * 32);
          ++cnt;
        }
      }
      counts[warp][lane] = static_cast<uint8_t>(cnt <= kRowList ? cnt : 255);
    }
    __syncwarp();
    const int nrows = row1 - rbase < 32 ? static_cast<int>(row1 - rbase) : 32;
    for (int rr = 0; rr < nrows; ++rr) {
      uint32_t acc[LW];
#pragma unroll
      for (int h = 0; h < LW; ++h) acc[h] = 0u;
      const int cnt = counts[warp][rr];
      if (cnt != 255) {
        const uint32_t* l2 = reinterpret_cast<const uint32_t*>(lists[warp][rr]);
        int k = 0;
        for (; k + 1 < cnt; k += 2) {
          const uint32_t pr = l2[k >> 1];
          xor_plane<LW>(acc, planes, static_cast<int>(pr & 0xffffu) + lane);
          xor_plane<LW>(acc, planes, static_cast<int>(pr >> 16) + lane);
        }
        if (k < cnt) xor_plane<LW>(acc, planes, lists[warp][rr][k] + lane);
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const uint64_t ax = __shfl_sync(0xffffffffu, mx[w], rr);
          const uint64_t az = __shfl_sync(0xffffffffu, mz[w], rr);
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int qb = w * 64 + half * 32;
            for (uint32_t m = static_cast<uint32_t>(ax >> (32 * half)); m; m &= m - 1)
              xor_plane<LW>(acc, planes, ((qb + __ffs(m) - 1) * 2 + 1) * 32 + lane);
            for (uint32_t m = static_cast<uint32_t>(az >> (32 * half)); m; m &= m - 1)
              xor_plane<LW>(acc, planes, ((qb + __ffs(m) - 1) * 2 + 0) * 32 + lane);
          }
        }
      }
      uint32_t* out = bits + (rbase + rr) * pitch + wi[0];
      if (write_ok[LW - 1] && (reinterpret_cast<uintptr_t>(out) & (4 * LW - 1)) == 0) {
        if constexpr (LW == 4)
          *reinterpret_cast<uint4*>(out) =
              make_uint4(~acc[0] & valid[0], ~acc[1] & valid[1], ~acc[2] & valid[2], ~acc[3] & valid[3]);
        else
          *reinterpret_cast<uint2*>(out) = make_uint2(~acc[0] & valid[0], ~acc[1] & valid[1]);
      } else {
#pragma unroll
        for (int h = 0; h < LW; ++h)
          if (write_ok[h]) out[h] = ~acc[h] & valid[h];
      }
    }
    __syncwarp();  // every lane is done with this batch's lists
  }
}

template <int W>
void launch_ballot(const uint64_t* lx, const uint64_t* lz, size_t n_l, const uint64_t* rx,
                   const uint64_t* rz, size_t n_r, uint32_t* bits, size_t pitch, cudaStream_t s) {
  const size_t col_tiles = (n_r + kWarpCols - 1) / kWarpCols;
  const size_t row_chunks = (n_l + kWarps * kRowsPerWarpIter - 1) / (kWarps * kRowsPerWarpIter);
  if (row_chunks > 65535) {
    // Split the launch along rows to respect gridDim.y.
    const size_t rows_per_launch = 65535ull * kWarps * kRowsPerWarpIter;
    for (size_t r0 = 0; r0 < n_l; r0 += rows_per_launch) {
      const size_t nrows = min(rows_per_launch, n_l - r0);
      launch_ballot<W>(lx + r0 * W, lz + r0 * W, nrows, rx, rz, n_r, bits + r0 * pitch, pitch, s);
    }
    return;
  }
  dim3 grid(static_cast<unsigned>(col_tiles), static_cast<unsigned>(row_chunks));
  WG_TIMED("commute_ballot_kernel", s,
    commute_ballot_kernel<W><<<grid, kThreads, 0, s>>>(lx, lz, n_l, rx, rz, n_r, bits, pitch));
  wg::check_launch("launch commutation (ballot)");
}

template <int W, int LW, int THREADS>
void launch_plane_as(const uint64_t* lx, const uint64_t* lz, size_t n_l, const uint64_t* rx, const uint64_t* rz,
                     size_t n_r, uint32_t* bits, size_t pitch, int device, cudaStream_t s, size_t max_rows = 16384) {
  constexpr int kWordsCta = 32 * LW;
  auto* kernel = commute_plane_kernel<W, LW, THREADS>;
  const size_t smem = static_cast<size_t>(64 * W) * 2 * kWordsCta * sizeof(uint32_t);
  // The shared-memory opt-in is per device and per kernel; set once per device
  // (std::call_once also orders host threads that launch concurrently).
  static std::once_flag configured[kMaxConfiguredDevices];
  if (device < 0 || device >= kMaxConfiguredDevices) wg::throw_invalid("CUDA device ordinal is out of range");
  std::call_once(configured[device], [&] {  // a throw leaves the flag unset: the next call retries
    wg::check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                   "configure bit-plane commutation");
  });
  const size_t col_blocks = (n_r + 32 * kWordsCta - 1) / (32 * kWordsCta);
  // Enough row chunks to fill the machine (at least four CTAs per SM); as many
  // rows per CTA as that allows, to amortise the plane building: on 262,144^2
  // terms 2,048 rows per CTA took 5.93 ms, 4,096 4.57, 8,192 3.88, 16,384 3.52
  // (32,768 rows at two CTAs per SM 3.80: the last wave runs part empty).
  const size_t sms = wg::device_props(device).sm_count;
  size_t rows_per_cta = max_rows;
  while (rows_per_cta > 256 && col_blocks * ((n_l + rows_per_cta - 1) / rows_per_cta) < 4 * sms)
    rows_per_cta /= 2;
  size_t row_chunks = (n_l + rows_per_cta - 1) / rows_per_cta;
  while (row_chunks > 65535) {
    rows_per_cta *= 2;
    row_chunks = (n_l + rows_per_cta - 1) / rows_per_cta;
  }
  dim3 grid(static_cast<unsigned>(col_blocks), static_cast<unsigned>(row_chunks));
  WG_TIMED("commute_plane_kernel", s,
    kernel<<<grid, THREADS, smem, s>>>(lx, lz, n_l, rx, rz, n_r, bits, pitch, rows_per_cta));
  wg::check_launch("launch commutation (bit-plane)");
}

// Candidates of the commutation autotuner (wg_tune.cu) on 1-4 mask words:
//   0 ballot kernel;
//   1 bit-plane, two output words per lane, 256 threads (2,048-column tiles);
//   2 bit-plane, four output words per lane, 1,024 threads (4,096-column
//     tiles; 1-2 mask words only: the planes of 4,096 columns take 64 KB of
//     shared memory per mask word and side);
//   3, 4 as 1, 2 with at most 2,048 lhs rows per CTA (more CTAs, each
//     building its plane tile for fewer rows).
// Returns false when the candidate does not serve this width.
template <int W>
bool launch_candidate_w(int c, const uint64_t* lx, const uint64_t* lz, size_t n_l, const uint64_t* rx,
                        const uint64_t* rz, size_t n_r, uint32_t* bits, size_t pitch, int device, cudaStream_t s) {
  switch (c) {
    case 0: launch_ballot<W>(lx, lz, n_l, rx, rz, n_r, bits, pitch, s); return true;
    case 1: launch_plane_as<W, 2, 256>(lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s); return true;
    case 3: launch_plane_as<W, 2, 256>(lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s, 2048); return true;
    case 2:
    case 4:
      if constexpr (W <= 2) {
        launch_plane_as<W, 4, 1024>(lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s, c == 2 ? 16384 : 2048);
        return true;
      }
      return false;
    default: return false;
  }
}

bool launch_candidate(int c, size_t words, const uint64_t* lx, const uint64_t* lz, size_t n_l, const uint64_t* rx,
                      const uint64_t* rz, size_t n_r, uint32_t* bits, size_t pitch, int device, cudaStream_t s) {
  switch (words) {
    case 1: return launch_candidate_w<1>(c, lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s);
    case 2: return launch_candidate_w<2>(c, lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s);
    case 3: return launch_candidate_w<3>(c, lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s);
    case 4: return launch_candidate_w<4>(c, lx, lz, n_l, rx, rz, n_r, bits, pitch, device, s);
    default: return false;
  }
}

// The measured default tile for the bit-plane kernel: four output words per
// lane and 1,024 threads (4,096-column tiles) for one or two mask words when
// both sides are large: 5.9 against 7.2 ms on 262,144^2 terms.  Smaller
// products keep two words per lane and 256 threads, where the wider tile's
// plane building would not be amortised over enough rows (32,768^2 terms: 433
// against 253 us).
int default_plane_candidate(size_t W, size_t n_l, size_t n_r) {
  return (W <= 2 && n_l >= 65536 && n_r >= 65536) ? 2 : 1;
}

// Default choice between the two algorithms, from the sizes and the word
// count alone: it reads no term data, so it costs no device-to-host copy and
// no synchronisation, and a call that uses it can be captured in a CUDA graph.
// Cost model per output word:
//   ballot: 32 pairs * (4W LOP3 + 1 POPC + pack)  ~ 32 * (4W + 2) instructions
//   plane : about 8 per set bit of the lhs row (find bit, offsets, 16-byte
//           shared load, XORs) + 16, plus the plane tile built once per CTA.
// The plane kernel wins up to a mean lhs weight of (32(4W+2) - 16) / 8, i.e.
// 22 set qubits at one word and 38 at two: every workload of this path's
// benchmark set is far below that (k-local and sparse operators of weight
// 2-8).  Small products keep the ballot kernel (no tile to amortise).  Callers
// that know the weight pass algo 1 or 2 themselves (the C++ layer estimates it
// from its host copy of the terms), and the autotuner's cached measurement
// replaces this rule for shape classes it has searched.
int default_algo(size_t W, size_t n_l, size_t n_r) {
  if (W > 4 || n_r < 512 || n_l < 64) return 1;
  return 2;
}

// wg_commutation_bits' work.  allow_search = false never measures (the
// no-allocation entry point): cached autotuner choices or the defaults only.
void commutation_bits(int device, size_t words, const uint64_t* lhs_x, const uint64_t* lhs_z, size_t n_lhs,
                      const uint64_t* rhs_x, const uint64_t* rhs_z, size_t n_rhs, uint32_t* bits,
                      size_t pitch_words, int algo, bool allow_search, cudaStream_t stream) {
    if (pitch_words < (n_rhs + 31) / 32) wg::throw_invalid("commutation bit matrix pitch is too small");
    if (algo < 0 || algo > 2) wg::throw_invalid("commutation algo must be 0, 1 or 2");
    if (n_lhs == 0 || n_rhs == 0) return;
    wg::DeviceGuard g(device);
    (void)wg::checked_mul(n_lhs, pitch_words, "commutation bit matrix");
    cudaStream_t s = stream;
    if (words == 0) {
      fill_ones_kernel<<<wg::grid_for(n_lhs * pitch_words, 256, device, 8), 256, 0, s>>>(bits, n_lhs, n_rhs,
                                                                                          pitch_words);
      wg::check_launch("launch commutation fill");
      return;
    }
    if (words <= 4) {
      const int plane = default_plane_candidate(words, n_lhs, n_rhs);
      const int fallback = algo == 1 ? 0 : algo == 2 ? plane : (default_algo(words, n_lhs, n_rhs) == 1 ? 0 : plane);
      int choice = fallback;
      bool done = false;
      if (algo == 0)
        choice = wg::tune_choose(
            wg::kTuneCommute, static_cast<int>(words), wg::ceil_log2(n_lhs), wg::ceil_log2(n_rhs), fallback,
            allow_search, s,
            [&](int c) {
              return launch_candidate(c, words, lhs_x, lhs_z, n_lhs, rhs_x, rhs_z, n_rhs, bits, pitch_words, device,
                                      s);
            },
            &done);
      if (!done && !launch_candidate(choice, words, lhs_x, lhs_z, n_lhs, rhs_x, rhs_z, n_rhs, bits, pitch_words,
                                     device, s))
        launch_candidate(fallback, words, lhs_x, lhs_z, n_lhs, rhs_x, rhs_z, n_rhs, bits, pitch_words, device, s);
      return;
    }
    const size_t items = n_lhs * ((n_rhs + 31) / 32);
    WG_TIMED("commute_generic_kernel", s,
      commute_generic_kernel<<<wg::grid_for(items * 32, 256, device, 8), 256, 0, s>>>(
          lhs_x, lhs_z, n_lhs, rhs_x, rhs_z, n_rhs, words, bits, pitch_words));
    wg::check_launch("launch commutation (generic)");
}

}  // namespace

extern "C" {

int wg_commutation_bits(int device, size_t words, const uint64_t* lhs_x, const uint64_t* lhs_z,
                        size_t n_lhs, const uint64_t* rhs_x, const uint64_t* rhs_z, size_t n_rhs,
                        uint32_t* bits, size_t pitch_words, int algo, wg_stream_t stream) {
  return wg::guarded([&] {
    commutation_bits(device, words, lhs_x, lhs_z, n_lhs, rhs_x, rhs_z, n_rhs, bits, pitch_words, algo, true,
                     stream);
  });
}

}  // extern "C"

namespace {

// One thread per output byte group of 4 (uint32 store of four 0/1 flags).
__global__ void bits_to_u8_kernel(const uint32_t* __restrict__ bits, size_t rows, size_t cols,
                                  size_t pitch, uint8_t* __restrict__ out) {
  const size_t quads = (cols + 3) / 4;
  const size_t total = rows * quads;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t row = i / quads;
    const size_t q = i - row * quads;
    const size_t c0 = q * 4;
    const uint32_t word = bits[row * pitch + c0 / 32];
    const uint32_t nib = (word >> (c0 % 32)) & 0xFu;
    const size_t base = row * cols + c0;
    if (c0 + 4 <= cols && ((reinterpret_cast<uintptr_t>(out) + base) & 3) == 0) {
      const uint32_t v = (nib & 1u) | ((nib >> 1) & 1u) << 8 | ((nib >> 2) & 1u) << 16 | ((nib >> 3) & 1u) << 24;
      *reinterpret_cast<uint32_t*>(out + base) = v;
    } else {
      for (size_t k = 0; k < 4 && c0 + k < cols; ++k) out[base + k] = (nib >> k) & 1u;
    }
  }
}

// Row counts: one warp per row.
__global__ void bits_row_count_kernel(const uint32_t* __restrict__ bits, size_t rows, size_t cols,
                                      size_t pitch, uint64_t* __restrict__ row_counts,
                                      unsigned long long* __restrict__ total) {
  const int lane = threadIdx.x & 31;
  const size_t words = (cols + 31) / 32;
  const size_t warp = (blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5;
  const size_t nwarps = (static_cast<size_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long mine = 0;
  for (size_t row = warp; row < rows; row += nwarps) {
    unsigned long long cnt = 0;
    for (size_t j = lane; j < words; j += 32) cnt += __popc(bits[row * pitch + j]);
#pragma unroll
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && row_counts) row_counts[row] = cnt;
    mine += cnt;
  }
  if (lane == 0 && total) atomicAdd(total, mine);
}

// Column counts: thread per column, rows in chunks (blockIdx.y), atomics per chunk.
__global__ void bits_col_count_kernel(const uint32_t* __restrict__ bits, size_t rows, size_t cols,
                                      size_t pitch, size_t rows_per_chunk,
                                      unsigned long long* __restrict__ col_counts) {
  const size_t c = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (c >= cols) return;
  const size_t r0 = blockIdx.y * rows_per_chunk;
  const size_t r1 = min(rows, r0 + rows_per_chunk);
  unsigned long long cnt = 0;
  for (size_t r = r0; r < r1; ++r) cnt += (bits[r * pitch + c / 32] >> (c % 32)) & 1u;
  atomicAdd(col_counts + c, cnt);
}

__global__ void u8_row_count_kernel(const uint8_t* __restrict__ f, size_t rows, size_t cols,
                                    uint64_t* __restrict__ row_counts, unsigned long long* __restrict__ total) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5;
  const size_t nwarps = (static_cast<size_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long mine = 0;
  for (size_t row = warp; row < rows; row += nwarps) {
    unsigned long long cnt = 0;
    for (size_t j = lane; j < cols; j += 32) cnt += f[row * cols + j] != 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && row_counts) row_counts[row] = cnt;
    mine += cnt;
  }
  if (lane == 0 && total) atomicAdd(total, mine);
}

__global__ void u8_col_count_kernel(const uint8_t* __restrict__ f, size_t rows, size_t cols,
                                    size_t rows_per_chunk, unsigned long long* __restrict__ col_counts) {
  const size_t c = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  if (c >= cols) return;
  const size_t r0 = blockIdx.y * rows_per_chunk;
  const size_t r1 = min(rows, r0 + rows_per_chunk);
  unsigned long long cnt = 0;
  for (size_t r = r0; r < r1; ++r) cnt += f[r * cols + c] != 0;
  atomicAdd(col_counts + c, cnt);
}

template <typename RowK, typename ColK>
void run_counts(int device, size_t rows, size_t cols, uint64_t* row_counts, uint64_t* col_counts,
                uint64_t* total, cudaStream_t s, RowK row_launch, ColK col_launch) {
  wg::Scratch tot(sizeof(unsigned long long), s);
  wg::check_cuda(cudaMemsetAsync(tot.get(), 0, sizeof(unsigned long long), s), "clear count");
  if (rows > 0 && cols > 0) {
    row_launch(tot.as<unsigned long long>());
    if (col_counts) {
      wg::check_cuda(cudaMemsetAsync(col_counts, 0, cols * sizeof(uint64_t), s), "clear column counts");
      col_launch(reinterpret_cast<unsigned long long*>(col_counts));
    }
  } else {
    if (row_counts && rows) wg::check_cuda(cudaMemsetAsync(row_counts, 0, rows * 8, s), "clear row counts");
    if (col_counts && cols) wg::check_cuda(cudaMemsetAsync(col_counts, 0, cols * 8, s), "clear column counts");
  }
  if (total) {
    unsigned long long h = 0;
    wg::check_cuda(cudaMemcpyAsync(&h, tot.get(), sizeof(h), cudaMemcpyDeviceToHost, s), "read count");
    wg::check_cuda(cudaStreamSynchronize(s), "read count");
    *total = h;
  }
}

}  // namespace

extern "C" {

int wg_bits_to_u8(int device, const uint32_t* bits, size_t rows, size_t cols, size_t pitch_words,
                  uint8_t* out, wg_stream_t stream) {
  return wg::guarded([&] {
    if (rows == 0 || cols == 0) return;
    wg::DeviceGuard g(device);
    const size_t total = rows * ((cols + 3) / 4);
    WG_TIMED("bits_to_u8_kernel", stream,
      bits_to_u8_kernel<<<wg::grid_for(total, 256, device, 8), 256, 0, stream>>>(bits, rows, cols, pitch_words, out));
    wg::check_launch("launch bits to u8");
  });
}

int wg_bits_count(int device, const uint32_t* bits, size_t rows, size_t cols, size_t pitch_words,
                  uint64_t* row_counts, uint64_t* col_counts, uint64_t* total, wg_stream_t stream) {
  return wg::guarded([&] {
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    run_counts(
        device, rows, cols, row_counts, col_counts, total, s,
        [&](unsigned long long* tot) {
          bits_row_count_kernel<<<wg::grid_for(rows * 32, 256, device, 8), 256, 0, s>>>(bits, rows, cols, pitch_words,
                                                                                       row_counts, tot);
          wg::check_launch("launch row counts");
        },
        [&](unsigned long long* cc) {
          const size_t chunk = 4096;
          dim3 grid(static_cast<unsigned>((cols + 255) / 256), static_cast<unsigned>((rows + chunk - 1) / chunk));
          bits_col_count_kernel<<<grid, 256, 0, s>>>(bits, rows, cols, pitch_words, chunk, cc);
          wg::check_launch("launch column counts");
        });
  });
}

int wg_u8_count(int device, const uint8_t* flags, size_t rows, size_t cols, uint64_t* row_counts,
                uint64_t* col_counts, uint64_t* total, wg_stream_t stream) {
  return wg::guarded([&] {
    wg::DeviceGuard g(device);
    cudaStream_t s = stream;
    run_counts(
        device, rows, cols, row_counts, col_counts, total, s,
        [&](unsigned long long* tot) {
          u8_row_count_kernel<<<wg::grid_for(rows * 32, 256, device, 8), 256, 0, s>>>(flags, rows, cols, row_counts,
                                                                                     tot);
          wg::check_launch("launch row counts");
        },
        [&](unsigned long long* cc) {
          const size_t chunk = 4096;
          dim3 grid(static_cast<unsigned>((cols + 255) / 256), static_cast<unsigned>((rows + chunk - 1) / chunk));
          u8_col_count_kernel<<<grid, 256, 0, s>>>(flags, rows, cols, chunk, cc);
          wg::check_launch("launch column counts");
        });
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Commutation flags without any device allocation.
//
// Some callers cannot allocate device memory while they use this library: a
// host framework that owns the whole device budget and accounts for every byte
// itself, a caller that must not call cudaMalloc/cudaFree in a latency-critical
// loop (those calls synchronise the device), or a caller that has to keep its
// memory footprint fixed after start-up.  For them the bit-packed matrix that
// the ordinary path keeps in a caller or pool buffer lives here instead, in one
// static device array of kNoAllocScratchBytes.  Every GPU that loads this
// library holds that array until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;  // 32 MiB
static __device__ __align__(256) uint32_t g_noalloc_bits[kNoAllocScratchBytes / sizeof(uint32_t)];

namespace {

// Device address of g_noalloc_bits on `device`, resolved once per device with
// that device current.  (Host code cannot use the symbol's name as an address.)
uint32_t* noalloc_scratch(int device) {
  static std::mutex mu;
  static std::vector<uint32_t*> addr;
  std::lock_guard<std::mutex> lk(mu);
  if (addr.size() <= static_cast<size_t>(device)) addr.resize(device + 1, nullptr);
  if (!addr[device]) {
    void* p = nullptr;
    wg::check_cuda(cudaGetSymbolAddress(&p, g_noalloc_bits), "resolve the no-allocation scratch address");
    addr[device] = static_cast<uint32_t*>(p);
  }
  return addr[device];
}

}  // namespace

extern "C" int wg_commutation_u8_noalloc(int device, size_t words, const uint64_t* lhs_x, const uint64_t* lhs_z,
                                         size_t n_lhs, const uint64_t* rhs_x, const uint64_t* rhs_z, size_t n_rhs,
                                         uint8_t* out, wg_stream_t stream) {
  int status = wg::guarded([&] {
    if (n_lhs == 0 || n_rhs == 0) return;
    const size_t pitch = (n_rhs + 31) / 32;
    const size_t bytes = wg::checked_mul(wg::checked_mul(n_lhs, pitch, "commutation bit matrix"), 4,
                                         "commutation bit matrix");
    if (bytes > kNoAllocScratchBytes)
      wg::throw_invalid("commutation matrix too large for the no-allocation path: n_lhs * ceil(n_rhs/32) * 4 = " +
                        std::to_string(bytes) + " bytes exceeds the 32 MiB static scratch");
    wg::DeviceGuard g(device);
    uint32_t* bits = noalloc_scratch(device);
    // The ordinary path's kernels do the work; they allocate nothing
    // themselves.  The kernel choice reads no term data and never measures
    // (the autotuner's cached choice or the size rule), so a call after the
    // first synchronises nothing.
    commutation_bits(device, words, lhs_x, lhs_z, n_lhs, rhs_x, rhs_z, n_rhs, bits, pitch, 0, false, stream);
    const int rc = wg_bits_to_u8(device, bits, n_lhs, n_rhs, pitch, out, stream);
    if (rc != WG_OK) throw wg::Error(rc, wg_last_error());
  });
  return status;
}
