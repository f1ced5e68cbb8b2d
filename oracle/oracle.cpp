// oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A scalar restatement of the CPU semantics of sghowell/wolfgang 0.2.3 for the
// packed-Pauli hot path.  It is written from the reference's documented
// behaviour; each function names the reference lines it follows.  It is built
// with -O2 -ffp-contract=off and no -march flag, the same floating-point
// environment as the reference (CMakeLists.txt:77-79 forbids -march=native), so
// std::complex products and sums round exactly as the reference's do.
//
// Parity pin: tests/test_oracle_vs_reference.py checks every function here
// bit-for-bit against the reference's own C++ core compiled from its sources
// (oracle/Makefile -> oracle/_ref/libwgref.so) and against the golden vectors
// under tests/golden/.

#include "oracle.h"

#include <algorithm>
#include <bit>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

using cplx = std::complex<double>;
thread_local std::string g_err;

int fail(const char* msg) {
  g_err = msg;
  return 1;
}

cplx load_c(const double* c, size_t i) { return {c[2 * i], c[2 * i + 1]}; }
void store_c(double* c, size_t i, cplx v) {
  c[2 * i] = v.real();
  c[2 * i + 1] = v.imag();
}

// Canonical order: word 0 first, x before z inside a word, each word compared
// as unsigned 64-bit (src/detail/packed_key.hpp:86-133).
int compare_keys(const uint64_t* ax, const uint64_t* az, const uint64_t* bx,
                 const uint64_t* bz, size_t words) {
  for (size_t w = 0; w < words; ++w) {
    if (ax[w] != bx[w]) return ax[w] < bx[w] ? -1 : 1;
    if (az[w] != bz[w]) return az[w] < bz[w] ? -1 : 1;
  }
  return 0;
}

// i^e rotation (src/detail/phase.hpp:22-36); exact sign swaps.
cplx rotate(cplx v, int64_t e) {
  switch (static_cast<uint64_t>(e) & 3U) {
    case 0: return v;
    case 1: return {-v.imag(), v.real()};
    case 2: return {-v.real(), -v.imag()};
    default: return {v.imag(), -v.real()};
  }
}

// Keys of one product term (x/z words) plus its coefficient.
struct ProductSet {
  size_t words;
  std::vector<uint64_t> x, z;
  std::vector<cplx> c;
};

// Nested-loop product generation: lhs outer, rhs inner; rhs acts first
// (src/multiply.cpp:89-105 for the Y parities, :263-389 for the products).
void products(size_t nl, size_t nr, size_t w, const uint64_t* lx,
              const uint64_t* lz, const double* lc, const uint64_t* rx,
              const uint64_t* rz, const double* rc, ProductSet& out) {
  out.words = w;
  out.x.assign(nl * nr * w, 0);
  out.z.assign(nl * nr * w, 0);
  out.c.assign(nl * nr, cplx{});
  std::vector<int64_t> ly(nl, 0), ry(nr, 0);
  for (size_t a = 0; a < nl; ++a)
    for (size_t k = 0; k < w; ++k) ly[a] += std::popcount(lx[a * w + k] & lz[a * w + k]);
  for (size_t b = 0; b < nr; ++b)
    for (size_t k = 0; k < w; ++k) ry[b] += std::popcount(rx[b * w + k] & rz[b * w + k]);
  size_t o = 0;
  for (size_t a = 0; a < nl; ++a) {
    const cplx ca = load_c(lc, a);
    for (size_t b = 0; b < nr; ++b, ++o) {
      int64_t e = -ly[a] - ry[b];
      for (size_t k = 0; k < w; ++k) {
        const uint64_t ox = lx[a * w + k] ^ rx[b * w + k];
        const uint64_t oz = lz[a * w + k] ^ rz[b * w + k];
        out.x[o * w + k] = ox;
        out.z[o * w + k] = oz;
        e += std::popcount(ox & oz);
        e += 2 * static_cast<int64_t>(std::popcount(lx[a * w + k] & rz[b * w + k]));
      }
      out.c[o] = rotate(ca * load_c(rc, b), e);
    }
  }
}

// Sort-reduce-cull: stable order by (key, input index); each equal-key run is
// summed left to right starting from 0 (src/simplify.cpp:215-262, :375-416;
// the hash paths :163-213, :266-319 sum in the same input order and differ only
// in the sign of an exact zero, which the cull drops).  Keeps |sum| > thr.
void reduce_sorted(size_t T, size_t w, const uint64_t* x, const uint64_t* z,
                   const cplx* c, double thr, uint64_t* ox, uint64_t* oz,
                   double* oc, size_t* out_terms) {
  std::vector<size_t> idx(T);
  std::iota(idx.begin(), idx.end(), size_t{0});
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    return compare_keys(x + a * w, z + a * w, x + b * w, z + b * w, w) < 0;
  });
  size_t u = 0;
  size_t p = 0;
  while (p < T) {
    const size_t first = idx[p];
    cplx acc{0.0, 0.0};
    size_t q = p;
    while (q < T && compare_keys(x + first * w, z + first * w, x + idx[q] * w,
                                 z + idx[q] * w, w) == 0) {
      acc += c[idx[q]];
      ++q;
    }
    if (std::abs(acc) > thr) {
      for (size_t k = 0; k < w; ++k) {
        ox[u * w + k] = x[first * w + k];
        oz[u * w + k] = z[first * w + k];
      }
      store_c(oc, u, acc);
      ++u;
    }
    p = q;
  }
  *out_terms = u;
}

bool tolerances_ok(double atol, double rtol) {
  // src/simplify.cpp:148-150
  return !(atol < 0.0 || rtol < 0.0 || !std::isfinite(atol) || !std::isfinite(rtol));
}

// Duplicate-heavy sample used by matmul's fused path (src/multiply.cpp:29-69):
// at least 128 terms and >= 25 % duplicates among the first min(T, 512) keys.
bool operand_duplicate_heavy(size_t T, size_t w, const uint64_t* x, const uint64_t* z) {
  if (T < 128) return false;
  const size_t s = std::min<size_t>(T, 512);
  std::vector<size_t> idx(s);
  std::iota(idx.begin(), idx.end(), size_t{0});
  std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    return compare_keys(x + a * w, z + a * w, x + b * w, z + b * w, w) < 0;
  });
  size_t unique = s == 0 ? 0 : 1;
  for (size_t i = 1; i < s; ++i)
    if (compare_keys(x + idx[i - 1] * w, z + idx[i - 1] * w, x + idx[i] * w,
                     z + idx[i] * w, w) != 0)
      ++unique;
  const double rate = 1.0 - static_cast<double>(unique) / static_cast<double>(s);
  return rate >= 0.25;
}

bool fused_path(size_t nl, size_t nr, size_t w, const uint64_t* lx,
                const uint64_t* lz, const uint64_t* rx, const uint64_t* rz,
                int simplify) {
  // src/multiply.cpp:107-109 (words == 1) and :179-181 (words == 2).
  if (!simplify || (w != 1 && w != 2)) return false;
  return operand_duplicate_heavy(nl, w, lx, lz) || operand_duplicate_heavy(nr, w, rx, rz);
}

template <typename C>
cplx widen(const C& v) {
  return static_cast<cplx>(v);
}

}  // namespace

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

double or_abs(double re, double im) { return std::abs(cplx{re, im}); }

int or_simplify(size_t T, size_t words, const uint64_t* x, const uint64_t* z,
                const double* c, double atol, double rtol, uint64_t* ox,
                uint64_t* oz, double* oc, size_t* out_terms) {
  if (!tolerances_ok(atol, rtol))
    return fail("simplify tolerances must be non-negative finite values");
  *out_terms = 0;
  if (T == 0) return 0;  // src/simplify.cpp:152-154
  std::vector<cplx> cc(T);
  double max_abs = 0.0;  // src/simplify.cpp:156-160
  for (size_t i = 0; i < T; ++i) {
    cc[i] = load_c(c, i);
    max_abs = std::max(max_abs, std::abs(cc[i]));
  }
  const double thr = atol + rtol * max_abs;
  reduce_sorted(T, words, x, z, cc.data(), thr, ox, oz, oc, out_terms);
  return 0;
}

int or_matmul_uses_fused_path(size_t nl, size_t nr, size_t words,
                              const uint64_t* lx, const uint64_t* lz,
                              const uint64_t* rx, const uint64_t* rz,
                              int simplify) {
  return fused_path(nl, nr, words, lx, lz, rx, rz, simplify) ? 1 : 0;
}

int or_matmul(size_t nl, size_t nr, size_t words, const uint64_t* lx,
              const uint64_t* lz, const double* lc, const uint64_t* rx,
              const uint64_t* rz, const double* rc, int simplify,
              uint64_t* ox, uint64_t* oz, double* oc, size_t* out_terms) {
  *out_terms = 0;
  const size_t P = nl * nr;
  if (P == 0) return 0;  // src/multiply.cpp:85-87
  ProductSet ps;
  products(nl, nr, words, lx, lz, lc, rx, rz, rc, ps);
  if (!simplify) {
    std::memcpy(ox, ps.x.data(), ps.x.size() * sizeof(uint64_t));
    std::memcpy(oz, ps.z.data(), ps.z.size() * sizeof(uint64_t));
    for (size_t i = 0; i < P; ++i) store_c(oc, i, ps.c[i]);
    *out_terms = P;
    return 0;
  }
  double thr;
  if (fused_path(nl, nr, words, lx, lz, rx, rz, simplify)) {
    thr = 1.0e-12;  // hard-coded cull of the fused path, src/multiply.cpp:144, :226
  } else {
    double max_abs = 0.0;  // simplify() at its defaults atol=1e-12, rtol=0
    for (size_t i = 0; i < P; ++i) max_abs = std::max(max_abs, std::abs(ps.c[i]));
    thr = 1.0e-12 + 0.0 * max_abs;
  }
  reduce_sorted(P, words, ps.x.data(), ps.z.data(), ps.c.data(), thr, ox, oz, oc, out_terms);
  return 0;
}

int or_matmul_keyrange(size_t nl, size_t nr, size_t words, const uint64_t* lx,
                       const uint64_t* lz, const double* lc, const uint64_t* rx,
                       const uint64_t* rz, const double* rc,
                       const uint64_t* key_lo, const uint64_t* key_hi,
                       int fused_threshold, size_t cap, uint64_t* ox,
                       uint64_t* oz, double* oc, size_t* out_terms) {
  // Same products and order as or_matmul, but only keys in [key_lo, key_hi)
  // are kept, so a full-size product set can be checked slice by slice.
  const size_t w = words;
  std::vector<uint64_t> klo_x(w), klo_z(w), khi_x(w), khi_z(w);
  for (size_t k = 0; k < w; ++k) {
    klo_x[k] = key_lo[2 * k];
    klo_z[k] = key_lo[2 * k + 1];
    khi_x[k] = key_hi[2 * k];
    khi_z[k] = key_hi[2 * k + 1];
  }
  std::vector<int64_t> ly(nl, 0), ry(nr, 0);
  for (size_t a = 0; a < nl; ++a)
    for (size_t k = 0; k < w; ++k) ly[a] += std::popcount(lx[a * w + k] & lz[a * w + k]);
  for (size_t b = 0; b < nr; ++b)
    for (size_t k = 0; k < w; ++k) ry[b] += std::popcount(rx[b * w + k] & rz[b * w + k]);
  std::vector<uint64_t> sx, sz;
  std::vector<cplx> sc;
  std::vector<uint64_t> px(w), pz(w);
  // The threshold atol + 0 * max|product| (src/simplify.cpp:156-160) is atol
  // unless some product's magnitude is infinite (0 * inf = NaN culls all).
  // When every input coefficient is finite and max|a| * max|b| is far below
  // the overflow limit, no product can be infinite, and the magnitudes of the
  // products outside the range need not be formed; otherwise every product's
  // magnitude enters the maximum, as in or_matmul.
  double amax = 0.0, bmax = 0.0;
  bool finite = true;
  for (size_t a = 0; a < nl; ++a) {
    const cplx v = load_c(lc, a);
    finite = finite && std::isfinite(v.real()) && std::isfinite(v.imag());
    amax = std::max(amax, std::abs(v));
  }
  for (size_t b = 0; b < nr; ++b) {
    const cplx v = load_c(rc, b);
    finite = finite && std::isfinite(v.real()) && std::isfinite(v.imag());
    bmax = std::max(bmax, std::abs(v));
  }
  const bool need_max = !fused_threshold && !(finite && amax < 1e150 && bmax < 1e150);
  double max_abs = 0.0;
  for (size_t a = 0; a < nl; ++a) {
    const cplx ca = load_c(lc, a);
    for (size_t b = 0; b < nr; ++b) {
      for (size_t k = 0; k < w; ++k) {
        px[k] = lx[a * w + k] ^ rx[b * w + k];
        pz[k] = lz[a * w + k] ^ rz[b * w + k];
      }
      const bool in_range = compare_keys(px.data(), pz.data(), klo_x.data(), klo_z.data(), w) >= 0 &&
                            compare_keys(px.data(), pz.data(), khi_x.data(), khi_z.data(), w) < 0;
      if (!in_range && !need_max) continue;
      int64_t e = -ly[a] - ry[b];
      for (size_t k = 0; k < w; ++k) {
        e += std::popcount(px[k] & pz[k]);
        e += 2 * static_cast<int64_t>(std::popcount(lx[a * w + k] & rz[b * w + k]));
      }
      const cplx v = rotate(ca * load_c(rc, b), e);
      if (need_max) max_abs = std::max(max_abs, std::abs(v));
      if (!in_range) continue;
      sx.insert(sx.end(), px.begin(), px.end());
      sz.insert(sz.end(), pz.begin(), pz.end());
      sc.push_back(v);
    }
  }
  const double thr = fused_threshold ? 1.0e-12 : 1.0e-12 + 0.0 * max_abs;
  const size_t S = sc.size();
  // reduce into scratch sized for every in-range product, then hand over the
  // survivors: cap only bounds the result
  std::vector<uint64_t> tx(S * w + 1), tz(S * w + 1);
  std::vector<double> tc(2 * S + 2);
  size_t u = 0;
  reduce_sorted(S, w, sx.data(), sz.data(), sc.data(), thr, tx.data(), tz.data(), tc.data(), &u);
  if (u > cap) return fail("or_matmul_keyrange capacity too small");
  std::copy(tx.begin(), tx.begin() + static_cast<std::ptrdiff_t>(u * w), ox);
  std::copy(tz.begin(), tz.begin() + static_cast<std::ptrdiff_t>(u * w), oz);
  std::copy(tc.begin(), tc.begin() + static_cast<std::ptrdiff_t>(2 * u), oc);
  *out_terms = u;
  return 0;
}

int or_commutes(size_t nl, size_t nr, size_t words, const uint64_t* lx,
                const uint64_t* lz, const uint64_t* rx, const uint64_t* rz,
                uint8_t* out) {
  for (size_t a = 0; a < nl; ++a) {
    for (size_t b = 0; b < nr; ++b) {
      unsigned odd = 0;
      for (size_t k = 0; k < words; ++k) {
        const uint64_t conflicts =
            (lx[a * words + k] & rz[b * words + k]) ^ (lz[a * words + k] & rx[b * words + k]);
        odd ^= static_cast<unsigned>(std::popcount(conflicts)) & 1U;
      }
      out[a * nr + b] = odd == 0 ? 1 : 0;
    }
  }
  return 0;
}

int or_group_commuting(size_t T, size_t words, const uint64_t* x,
                       const uint64_t* z, int mode_full, size_t* order_out,
                       size_t* sizes_out, size_t* n_groups) {
  *n_groups = 0;
  if (T == 0) return 0;
  const size_t w = words;
  // Deterministic order: weight descending, canonical key, index
  // (src/grouping.cpp:36-62; weight = popcount(x|z), src/detail/bitops.hpp:36-46).
  std::vector<size_t> weight(T, 0);
  for (size_t t = 0; t < T; ++t)
    for (size_t k = 0; k < w; ++k) weight[t] += std::popcount(x[t * w + k] | z[t * w + k]);
  std::vector<size_t> order(T);
  std::iota(order.begin(), order.end(), size_t{0});
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    if (weight[a] != weight[b]) return weight[a] > weight[b];
    const int cmp = compare_keys(x + a * w, z + a * w, x + b * w, z + b * w, w);
    if (cmp != 0) return cmp < 0;
    return a < b;
  });
  std::vector<std::vector<size_t>> groups;
  if (!mode_full) {
    // qwc: first group whose OR-basis has no conflict (src/grouping.cpp:64-84, :214-237).
    std::vector<std::vector<uint64_t>> bx, bz;
    for (size_t t : order) {
      bool placed = false;
      for (size_t g = 0; g < groups.size() && !placed; ++g) {
        bool ok = true;
        for (size_t k = 0; k < w && ok; ++k)
          ok = ((x[t * w + k] & bz[g][k]) ^ (z[t * w + k] & bx[g][k])) == 0;
        if (ok) {
          for (size_t k = 0; k < w; ++k) {
            bx[g][k] |= x[t * w + k];
            bz[g][k] |= z[t * w + k];
          }
          groups[g].push_back(t);
          placed = true;
        }
      }
      if (!placed) {
        groups.push_back({t});
        bx.emplace_back(x + t * w, x + t * w + w);
        bz.emplace_back(z + t * w, z + t * w + w);
      }
    }
  } else {
    // full: first group all of whose members commute with t
    // (src/grouping.cpp:96-126, :238-260; the precomputed graph and the
    // streaming check give the same answers).
    for (size_t t : order) {
      bool placed = false;
      for (auto& g : groups) {
        bool ok = true;
        for (size_t m : g) {
          unsigned odd = 0;
          for (size_t k = 0; k < w; ++k)
            odd ^= std::popcount((x[t * w + k] & z[m * w + k]) ^ (z[t * w + k] & x[m * w + k])) & 1U;
          if (odd) {
            ok = false;
            break;
          }
        }
        if (ok) {
          g.push_back(t);
          placed = true;
          break;
        }
      }
      if (!placed) groups.push_back({t});
    }
  }
  size_t p = 0;
  for (size_t g = 0; g < groups.size(); ++g) {
    sizes_out[g] = groups[g].size();
    for (size_t t : groups[g]) order_out[p++] = t;
  }
  *n_groups = groups.size();
  return 0;
}

}  // extern "C"

namespace {

template <typename C>
int expectation_impl(size_t T, size_t n, const uint64_t* x, const uint64_t* z,
                     const double* c, const C* psi, double* out) {
  // src/expectation.cpp:37-155
  const size_t words = n == 0 ? 0 : (n + 63) / 64;
  if (n > 63) return fail("expectation_statevector requires num_qubits <= 63");
  const size_t N = size_t{1} << n;
  out[0] = out[1] = 0.0;
  if (T == 0) return 0;
  bool diagonal = true;
  for (size_t i = 0; i < T * words; ++i)
    if (x[i] != 0) {
      diagonal = false;
      break;
    }
  cplx result{0.0, 0.0};
  if (diagonal) {
    std::vector<double> prob(N);
    for (size_t b = 0; b < N; ++b) prob[b] = std::norm(widen(psi[b]));
    if (T >= 64) {
      // Coefficients summed per distinct z mask in first-seen order (:66-99).
      std::unordered_map<uint64_t, size_t> slot;
      std::vector<uint64_t> masks;
      std::vector<cplx> sums;
      for (size_t t = 0; t < T; ++t) {
        const uint64_t zm = words == 0 ? 0 : z[t * words];
        auto it = slot.find(zm);
        if (it == slot.end()) {
          slot.emplace(zm, masks.size());
          masks.push_back(zm);
          sums.push_back(load_c(c, t));
        } else {
          sums[it->second] += load_c(c, t);
        }
      }
      for (size_t m = 0; m < masks.size(); ++m) {
        double e = 0.0;
        for (size_t b = 0; b < N; ++b)
          e += (std::popcount(masks[m] & static_cast<uint64_t>(b)) & 1U) ? -prob[b] : prob[b];
        result += sums[m] * e;
      }
    } else {
      for (size_t t = 0; t < T; ++t) {
        const uint64_t zm = words == 0 ? 0 : z[t * words];
        double e = 0.0;
        for (size_t b = 0; b < N; ++b)
          e += (std::popcount(zm & static_cast<uint64_t>(b)) & 1U) ? -prob[b] : prob[b];
        result += load_c(c, t) * e;
      }
    }
    out[0] = result.real();
    out[1] = result.imag();
    return 0;
  }
  for (size_t t = 0; t < T; ++t) {
    const uint64_t xm = words == 0 ? 0 : x[t * words];
    const uint64_t zm = words == 0 ? 0 : z[t * words];
    const cplx yz = rotate(cplx{1.0, 0.0}, std::popcount(xm & zm));
    double e = 0.0;
    if (xm == 0) {
      for (size_t b = 0; b < N; ++b) {
        const double p = std::norm(widen(psi[b]));
        e += (std::popcount(zm & static_cast<uint64_t>(b)) & 1U) ? -p : p;
      }
    } else {
      const uint64_t pivot = xm & (0 - xm);
      for (size_t b = 0; b < N; ++b) {
        if (static_cast<uint64_t>(b) & pivot) continue;
        const size_t tg = b ^ static_cast<size_t>(xm);
        const cplx ph = (std::popcount(zm & static_cast<uint64_t>(b)) & 1U) ? -yz : yz;
        const cplx amp = std::conj(widen(psi[tg])) * widen(psi[b]);
        e += 2.0 * (ph * amp).real();
      }
    }
    result += load_c(c, t) * e;
  }
  out[0] = result.real();
  out[1] = result.imag();
  return 0;
}

// Neumaier-compensated running sum.
struct KSum {
  double s = 0.0, comp = 0.0;
  void add(double v) {
    const double t = s + v;
    if (std::fabs(s) >= std::fabs(v))
      comp += (s - t) + v;
    else
      comp += (v - t) + s;
    s = t;
  }
  double value() const { return s + comp; }
};

template <typename C>
int term_expectations_impl(size_t T, size_t n, const uint64_t* x, const uint64_t* z,
                           const C* psi, double* out) {
  if (n > 63) return fail("expectation_statevector requires num_qubits <= 63");
  const size_t words = n == 0 ? 0 : 1;
  const size_t N = size_t{1} << n;
  for (size_t t = 0; t < T; ++t) {
    const uint64_t xm = words == 0 ? 0 : x[t * words];
    const uint64_t zm = words == 0 ? 0 : z[t * words];
    const cplx yz = rotate(cplx{1.0, 0.0}, std::popcount(xm & zm));
    KSum e;
    if (xm == 0) {
      for (size_t b = 0; b < N; ++b) {
        const double p = std::norm(widen(psi[b]));
        e.add((std::popcount(zm & static_cast<uint64_t>(b)) & 1U) ? -p : p);
      }
    } else {
      const uint64_t pivot = xm & (0 - xm);
      for (size_t b = 0; b < N; ++b) {
        if (static_cast<uint64_t>(b) & pivot) continue;
        const size_t tg = b ^ static_cast<size_t>(xm);
        const cplx ph = (std::popcount(zm & static_cast<uint64_t>(b)) & 1U) ? -yz : yz;
        const cplx amp = std::conj(widen(psi[tg])) * widen(psi[b]);
        e.add(2.0 * (ph * amp).real());
      }
    }
    out[t] = e.value();
  }
  return 0;
}

}  // namespace

extern "C" {

int or_expectation(size_t T, size_t n_qubits, const uint64_t* x,
                   const uint64_t* z, const double* c, const void* psi,
                   int dtype, double* out) {
  if (dtype == 0)
    return expectation_impl(T, n_qubits, x, z, c, static_cast<const std::complex<double>*>(psi), out);
  return expectation_impl(T, n_qubits, x, z, c, static_cast<const std::complex<float>*>(psi), out);
}

int or_term_expectations(size_t T, size_t n_qubits, const uint64_t* x,
                         const uint64_t* z, const void* psi, int dtype,
                         double* out) {
  if (dtype == 0)
    return term_expectations_impl(T, n_qubits, x, z, static_cast<const std::complex<double>*>(psi), out);
  return term_expectations_impl(T, n_qubits, x, z, static_cast<const std::complex<float>*>(psi), out);
}

int or_hpsi(size_t T, size_t n_qubits, const uint64_t* x, const uint64_t* z,
            const double* c, const double* psi, double* out) {
  if (n_qubits > 63) return fail("expectation_statevector requires num_qubits <= 63");
  const size_t words = n_qubits == 0 ? 0 : 1;
  const size_t N = size_t{1} << n_qubits;
  std::vector<KSum> re(N), im(N);
  for (size_t t = 0; t < T; ++t) {
    const uint64_t xm = words == 0 ? 0 : x[t * words];
    const uint64_t zm = words == 0 ? 0 : z[t * words];
    const cplx d = rotate(load_c(c, t), std::popcount(xm & zm));
    for (size_t j = 0; j < N; ++j) {
      const size_t src = j ^ static_cast<size_t>(xm);
      const cplx v = d * load_c(psi, src);
      const bool neg = std::popcount(zm & static_cast<uint64_t>(src)) & 1U;
      re[j].add(neg ? -v.real() : v.real());
      im[j].add(neg ? -v.imag() : v.imag());
    }
  }
  for (size_t j = 0; j < N; ++j) {
    out[2 * j] = re[j].value();
    out[2 * j + 1] = im[j].value();
  }
  return 0;
}

int or_hpsi_at(size_t T, size_t n_qubits, const uint64_t* x, const uint64_t* z,
               const double* c, const double* psi, size_t m, const uint64_t* idx,
               double* out) {
  // or_hpsi's sum, term by term in the same order, evaluated at the m
  // requested amplitudes only.
  if (n_qubits > 63) return fail("expectation_statevector requires num_qubits <= 63");
  const size_t words = n_qubits == 0 ? 0 : 1;
  const size_t N = size_t{1} << n_qubits;
  for (size_t i = 0; i < m; ++i)
    if (idx[i] >= N) return fail("or_hpsi_at index is out of range");
  std::vector<KSum> re(m), im(m);
  for (size_t t = 0; t < T; ++t) {
    const uint64_t xm = words == 0 ? 0 : x[t * words];
    const uint64_t zm = words == 0 ? 0 : z[t * words];
    const cplx d = rotate(load_c(c, t), std::popcount(xm & zm));
    for (size_t i = 0; i < m; ++i) {
      const size_t src = static_cast<size_t>(idx[i]) ^ static_cast<size_t>(xm);
      const cplx v = d * load_c(psi, src);
      const bool neg = std::popcount(zm & static_cast<uint64_t>(src)) & 1U;
      re[i].add(neg ? -v.real() : v.real());
      im[i].add(neg ? -v.imag() : v.imag());
    }
  }
  for (size_t i = 0; i < m; ++i) {
    out[2 * i] = re[i].value();
    out[2 * i + 1] = im[i].value();
  }
  return 0;
}

int or_expectation_z_counts(size_t T, size_t words, const uint64_t* x,
                            const uint64_t* z, const double* c, size_t rows,
                            const uint64_t* packed, const double* counts,
                            double* out) {
  // src/expectation.cpp:157-247 (validation, then per-term weighted parity sum).
  for (size_t i = 0; i < T * words; ++i)
    if (x[i] != 0) return fail("expectation_z_counts requires diagonal Pauli terms");
  double total = 0.0;
  for (size_t r = 0; r < rows; ++r) {
    if (counts[r] < 0.0) return fail("Z-count values must be non-negative");
    if (!std::isfinite(counts[r])) return fail("Z-count values must be finite");
    total += counts[r];
  }
  if (total <= 0.0) return fail("Z-count total count must be positive");
  cplx result{0.0, 0.0};
  for (size_t t = 0; t < T; ++t) {
    double weighted = 0.0;
    for (size_t r = 0; r < rows; ++r) {
      bool odd = false;
      for (size_t k = 0; k < words; ++k)
        odd ^= (std::popcount(z[t * words + k] & packed[r * words + k]) & 1U) != 0;
      weighted += counts[r] * (odd ? -1.0 : 1.0);
    }
    result += load_c(c, t) * (weighted / total);
  }
  out[0] = result.real();
  out[1] = result.imag();
  return 0;
}

}  // extern "C"
