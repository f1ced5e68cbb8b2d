// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the reference's own public C++ API
// (include/wolfgang/pauli_sum.hpp of sghowell/wolfgang 0.2.3).  oracle/Makefile
// compiles it together with the reference's CPU sources, read in place from the
// reference checkout, into oracle/_ref/libwgref.so.  Tests use it to pin the
// scalar oracle (oracle.cpp) and bench.py uses it as the timed CPU baseline
// ("cpu_baseline.kind": "reference").  Nothing of the reference is copied here:
// this file only converts plain buffers to and from wolfgang::PauliSum.
//
// Argument layout matches oracle.h: x/z packed words, interleaved (re, im).

#include "wolfgang/pauli_sum.hpp"
#include "wolfgang/cpu_backend.hpp"

#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

// The packed constructor is private, so build operators from sparse terms:
// bit q of x/z word q/64 becomes local Pauli letter on qubit q.
wolfgang::PauliSum make_sum(size_t n, size_t T, size_t words, const uint64_t* x,
                            const uint64_t* z, const double* c) {
  std::vector<wolfgang::PauliSum::SparseTerm> terms(T);
  for (size_t t = 0; t < T; ++t) {
    auto& s = terms[t];
    s.coefficient = {c[2 * t], c[2 * t + 1]};
    for (size_t q = 0; q < n; ++q) {
      const bool xb = (x[t * words + q / 64] >> (q % 64)) & 1U;
      const bool zb = (z[t * words + q / 64] >> (q % 64)) & 1U;
      if (!xb && !zb) continue;
      s.local_pauli_string.push_back(xb && zb ? 'Y' : (xb ? 'X' : 'Z'));
      s.qubit_indices.push_back(q);
    }
  }
  return wolfgang::PauliSum::from_sparse_list(terms, n);
}

void export_sum(const wolfgang::PauliSum& p, uint64_t* ox, uint64_t* oz, double* oc,
                size_t* out_terms) {
  const auto& x = p.x_words();
  const auto& z = p.z_words();
  const auto& c = p.coeffs();
  if (!x.empty()) std::memcpy(ox, x.data(), x.size() * sizeof(uint64_t));
  if (!z.empty()) std::memcpy(oz, z.data(), z.size() * sizeof(uint64_t));
  for (size_t i = 0; i < c.size(); ++i) {
    oc[2 * i] = c[i].real();
    oc[2 * i + 1] = c[i].imag();
  }
  *out_terms = p.num_terms();
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

}  // namespace

extern "C" {

const char* wgref_last_error(void) { return g_err.c_str(); }

int wgref_simplify(size_t n, size_t T, size_t words, const uint64_t* x,
                   const uint64_t* z, const double* c, double atol, double rtol,
                   uint64_t* ox, uint64_t* oz, double* oc, size_t* out_terms) {
  return guarded([&] {
    export_sum(make_sum(n, T, words, x, z, c).simplify(atol, rtol), ox, oz, oc, out_terms);
  });
}

int wgref_matmul(size_t n, size_t nl, size_t nr, size_t words, const uint64_t* lx,
                 const uint64_t* lz, const double* lc, const uint64_t* rx,
                 const uint64_t* rz, const double* rc, int simplify,
                 size_t max_intermediate, uint64_t* ox, uint64_t* oz, double* oc,
                 size_t* out_terms) {
  return guarded([&] {
    const auto l = make_sum(n, nl, words, lx, lz, lc);
    const auto r = make_sum(n, nr, words, rx, rz, rc);
    export_sum(l.matmul(r, simplify != 0, max_intermediate), ox, oz, oc, out_terms);
  });
}

int wgref_commutes(size_t n, size_t nl, size_t nr, size_t words, const uint64_t* lx,
                   const uint64_t* lz, const uint64_t* rx, const uint64_t* rz,
                   size_t max_entries, uint8_t* out) {
  return guarded([&] {
    const std::vector<double> lc(2 * nl, 1.0), rc(2 * nr, 1.0);
    const auto l = make_sum(n, nl, words, lx, lz, lc.data());
    const auto r = make_sum(n, nr, words, rx, rz, rc.data());
    const auto flags = l.commutes_with(r, max_entries);
    if (!flags.empty()) std::memcpy(out, flags.data(), flags.size());
  });
}

int wgref_group_commuting(size_t n, size_t T, size_t words, const uint64_t* x,
                          const uint64_t* z, const double* c, int mode_full,
                          size_t max_terms_for_graph, uint64_t* ox, uint64_t* oz,
                          double* oc, size_t* sizes_out, size_t* n_groups) {
  return guarded([&] {
    const auto op = make_sum(n, T, words, x, z, c);
    const auto groups = op.group_commuting(mode_full ? "full" : "qwc", "largest_first",
                                           max_terms_for_graph);
    size_t off = 0;
    for (size_t g = 0; g < groups.size(); ++g) {
      size_t m = 0;
      export_sum(groups[g], ox + off * words, oz + off * words, oc + 2 * off, &m);
      sizes_out[g] = m;
      off += m;
    }
    *n_groups = groups.size();
  });
}

int wgref_expectation(size_t n, size_t T, size_t words, const uint64_t* x,
                      const uint64_t* z, const double* c, const void* psi, int dtype,
                      double* out) {
  return guarded([&] {
    const auto op = make_sum(n, T, words, x, z, c);
    const size_t N = size_t{1} << n;
    std::complex<double> r;
    if (dtype == 0)
      r = op.expectation_statevector_complex128(
          std::span<const std::complex<double>>(static_cast<const std::complex<double>*>(psi), N));
    else
      r = op.expectation_statevector_complex64(
          std::span<const std::complex<float>>(static_cast<const std::complex<float>*>(psi), N));
    out[0] = r.real();
    out[1] = r.imag();
  });
}

// PauliSum::expectation_z_counts with the bitstrings given packed (row-major,
// `words` words per row, qubit q = bit q%64 of word q/64); they are written
// back out as the reference's strings, whose first character is qubit n-1.
int wgref_expectation_z_counts(size_t n, size_t T, size_t words, const uint64_t* x,
                               const uint64_t* z, const double* c, size_t rows,
                               const uint64_t* packed, const double* counts, double* out) {
  return guarded([&] {
    const auto op = make_sum(n, T, words, x, z, c);
    std::vector<std::string> bitstrings(rows, std::string(n, '0'));
    for (size_t r = 0; r < rows; ++r)
      for (size_t q = 0; q < n; ++q)
        if ((packed[r * words + q / 64] >> (q % 64)) & 1U) bitstrings[r][n - 1 - q] = '1';
    const std::vector<double> cnt(counts, counts + rows);
    const std::complex<double> v = op.expectation_z_counts(bitstrings, cnt);
    out[0] = v.real();
    out[1] = v.imag();
  });
}

// Reports the CPU dispatch the reference would use for commutes_with in this
// process: the active backend and the candidates' availability.
int wgref_cpu_backend(char* buf, size_t cap) {
  return guarded([&] {
    const auto rep = wolfgang::cpu_backend_report_from_environment();
    std::string s = "requested=" + rep.requested_backend + ";active=" + rep.active_backend + ";";
    for (const auto& cand : rep.candidates) s += cand.name + ":" + cand.status + ",";
    std::strncpy(buf, s.c_str(), cap - 1);
    buf[cap - 1] = 0;
  });
}

}  // extern "C"
