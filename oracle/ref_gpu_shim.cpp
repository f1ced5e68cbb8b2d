// ref_gpu_shim.cpp -- TEST AND BASELINE INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the reference's own CUDA path: the public
// wolfgang::DevicePauliSum / DeviceCommutationMatrix API of sghowell/wolfgang
// 0.2.3 (include/wolfgang/device_pauli_sum.hpp:93-175), compiled by
// oracle/Makefile (target refgpu) together with the reference's src/cuda/*.cu
// built for sm_100a and its CPU core into oracle/_ref/libwgref_cuda.so.
// bench.py --impl reference-gpu uses it to time the reference's kernels
// device-resident on the same GPU as this repository's: operands are uploaded
// once (DevicePauliSum::from_host), then every call goes through the
// reference's stock code path, which synchronises before it returns, and is
// timed by the host clock around the call.  Nothing of the reference is copied
// here: this file only converts plain buffers to and from its classes.
//
// It defines the same class names as this repository's C++ layer
// (libwolfgang.so), so it is never loaded into a process that uses that layer.

#include "wolfgang/device_commutation_matrix.hpp"
#include "wolfgang/device_pauli_sum.hpp"
#include "wolfgang/pauli_sum.hpp"

#include <cuda_runtime.h>

#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

wolfgang::PauliSum make_sum(size_t n, size_t T, size_t words, const uint64_t* x, const uint64_t* z,
                            const double* c) {
  std::vector<wolfgang::PauliSum::SparseTerm> terms(T);
  for (size_t t = 0; t < T; ++t) {
    auto& s = terms[t];
    s.coefficient = c ? std::complex<double>{c[2 * t], c[2 * t + 1]} : std::complex<double>{1.0, 0.0};
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

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
  } catch (...) {
    g_err = "unknown error";
  }
  return 1;
}

// Mean milliseconds of `reps` calls after `warmup` untimed ones.
template <class F>
double time_calls(int warmup, int reps, F&& call) {
  for (int i = 0; i < warmup; ++i) call();
  double total = 0.0;
  for (int i = 0; i < reps; ++i) {
    const auto t0 = std::chrono::steady_clock::now();
    call();
    total += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return reps > 0 ? total / reps : 0.0;
}

}  // namespace

extern "C" {

const char* wgrefgpu_last_error(void) { return g_err.c_str(); }

int wgrefgpu_available(int* available) {
  return guarded([&] { *available = wolfgang::DevicePauliSum::cuda_available() ? 1 : 0; });
}

// DevicePauliSum::matmul(rhs, simplify_output, max_intermediate_terms)
int wgrefgpu_matmul(size_t n, size_t nl, size_t nr, size_t words, const uint64_t* lx, const uint64_t* lz,
                    const double* lc, const uint64_t* rx, const uint64_t* rz, const double* rc, int simplify,
                    size_t max_intermediate, int warmup, int reps, double* ms, size_t* terms) {
  return guarded([&] {
    const auto l = wolfgang::DevicePauliSum::from_host(make_sum(n, nl, words, lx, lz, lc), 0);
    const auto r = wolfgang::DevicePauliSum::from_host(make_sum(n, nr, words, rx, rz, rc), 0);
    size_t u = 0;
    *ms = time_calls(warmup, reps, [&] { u = l.matmul(r, simplify != 0, max_intermediate).num_terms(); });
    *terms = u;
  });
}

// DevicePauliSum::simplify(atol, rtol)
int wgrefgpu_simplify(size_t n, size_t T, size_t words, const uint64_t* x, const uint64_t* z, const double* c,
                      double atol, double rtol, int warmup, int reps, double* ms, size_t* terms) {
  return guarded([&] {
    const auto d = wolfgang::DevicePauliSum::from_host(make_sum(n, T, words, x, z, c), 0);
    size_t u = 0;
    *ms = time_calls(warmup, reps, [&] { u = d.simplify(atol, rtol).num_terms(); });
    *terms = u;
  });
}

// DevicePauliSum::commutes_with_device_into a preallocated uint8 matrix (the
// reference's fastest device-resident commutation form); commuting = the
// matrix's count of commuting pairs after the last call.
int wgrefgpu_commutes_device(size_t n, size_t nl, size_t nr, size_t words, const uint64_t* lx, const uint64_t* lz,
                             const uint64_t* rx, const uint64_t* rz, size_t max_entries, int warmup, int reps,
                             double* ms, uint64_t* commuting) {
  return guarded([&] {
    const auto l = wolfgang::DevicePauliSum::from_host(make_sum(n, nl, words, lx, lz, nullptr), 0);
    const auto r = wolfgang::DevicePauliSum::from_host(make_sum(n, nr, words, rx, rz, nullptr), 0);
    auto out = wolfgang::DeviceCommutationMatrix::empty(nl, nr, 0);
    *ms = time_calls(warmup, reps, [&] { l.commutes_with_device_into(r, out, max_entries); });
    *commuting = out.count_commuting();
  });
}

// DevicePauliSum::expectation_statevector_device_pointer on a complex128
// statevector uploaded once (cudaMalloc + one copy, outside the timing).
int wgrefgpu_expectation(size_t n, size_t T, size_t words, const uint64_t* x, const uint64_t* z, const double* c,
                         const double* psi, int warmup, int reps, double* ms, double* out) {
  return guarded([&] {
    const auto d = wolfgang::DevicePauliSum::from_host(make_sum(n, T, words, x, z, c), 0);
    const size_t N = size_t{1} << n;
    void* dpsi = nullptr;
    if (cudaMalloc(&dpsi, N * 16) != cudaSuccess) throw std::runtime_error("cudaMalloc statevector failed");
    try {
      if (cudaMemcpy(dpsi, psi, N * 16, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("statevector upload failed");
      std::complex<double> v;
      *ms = time_calls(warmup, reps, [&] {
        v = d.expectation_statevector_device_pointer(reinterpret_cast<std::uintptr_t>(dpsi),
                                                     wolfgang::DeviceStatevectorDtype::Complex128, N);
      });
      out[0] = v.real();
      out[1] = v.imag();
    } catch (...) {
      (void)cudaFree(dpsi);
      throw;
    }
    (void)cudaFree(dpsi);
  });
}

}  // extern "C"
