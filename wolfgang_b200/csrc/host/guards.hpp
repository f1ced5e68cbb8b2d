#pragma once
// Size guardrails with the reference's messages (src/detail/checked_arithmetic.hpp
// :10-63, src/detail/accelerator_host_helpers.hpp:11-80).  They run before any
// device allocation, so oversized requests fail without touching the GPU.

#include <cstddef>
#include <limits>
#include <stdexcept>
#include <string>

namespace wolfgang::guards {

inline std::size_t word_count(std::size_t num_qubits) {
  if (num_qubits == 0) return 0;
  if (num_qubits > std::numeric_limits<std::size_t>::max() - 63) throw std::invalid_argument("num_qubits is too large");
  return (num_qubits + 63) / 64;
}

inline std::size_t product(std::size_t a, std::size_t b, const char* field) {
  if (a != 0 && b > std::numeric_limits<std::size_t>::max() / a)
    throw std::invalid_argument(std::string(field) + " size overflows size_t");
  return a * b;
}

inline std::size_t sum(std::size_t a, std::size_t b, const char* field) {
  if (b > std::numeric_limits<std::size_t>::max() - a)
    throw std::invalid_argument(std::string(field) + " size overflows size_t");
  return a + b;
}

inline std::size_t matmul_terms(std::size_t l, std::size_t r, std::size_t max_terms) {
  if (l != 0 && r > std::numeric_limits<std::size_t>::max() / l)
    throw std::invalid_argument("matmul intermediate term count overflows size_t");
  const std::size_t p = l * r;
  if (p > max_terms) throw std::invalid_argument("matmul intermediate term count exceeds max_intermediate_terms");
  return p;
}

inline std::size_t commutation_entries(std::size_t l, std::size_t r, std::size_t max_entries) {
  if (l != 0 && r > std::numeric_limits<std::size_t>::max() / l)
    throw std::invalid_argument("commutation matrix entry count overflows size_t");
  const std::size_t e = l * r;
  if (e > max_entries)
    throw std::invalid_argument("commutation matrix entry count exceeds max_commutation_matrix_entries");
  return e;
}

inline void statevector_length(std::size_t num_qubits, std::size_t actual) {
  if (num_qubits > 63) throw std::invalid_argument("expectation_statevector requires num_qubits <= 63");
  if (actual != (std::size_t{1} << num_qubits))
    throw std::invalid_argument("expectation_statevector requires len(psi) == 2 ** num_qubits");
}

}  // namespace wolfgang::guards
