#pragma once
// PauliSum: the host operator type.  Same public interface as
// include/wolfgang/pauli_sum.hpp of sghowell/wolfgang 0.2.3, so code written
// against the reference compiles unchanged.  Storage, I/O and arithmetic stay
// on the host; simplify, matmul, commutes_with, group_commuting and the
// expectations run on the B200 through the wg_* C-ABI (include/wg_pauli.h)
// and throw std::runtime_error when no CUDA device is visible -- there is no
// CPU fallback.

#include <complex>
#include <cstddef>
#include <cstdint>
#include <span>
#include <string>
#include <string_view>
#include <vector>

namespace wolfgang {

class PauliSum {
 public:
  // Sparse I/O term: local_pauli_string[k] acts on qubit_indices[k].
  struct SparseTerm {
    std::string local_pauli_string;
    std::vector<std::size_t> qubit_indices;
    std::complex<double> coefficient;
  };

  // num_terms identity terms with zero coefficients.
  PauliSum(std::size_t num_qubits, std::size_t num_terms);

  [[nodiscard]] static PauliSum empty(std::size_t num_qubits);

  // Dense labels in Qiskit display order: the right-most character is qubit 0.
  [[nodiscard]] static PauliSum from_labels(const std::vector<std::string>& labels,
                                            const std::vector<std::complex<double>>& coeffs);

  [[nodiscard]] static PauliSum from_sparse_list(const std::vector<SparseTerm>& terms,
                                                 std::size_t num_qubits);

  // Packed constructor for bulk ingestion: x/z hold num_terms*words words,
  // coeffs num_terms values; unused high bits of the last word must be zero.
  [[nodiscard]] static PauliSum from_packed(std::size_t num_qubits, std::vector<std::uint64_t> x,
                                            std::vector<std::uint64_t> z,
                                            std::vector<std::complex<double>> coeffs);

  [[nodiscard]] std::size_t num_qubits() const noexcept;
  [[nodiscard]] std::size_t num_terms() const noexcept;
  [[nodiscard]] std::size_t words() const noexcept;

  [[nodiscard]] std::vector<std::string> to_labels() const;
  [[nodiscard]] std::vector<SparseTerm> to_sparse_list() const;

  // Combine duplicate keys, drop |c| <= atol + rtol*max|c_in|, canonical order
  // x0, z0, x1, z1, ... (device).
  [[nodiscard]] PauliSum simplify(double atol = 1.0e-12, double rtol = 0.0) const;

  // Concatenation without simplify (host).
  [[nodiscard]] PauliSum add(const PauliSum& rhs) const;

  // Coefficient scaling (host).
  [[nodiscard]] PauliSum scalar_multiply(std::complex<double> scalar) const;

  // Matrix product: rhs acts first.  simplify_output=false keeps the
  // nested-loop product order (lhs outer) (device).
  [[nodiscard]] PauliSum matmul(const PauliSum& rhs, bool simplify_output = true,
                                std::size_t max_intermediate_terms = 50000000) const;

  // Row-major pairwise commutation flags, 1 = commute (device).
  [[nodiscard]] std::vector<std::uint8_t> commutes_with(
      const PauliSum& rhs, std::size_t max_commutation_matrix_entries = 100000000) const;

  // Deterministic greedy commuting groups; mode "qwc" or "full", strategy
  // "largest_first" (device greedy).
  [[nodiscard]] std::vector<PauliSum> group_commuting(std::string_view mode = "qwc",
                                                      std::string_view strategy = "largest_first",
                                                      std::size_t max_terms_for_graph = 50000) const;

  // <psi|H|psi>; the right-most label character is qubit 0 (device).
  [[nodiscard]] std::complex<double> expectation_statevector_complex128(
      std::span<const std::complex<double>> psi) const;
  [[nodiscard]] std::complex<double> expectation_statevector_complex64(
      std::span<const std::complex<float>> psi) const;

  // Expectation over computational-basis counts (diagonal terms) (device).
  [[nodiscard]] std::complex<double> expectation_z_counts(const std::vector<std::string>& bitstrings,
                                                          const std::vector<double>& counts) const;

  [[nodiscard]] static std::size_t checked_matmul_intermediate_terms_for_testing(
      std::size_t lhs_terms, std::size_t rhs_terms, std::size_t max_intermediate_terms);
  [[nodiscard]] static std::size_t checked_commutation_matrix_entries_for_testing(
      std::size_t lhs_terms, std::size_t rhs_terms, std::size_t max_commutation_matrix_entries);

  [[nodiscard]] const std::vector<std::uint64_t>& x_words() const noexcept;
  [[nodiscard]] const std::vector<std::uint64_t>& z_words() const noexcept;
  [[nodiscard]] const std::vector<std::complex<double>>& coeffs() const noexcept;

 private:
  friend class DevicePauliSum;

  PauliSum(std::size_t num_qubits, std::size_t words, std::size_t num_terms,
           std::vector<std::uint64_t> x, std::vector<std::uint64_t> z,
           std::vector<std::complex<double>> coeffs);

  // Takes ownership of device result buffers (library-allocated) and copies
  // them into a host PauliSum; their masks come from valid inputs, so they are
  // not re-checked.
  static PauliSum download_device_result(std::size_t num_qubits, std::size_t words, int device,
                                         std::uint64_t* x, std::uint64_t* z, double* coeffs,
                                         std::size_t num_terms);

  std::size_t num_qubits_;
  std::size_t words_;
  std::size_t num_terms_;
  std::vector<std::uint64_t> x_;
  std::vector<std::uint64_t> z_;
  std::vector<std::complex<double>> coeffs_;
};

}  // namespace wolfgang
