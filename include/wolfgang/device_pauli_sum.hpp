#pragma once
// DevicePauliSum: device-resident operator (include/wolfgang/device_pauli_sum.hpp
// of sghowell/wolfgang 0.2.3), backed by the sm_100a kernels of libwgpauli.so.
// Move-only owner of device buffers; results are new objects; every public
// call synchronises before returning, as in the reference.

#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "wolfgang/accelerator_status.hpp"
#include "wolfgang/device_commutation_matrix.hpp"
#include "wolfgang/pauli_sum.hpp"

namespace wolfgang {

struct CudaDeviceInfo {
  int ordinal = -1;
  std::string name;
  int compute_capability_major = 0;
  int compute_capability_minor = 0;
  std::size_t total_memory_bytes = 0;
};

struct CudaStatus {
  bool built = false;
  bool runtime_available = false;
  int device_count = 0;
  std::string skip_reason;
  std::string runtime_version;
  std::string driver_version;
  std::vector<CudaDeviceInfo> devices;
};

enum class DeviceStatevectorDtype {
  Complex64,
  Complex128,
};

// Bit-packed commutation matrix (new: no reference counterpart).  Row-major
// uint32 words, pitch = ceil(cols/32); bit (c%32) of word c/32 is 1 iff the
// pair commutes.  8x smaller than the uint8 matrix, so it is the form used for
// large term counts.
class DeviceCommutationBits {
 public:
  DeviceCommutationBits() noexcept;
  ~DeviceCommutationBits();
  DeviceCommutationBits(DeviceCommutationBits&& other) noexcept;
  DeviceCommutationBits& operator=(DeviceCommutationBits&& other) noexcept;
  DeviceCommutationBits(const DeviceCommutationBits&) = delete;
  DeviceCommutationBits& operator=(const DeviceCommutationBits&) = delete;

  [[nodiscard]] std::size_t rows() const noexcept;
  [[nodiscard]] std::size_t cols() const noexcept;
  [[nodiscard]] std::size_t pitch_words() const noexcept;
  [[nodiscard]] int device() const noexcept;
  [[nodiscard]] std::uintptr_t data_pointer() const noexcept;
  [[nodiscard]] std::vector<std::uint32_t> to_host() const;
  [[nodiscard]] std::uint64_t count_commuting() const;
  [[nodiscard]] std::vector<std::uint64_t> count_commuting_rows() const;
  [[nodiscard]] std::vector<std::uint64_t> count_commuting_cols() const;

 private:
  friend class DevicePauliSum;
  struct Impl;
  explicit DeviceCommutationBits(std::unique_ptr<Impl> impl) noexcept;
  std::unique_ptr<Impl> impl_;
};

class DevicePauliSum {
 public:
  DevicePauliSum() noexcept;
  ~DevicePauliSum();
  DevicePauliSum(DevicePauliSum&& other) noexcept;
  DevicePauliSum& operator=(DevicePauliSum&& other) noexcept;
  DevicePauliSum(const DevicePauliSum&) = delete;
  DevicePauliSum& operator=(const DevicePauliSum&) = delete;

  [[nodiscard]] static DevicePauliSum from_host(const PauliSum& host, int device = 0);
  [[nodiscard]] static DevicePauliSum from_host(const PauliSum& host, AcceleratorBackend backend,
                                                int device = 0);
  [[nodiscard]] static CudaStatus cuda_status();
  [[nodiscard]] static bool cuda_available();

  [[nodiscard]] PauliSum to_host() const;
  [[nodiscard]] DevicePauliSum simplify(double atol = 1.0e-12, double rtol = 0.0) const;
  [[nodiscard]] std::complex<double> expectation_statevector_complex128(
      std::span<const std::complex<double>> psi) const;
  [[nodiscard]] std::complex<double> expectation_statevector_complex64(
      std::span<const std::complex<float>> psi) const;
  [[nodiscard]] std::complex<double> expectation_statevector_device_pointer(
      std::uintptr_t device_pointer, DeviceStatevectorDtype dtype, std::size_t length) const;
  [[nodiscard]] std::vector<std::uint8_t> commutes_with(
      const DevicePauliSum& rhs, std::size_t max_commutation_matrix_entries = 100000000) const;
  void commutes_with_into(const DevicePauliSum& rhs, std::span<std::uint8_t> output,
                          std::size_t max_commutation_matrix_entries = 100000000) const;
  [[nodiscard]] DeviceCommutationMatrix commutes_with_device(
      const DevicePauliSum& rhs, std::size_t max_commutation_matrix_entries = 100000000) const;
  void commutes_with_device_into(const DevicePauliSum& rhs, DeviceCommutationMatrix& output,
                                 std::size_t max_commutation_matrix_entries = 100000000) const;
  // Bit-packed matrix (new); guarded by max_bits_entries (default 2^40).
  [[nodiscard]] DeviceCommutationBits commutes_with_bits(const DevicePauliSum& rhs,
                                                         std::size_t max_entries = std::size_t{1} << 40,
                                                         int algo = 0) const;
  [[nodiscard]] DevicePauliSum matmul(const DevicePauliSum& rhs, bool simplify_output = true,
                                      std::size_t max_intermediate_terms = 50000000) const;
  [[nodiscard]] std::vector<PauliSum> group_commuting(std::string_view mode = "qwc",
                                                      std::string_view strategy = "largest_first") const;
  [[nodiscard]] std::size_t num_qubits() const noexcept;
  [[nodiscard]] std::size_t num_terms() const noexcept;
  [[nodiscard]] std::size_t words() const noexcept;
  [[nodiscard]] int device() const noexcept;
  [[nodiscard]] std::string backend() const;

  // Device buffers (x/z: num_terms*words uint64; coeffs: 2*num_terms doubles).
  [[nodiscard]] std::uintptr_t x_pointer() const noexcept;
  [[nodiscard]] std::uintptr_t z_pointer() const noexcept;
  [[nodiscard]] std::uintptr_t coeffs_pointer() const noexcept;

  struct Impl;  // opaque device state

 private:
  explicit DevicePauliSum(std::unique_ptr<Impl> impl) noexcept;
  std::unique_ptr<Impl> impl_;
  friend class PauliSum;
};

}  // namespace wolfgang
