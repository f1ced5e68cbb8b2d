// DevicePauliSum, DeviceCommutationMatrix, DeviceCommutationBits and the
// accelerator-status helpers, implemented over the wg_* C-ABI.
//
// Error messages and validation order follow the reference's CUDA backend
// (src/cuda/device_pauli_sum.cu, matmul_cuda.cu, commutation_cuda.cu,
// expectation_cuda.cu, device_commutation_matrix.cu, src/accelerator_status.cpp)
// so code and tests written against it see the same exceptions.

#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "abi.hpp"
#include "guards.hpp"
#include "wolfgang/accelerator_status.hpp"
#include "wolfgang/device_commutation_matrix.hpp"
#include "wolfgang/device_pauli_sum.hpp"

namespace wolfgang {

using abi::DeviceBuffer;

// ------------------------------------------------------------ device helpers

int abi::visible_device_count() {
  int n = 0;
  if (wg_device_count(&n) != WG_OK) return 0;
  return n;
}

int abi::compute_device() {
  if (visible_device_count() == 0) throw std::runtime_error("no CUDA device is available");
  return 0;
}

namespace {

void validate_device_ordinal(int device) {
  const int n = abi::visible_device_count();
  if (n == 0) throw std::runtime_error("no CUDA device is available");
  if (device < 0 || device >= n) throw std::invalid_argument("CUDA device ordinal is out of range");
}

std::string version_string(int v) {
  if (v <= 0) return "unknown";
  return std::to_string(v / 1000) + "." + std::to_string((v % 1000) / 10);
}

}  // namespace

// ------------------------------------------------------------ accelerator status

std::string_view accelerator_backend_name(AcceleratorBackend backend) noexcept {
  switch (backend) {
    case AcceleratorBackend::None: return "none";
    case AcceleratorBackend::Cuda: return "cuda";
    case AcceleratorBackend::Hip: return "hip";
    case AcceleratorBackend::Metal: return "metal";
  }
  return "unknown";
}

AcceleratorBackend accelerator_backend_from_name(std::string_view backend) {
  std::string s(backend);
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
  if (s == "auto") return AcceleratorBackend::None;
  if (s == "cuda") return AcceleratorBackend::Cuda;
  if (s == "hip") return AcceleratorBackend::Hip;
  if (s == "metal") return AcceleratorBackend::Metal;
  throw std::invalid_argument("backend must be None, 'auto', 'cuda', 'hip', or 'metal'");
}

std::string accelerator_not_built_message(AcceleratorBackend backend) {
  if (backend == AcceleratorBackend::Hip) return "Wolfgang was built without HIP support; this build targets CUDA sm_100a only.";
  if (backend == AcceleratorBackend::Metal)
    return "Wolfgang was built without Metal support; this build targets CUDA sm_100a only.";
  return "no CUDA device is available";
}

AcceleratorBackend select_accelerator_backend(AcceleratorBackend requested, bool cuda_built, bool cuda_available,
                                              bool hip_built, bool hip_available, bool metal_built,
                                              bool metal_available) {
  (void)cuda_built;
  (void)cuda_available;
  (void)hip_built;
  (void)hip_available;
  (void)metal_built;
  (void)metal_available;
  if (requested == AcceleratorBackend::Hip || requested == AcceleratorBackend::Metal)
    throw std::runtime_error(accelerator_not_built_message(requested));
  return AcceleratorBackend::Cuda;
}

void validate_same_accelerator_context(std::string_view operation, AcceleratorObjectIdentity left,
                                       AcceleratorObjectIdentity right) {
  if (left.backend == right.backend && left.device_ordinal == right.device_ordinal) return;
  throw std::invalid_argument(std::string(operation) +
                              " requires operands on the same accelerator backend and same device (operation=" +
                              std::string(operation) + ", left_backend=" +
                              std::string(accelerator_backend_name(left.backend)) +
                              ", left_device=" + std::to_string(left.device_ordinal) + ", right_backend=" +
                              std::string(accelerator_backend_name(right.backend)) +
                              ", right_device=" + std::to_string(right.device_ordinal) +
                              ", failure_stage=pre_allocation)");
}

// ------------------------------------------------------------ DevicePauliSum

struct DeviceCommutationBits::Impl {
  std::size_t rows = 0, cols = 0, pitch = 0;
  int device = 0;
  DeviceBuffer bits;
};


struct DevicePauliSum::Impl {
  std::size_t num_qubits = 0, words = 0, num_terms = 0;
  int device = 0;
  DeviceBuffer x, z, c;
  // x-grouped expectation plan, built on first use and reused: the operator is
  // immutable, so its grouping never changes.
  mutable wg_expect_plan_t plan = nullptr;
  ~Impl() {
    if (plan) (void)wg_expect_plan_destroy(plan);
  }
  wg_expect_plan_t get_plan() const {
    if (!plan)
      abi::check(wg_expect_plan_create(device, num_qubits, num_terms, x.as<std::uint64_t>(), z.as<std::uint64_t>(),
                                       c.as<double>(), &plan, nullptr));
    return plan;
  }
};

DevicePauliSum::DevicePauliSum() noexcept = default;
DevicePauliSum::DevicePauliSum(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
DevicePauliSum::~DevicePauliSum() = default;
DevicePauliSum::DevicePauliSum(DevicePauliSum&&) noexcept = default;
DevicePauliSum& DevicePauliSum::operator=(DevicePauliSum&&) noexcept = default;

namespace {
[[noreturn]] void moved_from() { throw std::runtime_error("DevicePauliSum is empty or moved-from"); }

std::unique_ptr<DevicePauliSum::Impl> make_like(const DevicePauliSum::Impl& a);
}  // namespace

DevicePauliSum DevicePauliSum::from_host(const PauliSum& host, int device) {
  return from_host(host, AcceleratorBackend::None, device);
}

DevicePauliSum DevicePauliSum::from_host(const PauliSum& host, AcceleratorBackend backend, int device) {
  (void)select_accelerator_backend(backend, true, true, false, false, false, false);
  validate_device_ordinal(device);
  auto impl = std::make_unique<Impl>();
  impl->num_qubits = host.num_qubits();
  impl->words = host.words();
  impl->num_terms = host.num_terms();
  impl->device = device;
  const std::size_t packed = guards::product(host.num_terms(), host.words(), "device packed words");
  impl->x = abi::upload_vector(device, host.x_words().data(), packed);
  impl->z = abi::upload_vector(device, host.z_words().data(), packed);
  impl->c = abi::upload_vector(device, host.coeffs().data(), host.num_terms());
  abi::check(wg_stream_synchronize(device, nullptr));
  return DevicePauliSum(std::move(impl));
}

CudaStatus DevicePauliSum::cuda_status() {
  CudaStatus st;
  st.built = true;
  int rt = 0, dr = 0;
  (void)wg_runtime_versions(&rt, &dr);
  st.runtime_version = version_string(rt);
  st.driver_version = version_string(dr);
  st.device_count = abi::visible_device_count();
  st.runtime_available = st.device_count > 0;
  if (!st.runtime_available) {
    st.skip_reason = "no CUDA device is available";
    return st;
  }
  for (int d = 0; d < st.device_count; ++d) {
    char name[256] = {0};
    int major = 0, minor = 0, sms = 0;
    std::size_t mem = 0;
    if (wg_device_info(d, name, sizeof(name), &major, &minor, &mem, &sms) != WG_OK) {
      st.runtime_available = false;
      st.skip_reason = std::string("CUDA runtime failed during device property discovery: ") + wg_last_error();
      st.devices.clear();
      return st;
    }
    st.devices.push_back(CudaDeviceInfo{d, name, major, minor, mem});
  }
  return st;
}

bool DevicePauliSum::cuda_available() { return cuda_status().runtime_available; }

PauliSum DevicePauliSum::to_host() const {
  if (!impl_) moved_from();
  const std::size_t packed = impl_->num_terms * impl_->words;
  std::vector<std::uint64_t> x(packed), z(packed);
  std::vector<std::complex<double>> c(impl_->num_terms);
  impl_->x.download(x.data(), packed * 8);
  impl_->z.download(z.data(), packed * 8);
  impl_->c.download(c.data(), c.size() * 16);
  return PauliSum(impl_->num_qubits, impl_->words, impl_->num_terms, std::move(x), std::move(z), std::move(c));
}

namespace {

std::unique_ptr<DevicePauliSum::Impl> make_like(const DevicePauliSum::Impl& a) {
  auto out = std::make_unique<DevicePauliSum::Impl>();
  out->num_qubits = a.num_qubits;
  out->words = a.words;
  out->device = a.device;
  return out;
}

void adopt_outputs(DevicePauliSum::Impl& out, std::uint64_t* ox, std::uint64_t* oz, double* oc, std::size_t U) {
  out.num_terms = U;
  out.x = DeviceBuffer::adopt(out.device, ox, U * out.words * 8);
  out.z = DeviceBuffer::adopt(out.device, oz, U * out.words * 8);
  out.c = DeviceBuffer::adopt(out.device, oc, U * 16);
}

}  // namespace

DevicePauliSum DevicePauliSum::simplify(double atol, double rtol) const {
  if (!impl_) moved_from();
  if (atol < 0.0 || rtol < 0.0 || !std::isfinite(atol) || !std::isfinite(rtol))
    throw std::invalid_argument("simplify tolerances must be non-negative finite values");
  auto out = make_like(*impl_);
  if (impl_->num_terms == 0) return DevicePauliSum(std::move(out));
  std::uint64_t *ox = nullptr, *oz = nullptr;
  double* oc = nullptr;
  std::size_t U = 0;
  abi::check(wg_simplify(impl_->device, impl_->words, impl_->num_terms, impl_->x.as<std::uint64_t>(),
                         impl_->z.as<std::uint64_t>(), impl_->c.as<double>(), atol, rtol, &ox, &oz, &oc, &U,
                         nullptr));
  adopt_outputs(*out, ox, oz, oc, U);
  return DevicePauliSum(std::move(out));
}

DevicePauliSum DevicePauliSum::matmul(const DevicePauliSum& rhs, bool simplify_output,
                                      std::size_t max_intermediate_terms) const {
  if (!impl_ || !rhs.impl_) moved_from();
  validate_same_accelerator_context("CUDA matmul", {AcceleratorBackend::Cuda, impl_->device},
                                    {AcceleratorBackend::Cuda, rhs.impl_->device});
  if (impl_->num_qubits != rhs.impl_->num_qubits)
    throw std::invalid_argument("PauliSum matmul requires the same num_qubits");
  const std::size_t P = guards::matmul_terms(impl_->num_terms, rhs.impl_->num_terms, max_intermediate_terms);
  auto out = make_like(*impl_);
  if (P == 0) return DevicePauliSum(std::move(out));
  std::uint64_t *ox = nullptr, *oz = nullptr;
  double* oc = nullptr;
  std::size_t U = 0;
  // The reference's device matmul always simplifies with simplify()'s
  // defaults (src/cuda/matmul_cuda.cu:459-462).
  abi::check(wg_pauli_products(impl_->device, impl_->words, impl_->x.as<std::uint64_t>(),
                               impl_->z.as<std::uint64_t>(), impl_->c.as<double>(), impl_->num_terms,
                               rhs.impl_->x.as<std::uint64_t>(), rhs.impl_->z.as<std::uint64_t>(),
                               rhs.impl_->c.as<double>(), rhs.impl_->num_terms,
                               simplify_output ? WG_PRODUCTS_SIMPLIFY : WG_PRODUCTS_RAW, 1.0e-12, 0.0, &ox, &oz, &oc,
                               &U, nullptr));
  adopt_outputs(*out, ox, oz, oc, U);
  return DevicePauliSum(std::move(out));
}

namespace {

template <typename C>
std::complex<double> run_plan_host_psi(const DevicePauliSum::Impl& im, std::span<const C> psi, int dtype) {
  guards::statevector_length(im.num_qubits, psi.size());
  if (im.num_terms == 0) return {0.0, 0.0};
  DeviceBuffer dpsi = abi::upload_vector(im.device, psi.data(), psi.size());
  DeviceBuffer res(im.device, 16);
  abi::check(wg_expect_plan_run(im.get_plan(), dpsi.get(), dtype, res.as<double>(), nullptr, nullptr, nullptr));
  double h[2];
  res.download(h, 16);
  return {h[0], h[1]};
}

}  // namespace

std::complex<double> DevicePauliSum::expectation_statevector_complex128(
    std::span<const std::complex<double>> psi) const {
  if (!impl_) moved_from();
  return run_plan_host_psi(*impl_, psi, WG_DTYPE_C128);
}

std::complex<double> DevicePauliSum::expectation_statevector_complex64(
    std::span<const std::complex<float>> psi) const {
  if (!impl_) moved_from();
  return run_plan_host_psi(*impl_, psi, WG_DTYPE_C64);
}

std::complex<double> DevicePauliSum::expectation_statevector_device_pointer(std::uintptr_t device_pointer,
                                                                          DeviceStatevectorDtype dtype,
                                                                          std::size_t length) const {
  if (!impl_) moved_from();
  guards::statevector_length(impl_->num_qubits, length);
  if (device_pointer == 0) throw std::invalid_argument("CUDA statevector data pointer must be non-null");
  const std::size_t item = dtype == DeviceStatevectorDtype::Complex128 ? 16 : 8;
  const std::size_t bytes = guards::product(length, item, "CUDA statevector allocation extent");
  int is_dev = 0, dev = -1, inside = 0;
  abi::check(wg_pointer_check(reinterpret_cast<const void*>(device_pointer), bytes, &is_dev, &dev, &inside));
  if (is_dev < 0) throw std::invalid_argument("CUDA statevector data pointer is not recognized device memory");
  if (is_dev == 0) throw std::invalid_argument("CUDA statevector must point to device memory");
  if (dev != impl_->device)
    throw std::invalid_argument("CUDA statevector must be on the same CUDA device as DevicePauliSum");
  if (!inside) throw std::invalid_argument("CUDA statevector byte range exceeds its backing allocation");
  if (impl_->num_terms == 0) return {0.0, 0.0};
  // The producer may have written psi on another stream (the reference
  // synchronises the device here too, src/cuda/expectation_cuda.cu:255-259).
  abi::check(wg_device_synchronize(impl_->device));
  DeviceBuffer res(impl_->device, 16);
  abi::check(wg_expect_plan_run(impl_->get_plan(), reinterpret_cast<const void*>(device_pointer),
                                dtype == DeviceStatevectorDtype::Complex128 ? WG_DTYPE_C128 : WG_DTYPE_C64,
                                res.as<double>(), nullptr, nullptr, nullptr));
  double h[2];
  res.download(h, 16);
  return {h[0], h[1]};
}

std::vector<std::uint8_t> DevicePauliSum::commutes_with(const DevicePauliSum& rhs,
                                                        std::size_t max_commutation_matrix_entries) const {
  if (!impl_ || !rhs.impl_) moved_from();
  const std::size_t entries =
      guards::commutation_entries(impl_->num_terms, rhs.impl_->num_terms, max_commutation_matrix_entries);
  std::vector<std::uint8_t> out(entries);
  commutes_with_into(rhs, std::span<std::uint8_t>(out), max_commutation_matrix_entries);
  return out;
}

namespace {

// Bit matrix of lhs x rhs on the lhs device.
DeviceBuffer commutation_bits(const DevicePauliSum::Impl& l, const DevicePauliSum::Impl& r, std::size_t pitch,
                              int algo) {
  DeviceBuffer bits(l.device, std::max<std::size_t>(4, l.num_terms * pitch * 4));
  abi::check(wg_commutation_bits(l.device, l.words, l.x.as<std::uint64_t>(), l.z.as<std::uint64_t>(), l.num_terms,
                                 r.x.as<std::uint64_t>(), r.z.as<std::uint64_t>(), r.num_terms,
                                 bits.as<std::uint32_t>(), pitch, algo, nullptr));
  return bits;
}

}  // namespace

void DevicePauliSum::commutes_with_into(const DevicePauliSum& rhs, std::span<std::uint8_t> output,
                                        std::size_t max_commutation_matrix_entries) const {
  if (!impl_ || !rhs.impl_) moved_from();
  validate_same_accelerator_context("CUDA commutes_with", {AcceleratorBackend::Cuda, impl_->device},
                                    {AcceleratorBackend::Cuda, rhs.impl_->device});
  if (impl_->num_qubits != rhs.impl_->num_qubits)
    throw std::invalid_argument("PauliSum commutes_with requires the same num_qubits");
  const std::size_t entries =
      guards::commutation_entries(impl_->num_terms, rhs.impl_->num_terms, max_commutation_matrix_entries);
  if (output.size() != entries)
    throw std::invalid_argument("CUDA commutes_with output buffer size does not match entry count");
  if (entries == 0) return;
  const std::size_t pitch = (rhs.impl_->num_terms + 31) / 32;
  DeviceBuffer bits = commutation_bits(*impl_, *rhs.impl_, pitch, 0);
  DeviceBuffer flags(impl_->device, entries);
  abi::check(wg_bits_to_u8(impl_->device, bits.as<std::uint32_t>(), impl_->num_terms, rhs.impl_->num_terms, pitch,
                           flags.as<std::uint8_t>(), nullptr));
  flags.download(output.data(), entries);
}

DeviceCommutationMatrix DevicePauliSum::commutes_with_device(const DevicePauliSum& rhs,
                                                             std::size_t max_commutation_matrix_entries) const {
  if (!impl_ || !rhs.impl_) moved_from();
  validate_same_accelerator_context("CUDA commutes_with_device", {AcceleratorBackend::Cuda, impl_->device},
                                    {AcceleratorBackend::Cuda, rhs.impl_->device});
  if (impl_->num_qubits != rhs.impl_->num_qubits)
    throw std::invalid_argument("PauliSum commutes_with requires the same num_qubits");
  (void)guards::commutation_entries(impl_->num_terms, rhs.impl_->num_terms, max_commutation_matrix_entries);
  DeviceCommutationMatrix out = DeviceCommutationMatrix::empty(impl_->num_terms, rhs.impl_->num_terms, impl_->device);
  commutes_with_device_into(rhs, out, max_commutation_matrix_entries);
  return out;
}

DeviceCommutationBits DevicePauliSum::commutes_with_bits(const DevicePauliSum& rhs, std::size_t max_entries,
                                                         int algo) const {
  if (!impl_ || !rhs.impl_) moved_from();
  validate_same_accelerator_context("CUDA commutes_with_bits", {AcceleratorBackend::Cuda, impl_->device},
                                    {AcceleratorBackend::Cuda, rhs.impl_->device});
  if (impl_->num_qubits != rhs.impl_->num_qubits)
    throw std::invalid_argument("PauliSum commutes_with requires the same num_qubits");
  (void)guards::commutation_entries(impl_->num_terms, rhs.impl_->num_terms, max_entries);
  const std::size_t pitch = (rhs.impl_->num_terms + 31) / 32;
  auto bi = std::make_unique<DeviceCommutationBits::Impl>();
  bi->rows = impl_->num_terms;
  bi->cols = rhs.impl_->num_terms;
  bi->pitch = pitch;
  bi->device = impl_->device;
  if (bi->rows && bi->cols) bi->bits = commutation_bits(*impl_, *rhs.impl_, pitch, algo);
  abi::check(wg_stream_synchronize(impl_->device, nullptr));
  return DeviceCommutationBits(std::move(bi));
}

std::vector<PauliSum> DevicePauliSum::group_commuting(std::string_view mode, std::string_view strategy) const {
  if (!impl_) moved_from();
  return to_host().group_commuting(mode, strategy);
}

std::size_t DevicePauliSum::num_qubits() const noexcept { return impl_ ? impl_->num_qubits : 0; }
std::size_t DevicePauliSum::num_terms() const noexcept { return impl_ ? impl_->num_terms : 0; }
std::size_t DevicePauliSum::words() const noexcept { return impl_ ? impl_->words : 0; }
int DevicePauliSum::device() const noexcept { return impl_ ? impl_->device : -1; }
std::string DevicePauliSum::backend() const { return impl_ ? "cuda" : "none"; }
std::uintptr_t DevicePauliSum::x_pointer() const noexcept {
  return impl_ ? reinterpret_cast<std::uintptr_t>(impl_->x.get()) : 0;
}
std::uintptr_t DevicePauliSum::z_pointer() const noexcept {
  return impl_ ? reinterpret_cast<std::uintptr_t>(impl_->z.get()) : 0;
}
std::uintptr_t DevicePauliSum::coeffs_pointer() const noexcept {
  return impl_ ? reinterpret_cast<std::uintptr_t>(impl_->c.get()) : 0;
}

// ------------------------------------------------------------ DeviceCommutationMatrix

struct DeviceCommutationMatrix::Impl {
  std::size_t rows = 0, cols = 0, entries = 0;
  int device = 0;
  DeviceBuffer data;  // dense uint8 flags, row-major
};

DeviceCommutationMatrix::DeviceCommutationMatrix() noexcept = default;
DeviceCommutationMatrix::DeviceCommutationMatrix(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
DeviceCommutationMatrix::~DeviceCommutationMatrix() = default;
DeviceCommutationMatrix::DeviceCommutationMatrix(DeviceCommutationMatrix&&) noexcept = default;
DeviceCommutationMatrix& DeviceCommutationMatrix::operator=(DeviceCommutationMatrix&&) noexcept = default;

namespace {
[[noreturn]] void matrix_moved() { throw std::runtime_error("DeviceCommutationMatrix is empty or moved-from"); }
}  // namespace

DeviceCommutationMatrix DeviceCommutationMatrix::empty(std::size_t rows, std::size_t cols, int device) {
  return empty(rows, cols, AcceleratorBackend::None, device);
}

DeviceCommutationMatrix DeviceCommutationMatrix::empty(std::size_t rows, std::size_t cols, AcceleratorBackend backend,
                                                       int device) {
  (void)select_accelerator_backend(backend, true, true, false, false, false, false);
  validate_device_ordinal(device);
  auto impl = std::make_unique<Impl>();
  impl->rows = rows;
  impl->cols = cols;
  impl->entries = guards::product(rows, cols, "device commutation matrix");
  impl->device = device;
  if (impl->entries) {
    impl->data = DeviceBuffer(device, impl->entries);
    abi::check(wg_memset(device, impl->data.get(), 0, impl->entries, nullptr));
    abi::check(wg_stream_synchronize(device, nullptr));
  }
  return DeviceCommutationMatrix(std::move(impl));
}

void DevicePauliSum::commutes_with_device_into(const DevicePauliSum& rhs, DeviceCommutationMatrix& output,
                                               std::size_t max_commutation_matrix_entries) const {
  if (!impl_ || !rhs.impl_) moved_from();
  if (!output.impl_) matrix_moved();
  validate_same_accelerator_context("CUDA commutes_with_device", {AcceleratorBackend::Cuda, impl_->device},
                                    {AcceleratorBackend::Cuda, rhs.impl_->device});
  validate_same_accelerator_context("CUDA commutes_with_device output", {AcceleratorBackend::Cuda, impl_->device},
                                    {AcceleratorBackend::Cuda, output.impl_->device});
  if (impl_->num_qubits != rhs.impl_->num_qubits)
    throw std::invalid_argument("PauliSum commutes_with requires the same num_qubits");
  const std::size_t entries =
      guards::commutation_entries(impl_->num_terms, rhs.impl_->num_terms, max_commutation_matrix_entries);
  if (output.impl_->rows != impl_->num_terms || output.impl_->cols != rhs.impl_->num_terms ||
      output.impl_->entries != entries)
    throw std::invalid_argument("CUDA commutes_with_device output shape does not match operand term counts");
  if (entries == 0) return;
  const std::size_t pitch = (rhs.impl_->num_terms + 31) / 32;
  DeviceBuffer bits = commutation_bits(*impl_, *rhs.impl_, pitch, 0);
  abi::check(wg_bits_to_u8(impl_->device, bits.as<std::uint32_t>(), impl_->num_terms, rhs.impl_->num_terms, pitch,
                           output.impl_->data.as<std::uint8_t>(), nullptr));
  abi::check(wg_stream_synchronize(impl_->device, nullptr));
}

std::uint64_t DeviceCommutationMatrix::count_commuting() const {
  if (!impl_) matrix_moved();
  std::uint64_t total = 0;
  abi::check(wg_u8_count(impl_->device, impl_->data.as<std::uint8_t>(), impl_->rows, impl_->cols, nullptr, nullptr,
                         &total, nullptr));
  return total;
}

namespace {
std::vector<std::uint64_t> axis_counts(int device, const std::uint8_t* data, std::size_t rows, std::size_t cols,
                                       bool by_row) {
  const std::size_t n = by_row ? rows : cols;
  std::vector<std::uint64_t> out(n, 0);
  if (n == 0) return out;
  DeviceBuffer buf(device, n * 8);
  abi::check(wg_u8_count(device, data, rows, cols, by_row ? buf.as<std::uint64_t>() : nullptr,
                         by_row ? nullptr : buf.as<std::uint64_t>(), nullptr, nullptr));
  buf.download(out.data(), n * 8);
  return out;
}
}  // namespace

std::vector<std::uint64_t> DeviceCommutationMatrix::count_commuting_rows() const {
  if (!impl_) matrix_moved();
  return axis_counts(impl_->device, impl_->data.as<std::uint8_t>(), impl_->rows, impl_->cols, true);
}

std::vector<std::uint64_t> DeviceCommutationMatrix::count_commuting_cols() const {
  if (!impl_) matrix_moved();
  return axis_counts(impl_->device, impl_->data.as<std::uint8_t>(), impl_->rows, impl_->cols, false);
}

std::vector<std::uint8_t> DeviceCommutationMatrix::to_host() const {
  if (!impl_) matrix_moved();
  std::vector<std::uint8_t> out(impl_->entries);
  impl_->data.download(out.data(), impl_->entries);
  return out;
}

std::size_t DeviceCommutationMatrix::rows() const noexcept { return impl_ ? impl_->rows : 0; }
std::size_t DeviceCommutationMatrix::cols() const noexcept { return impl_ ? impl_->cols : 0; }
std::size_t DeviceCommutationMatrix::num_entries() const noexcept { return impl_ ? impl_->entries : 0; }
int DeviceCommutationMatrix::device() const noexcept { return impl_ ? impl_->device : -1; }
std::string DeviceCommutationMatrix::backend() const { return impl_ ? "cuda" : "none"; }

std::uintptr_t DeviceCommutationMatrix::data_pointer_for_cuda_array_interface() const {
  if (!impl_) matrix_moved();
  return reinterpret_cast<std::uintptr_t>(impl_->data.get());
}

std::uintptr_t DeviceCommutationMatrix::data_pointer_for_dlpack() const {
  return data_pointer_for_cuda_array_interface();
}

int DeviceCommutationMatrix::dlpack_device_type() const {
  if (!impl_) matrix_moved();
  return 2;  // kDLCUDA
}

std::uint8_t* DeviceCommutationMatrix::mutable_data_for_device_write() {
  if (!impl_) matrix_moved();
  return impl_->data.as<std::uint8_t>();
}

void copy_device_commutation_matrix_from_host_for_testing(DeviceCommutationMatrix& matrix,
                                                          std::span<const std::uint8_t> values) {
  if (!matrix.impl_) matrix_moved();
  if (values.size() != matrix.impl_->entries)
    throw std::invalid_argument("DeviceCommutationMatrix testing copy size does not match matrix entries");
  if (values.empty()) return;
  matrix.impl_->data.upload(values.data(), values.size());
  abi::check(wg_stream_synchronize(matrix.impl_->device, nullptr));
}

// ------------------------------------------------------------ DeviceCommutationBits

DeviceCommutationBits::DeviceCommutationBits() noexcept = default;
DeviceCommutationBits::DeviceCommutationBits(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
DeviceCommutationBits::~DeviceCommutationBits() = default;
DeviceCommutationBits::DeviceCommutationBits(DeviceCommutationBits&&) noexcept = default;
DeviceCommutationBits& DeviceCommutationBits::operator=(DeviceCommutationBits&&) noexcept = default;

namespace {
[[noreturn]] void bits_moved() { throw std::runtime_error("DeviceCommutationBits is empty or moved-from"); }
}  // namespace

std::size_t DeviceCommutationBits::rows() const noexcept { return impl_ ? impl_->rows : 0; }
std::size_t DeviceCommutationBits::cols() const noexcept { return impl_ ? impl_->cols : 0; }
std::size_t DeviceCommutationBits::pitch_words() const noexcept { return impl_ ? impl_->pitch : 0; }
int DeviceCommutationBits::device() const noexcept { return impl_ ? impl_->device : -1; }
std::uintptr_t DeviceCommutationBits::data_pointer() const noexcept {
  return impl_ ? reinterpret_cast<std::uintptr_t>(impl_->bits.get()) : 0;
}

std::vector<std::uint32_t> DeviceCommutationBits::to_host() const {
  if (!impl_) bits_moved();
  std::vector<std::uint32_t> out(impl_->rows * impl_->pitch);
  if (!out.empty()) impl_->bits.download(out.data(), out.size() * 4);
  return out;
}

std::uint64_t DeviceCommutationBits::count_commuting() const {
  if (!impl_) bits_moved();
  std::uint64_t total = 0;
  abi::check(wg_bits_count(impl_->device, impl_->bits.as<std::uint32_t>(), impl_->rows, impl_->cols, impl_->pitch,
                           nullptr, nullptr, &total, nullptr));
  return total;
}

std::vector<std::uint64_t> DeviceCommutationBits::count_commuting_rows() const {
  if (!impl_) bits_moved();
  std::vector<std::uint64_t> out(impl_->rows, 0);
  if (out.empty()) return out;
  DeviceBuffer buf(impl_->device, out.size() * 8);
  abi::check(wg_bits_count(impl_->device, impl_->bits.as<std::uint32_t>(), impl_->rows, impl_->cols, impl_->pitch,
                           buf.as<std::uint64_t>(), nullptr, nullptr, nullptr));
  buf.download(out.data(), out.size() * 8);
  return out;
}

std::vector<std::uint64_t> DeviceCommutationBits::count_commuting_cols() const {
  if (!impl_) bits_moved();
  std::vector<std::uint64_t> out(impl_->cols, 0);
  if (out.empty()) return out;
  DeviceBuffer buf(impl_->device, out.size() * 8);
  abi::check(wg_bits_count(impl_->device, impl_->bits.as<std::uint32_t>(), impl_->rows, impl_->cols, impl_->pitch,
                           nullptr, buf.as<std::uint64_t>(), nullptr, nullptr));
  buf.download(out.data(), out.size() * 8);
  return out;
}

}  // namespace wolfgang
