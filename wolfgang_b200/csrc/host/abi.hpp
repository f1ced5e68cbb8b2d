#pragma once
// Host-side helpers over the wg_* C-ABI: status -> exception mapping and an
// owning device buffer.  The C++ drop-in classes reach the GPU only through
// these functions.

#include <cstddef>
#include <vector>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

#include "wg_pauli.h"

namespace wolfgang::abi {

// WG_ERR_INVALID -> std::invalid_argument (Python ValueError); everything else
// -> std::runtime_error, as the reference maps its own failures.
inline void check(int status) {
  if (status == WG_OK) return;
  const std::string msg = wg_last_error();
  if (status == WG_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

// Commutation algorithm for wg_commutation_bits when the caller holds the lhs
// terms on the host: the mean lhs weight (set qubits) over up to 256 rows,
// read from host memory, decides between the ballot kernel (1), whose cost is
// ~32 (4W + 2) instructions per output word whatever the weight, and the
// bit-plane kernel (2), ~8 per set bit + 16.  Without host terms the library's
// own size rule (algo 0) applies.
inline int commutation_algo_for(std::size_t words, const std::uint64_t* x, const std::uint64_t* z,
                                std::size_t n_lhs, std::size_t n_rhs) {
  if (words == 0 || words > 4 || n_rhs < 512 || n_lhs < 64) return 0;
  const std::size_t sample = n_lhs < 256 ? n_lhs : 256;
  std::size_t weight = 0;
  for (std::size_t i = 0; i < sample * words; ++i) weight += __builtin_popcountll(x[i] | z[i]);
  const double mean_w = static_cast<double>(weight) / static_cast<double>(sample);
  const double ballot_cost = 32.0 * (4.0 * static_cast<double>(words) + 2.0);
  const double plane_cost = 8.0 * mean_w + 16.0;
  return plane_cost < ballot_cost ? 2 : 1;
}

class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  DeviceBuffer(int device, std::size_t bytes) : device_(device), bytes_(bytes) {
    if (bytes) check(wg_malloc(device, bytes, nullptr, &ptr_));
  }
  // Adopts a buffer allocated by the library (e.g. wg_simplify outputs).
  static DeviceBuffer adopt(int device, void* ptr, std::size_t bytes) {
    DeviceBuffer b;
    b.device_ = device;
    b.ptr_ = ptr;
    b.bytes_ = bytes;
    return b;
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      reset();
      swap(o);
    }
    return *this;
  }
  ~DeviceBuffer() { reset(); }
  void reset() noexcept {
    if (ptr_) (void)wg_free(device_, ptr_, nullptr);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  void swap(DeviceBuffer& o) noexcept {
    std::swap(device_, o.device_);
    std::swap(ptr_, o.ptr_);
    std::swap(bytes_, o.bytes_);
  }
  void upload(const void* src, std::size_t bytes) {
    if (bytes) check(wg_memcpy_htod(device_, ptr_, src, bytes, nullptr));
  }
  void download(void* dst, std::size_t bytes) const {
    if (bytes) check(wg_memcpy_dtoh(device_, dst, ptr_, bytes, nullptr));
  }
  // Appends the buffer's first `count` elements to v, chunk by chunk, without
  // first filling v: reserve v's capacity beforehand.
  template <typename T>
  void append_to(std::vector<T>& v, std::size_t count) const {
    if (count == 0) return;
    auto fn = [](void* user, const void* chunk, std::size_t bytes) {
      auto* out = static_cast<std::vector<T>*>(user);
      const T* b = static_cast<const T*>(chunk);
      out->insert(out->end(), b, b + bytes / sizeof(T));
    };
    check(wg_memcpy_dtoh_chunked(device_, ptr_, count * sizeof(T), fn, &v, nullptr));
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr_);
  }
  void* get() const { return ptr_; }
  std::size_t bytes() const { return bytes_; }
  int device() const { return device_; }

 private:
  int device_ = 0;
  void* ptr_ = nullptr;
  std::size_t bytes_ = 0;
};

template <typename T>
DeviceBuffer upload_vector(int device, const T* data, std::size_t count) {
  DeviceBuffer b(device, count * sizeof(T));
  b.upload(data, count * sizeof(T));
  return b;
}

int visible_device_count();
// Device used by PauliSum (host) compute methods: ordinal 0, after checking a
// device is visible (std::runtime_error "no CUDA device is available").
int compute_device();

}  // namespace wolfgang::abi
