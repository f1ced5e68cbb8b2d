#pragma once
// Accelerator selection (include/wolfgang/accelerator_status.hpp of the
// reference).  This build has exactly one backend, CUDA on sm_100a; the other
// enumerators remain so that code written against the reference compiles, and
// selecting them raises "not built".

#include <string>
#include <string_view>

namespace wolfgang {

enum class AcceleratorBackend {
  None,
  Cuda,
  Hip,
  Metal,
};

struct AcceleratorObjectIdentity {
  AcceleratorBackend backend = AcceleratorBackend::None;
  int device_ordinal = -1;
};

[[nodiscard]] std::string_view accelerator_backend_name(AcceleratorBackend backend) noexcept;
[[nodiscard]] AcceleratorBackend accelerator_backend_from_name(std::string_view backend);
[[nodiscard]] std::string accelerator_not_built_message(AcceleratorBackend backend);

// Resolves None/Cuda to Cuda when a device is visible; Hip/Metal are not built.
[[nodiscard]] AcceleratorBackend select_accelerator_backend(AcceleratorBackend requested,
                                                            bool cuda_built, bool cuda_available,
                                                            bool hip_built, bool hip_available,
                                                            bool metal_built, bool metal_available);

// Throws std::invalid_argument when two operands live on different devices.
void validate_same_accelerator_context(std::string_view operation, AcceleratorObjectIdentity left,
                                       AcceleratorObjectIdentity right);

}  // namespace wolfgang
