#pragma once
// Exception base kept for source compatibility with
// include/wolfgang/errors.hpp of sghowell/wolfgang 0.2.3.  Invalid arguments
// are reported as std::invalid_argument, device failures as std::runtime_error.

#include <stdexcept>
#include <string>

namespace wolfgang {

class WolfgangError : public std::runtime_error {
 public:
  explicit WolfgangError(const std::string& message) : std::runtime_error(message) {}
};

}  // namespace wolfgang
