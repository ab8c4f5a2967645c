// Test infrastructure (oracle): the one symbol the gravity sources need from
// src/core/config.cpp (declared at include/cosmosim/core/config.hpp:1346-1349).
// config.cpp itself is not compiled: it does not build with g++ 13 at
// src/core/config.cpp:3867 and :4601.
#include "cosmosim/core/config.hpp"

namespace cosmosim::core {
ConfigError::ConfigError(const std::string& message) : std::runtime_error(message) {}
}  // namespace cosmosim::core
