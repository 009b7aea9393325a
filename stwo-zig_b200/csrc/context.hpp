// Definition of the opaque stwo_b200_context handle and the thread-local last
// error shared by the C ABI translation units.
#pragma once
#include <string>

#include "prover.hpp"

struct stwo_b200_context {
  sb::Context ctx;
};

namespace sb {
// Records the message returned by stwo_b200_last_error() and passes `code` through.
int32_t set_last_error(int32_t code, const std::string& msg);
}  // namespace sb
