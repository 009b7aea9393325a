// Host-side verification of the library's proofs (verifier.cu).
#pragma once
#include <cstdint>
#include <string>

namespace sb {

// OK, or E_CONSTRAINTS with the first failed check in `err`.
int32_t verify_wide_fib_json(const std::string& proof, uint32_t log_n, uint32_t W, bool has_seed, uint64_t seed,
                             std::string& err);
int32_t verify_logup_xor_json(const std::string& proof, uint32_t log_n, uint32_t log_table, bool has_seed,
                              uint64_t seed, std::string& err);

}  // namespace sb
