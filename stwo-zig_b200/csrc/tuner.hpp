// Launch-shape autotuner, process-wide and keyed by (op, log_size, n_cols).
//
// Some kernels come in variants that write the same bits but differ in speed with the shape: the
// fused or generic FFT high pass, the Merkle leaf kernel built for 4, 5 or 6 CTAs per SM, the
// quotient kernel with different loads in flight and occupancy. The first call of a key runs every
// variant of its op on that call's own inputs, timed with CUDA events on the call's stream (the
// best of three interleaved runs each), and records the fastest; every later call of the key runs that variant.
// An op whose outputs overwrite its inputs (an in-place transform) cannot be re-run and takes its
// first variant untimed. Forcing a variant (tests, A/B runs) bypasses the table.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <vector>

namespace sb {

enum TuneOp : uint32_t {
  TUNE_LDE1 = 0,       // interpolate + blow-up-2 extension of 2^16 .. 2^22 columns: fused, generic high pass
  TUNE_LEAVES = 1,     // Merkle leaf kernel: 5, 6, 4 CTAs per SM
  TUNE_QUOTIENTS = 2,  // DEEP quotients: 6 loads in flight at 3 CTAs/SM, 3 at 4, 9 at 2; bulk-staged
  TUNE_OPS = 3,
};
constexpr int TUNE_MAX_VARIANTS = 4;

struct TuneEntry {
  uint32_t op, log_size, n_cols;
  int32_t variant;                // chosen variant
  float ms[TUNE_MAX_VARIANTS];    // measured time of each variant (0 for none)
};

// Runs run(v) with the key's variant v, tuning the key on its first call when `rerunnable`.
cudaError_t tuned_run(TuneOp op, uint32_t log_size, uint32_t n_cols, int n_variants, bool rerunnable,
                      cudaStream_t stream, const std::function<cudaError_t(int)>& run);
// -1: tune (the default); v >= 0: every op runs variant min(v, its count - 1) and nothing is tuned.
void tune_force(int v);
std::vector<TuneEntry> tune_table();
void tune_clear();

}  // namespace sb
