// Allocation-free variant of the OODS point evaluation.
//
// stwo_b200_eval_at_point reduces each coefficient column in chunks and needs a
// scratch buffer of per-chunk partial sums, which it takes from the stream's
// memory pool. Some callers cannot allocate device memory at the moment they
// need this value: a serving loop that has admitted a request against an
// accounted device-memory budget and must not grow its footprint afterwards, an
// embedder whose own arena owns every byte of device memory, or code running
// where CUDA allocation calls are not allowed at all. This entry point keeps
// the partial sums in a fixed device array that lives in this file instead.
//
// Limits and sharing rules:
//  - The array holds STWO_B200_NOALLOC_EVAL_SCRATCH partial sums (16 bytes each,
//    1 MiB), i.e. n_cols * max(1, 2^(log_size - 12)) <= 65536; larger requests
//    are rejected with STWO_B200_E_INVALID.
//  - Every GPU that loads the library keeps its copy of the array until the
//    process exits.
//  - All calls on a device share the one array and it keeps the previous call's
//    contents. The kernels overwrite every partial they later read, so nothing
//    needs clearing, but two calls whose work overlaps on the GPU (different
//    streams, or different host threads) race on the array: serialize them.
//  - At most STWO_B200_EVAL_AT_POINT_MAX_COLS (65535) columns per call, the
//    grid's y extent, as for the allocating entry point.
//  - The first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) and caches it; make that first call before any
//    stream capture. The cached address belongs to the device's primary
//    context: an embedder that resets the device (cudaDeviceReset) must not
//    call this entry point again in the same process.
#include <mutex>
#include <string>

#include "../../include/stwo_b200.h"
#include "context.hpp"
#include "kernels.cuh"

namespace {

constexpr size_t kScratch = STWO_B200_NOALLOC_EVAL_SCRATCH;
static __device__ __align__(256) sb::QM31 g_eval_scratch[kScratch];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
sb::QM31* g_addr[kMaxDevices] = {};

// Host-side lookup of this device's copy of the array (the symbol itself is a
// host stand-in and must never be handed to a kernel). The caller has made
// `device` current.
int32_t scratch_address(int device, sb::QM31** out) {
  if (device < 0 || device >= kMaxDevices) return STWO_B200_E_INVALID;
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_eval_scratch);
    if (e != cudaSuccess || p == nullptr)
      return sb::set_last_error(STWO_B200_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_addr[device] = static_cast<sb::QM31*>(p);
  }
  *out = g_addr[device];
  return STWO_B200_OK;
}

}  // namespace

extern "C" {

int32_t stwo_b200_eval_at_point_noalloc(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols,
                                        const uint32_t* coeffs, uint64_t stride, stwo_b200_qm31 px,
                                        stwo_b200_qm31 py, stwo_b200_qm31* out_dev, void* stream) {
  if (!ctx) return sb::set_last_error(STWO_B200_E_INVALID, "null context");
  if (log_size > 28 || n_cols > sb::EVAL_AT_POINT_MAX_COLS || (n_cols && (!coeffs || !out_dev)))
    return sb::set_last_error(STWO_B200_E_INVALID, "bad eval_at_point_noalloc arguments");
  if (n_cols == 0) return STWO_B200_OK;
  if (!sb::eval_at_point_aligned(log_size, n_cols, coeffs, stride))
    return sb::set_last_error(STWO_B200_E_INVALID,
                              "coefficients must be 16-byte aligned with a stride of a multiple of 4");
  const size_t parts = sb::eval_at_point_partial_count(log_size, n_cols);
  if (parts > kScratch)
    return sb::set_last_error(STWO_B200_E_INVALID, "eval_at_point_noalloc: n_cols * max(1, 2^(log_size-12)) = " +
                                                       std::to_string(parts) + " partial sums exceed the fixed scratch of " +
                                                       std::to_string(kScratch));
  if (cudaSetDevice(ctx->ctx.device) != cudaSuccess) return sb::set_last_error(STWO_B200_E_CUDA, "cudaSetDevice failed");
  sb::QM31* scratch = nullptr;
  int32_t rc = scratch_address(ctx->ctx.device, &scratch);
  if (rc != STWO_B200_OK) return rc;
  sb::PointQ p{sb::qmake(px.a, px.b, px.c, px.d), sb::qmake(py.a, py.b, py.c, py.d)};
  cudaError_t e = sb::eval_at_point(ctx->ctx.tables, log_size, n_cols, coeffs, stride, p, nullptr, scratch,
                                    reinterpret_cast<sb::QM31*>(out_dev), reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return sb::set_last_error(STWO_B200_E_CUDA, std::string("eval_at_point_noalloc: ") + cudaGetErrorString(e));
  return STWO_B200_OK;
}

}  // extern "C"
