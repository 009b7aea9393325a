// C ABI of libstwo_b200 (declarations and reference citations: include/stwo_b200.h).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/stwo_b200.h"
#include "alloc.hpp"
#include "context.hpp"
#include "prover.hpp"
#include "server.hpp"
#include "tuner.hpp"
#include "verifier.hpp"

namespace sb {
static std::atomic<uint64_t> g_launches(0);
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace sb

static_assert(sizeof(sb::StageTimes) == sizeof(stwo_b200_stage_times), "stage times layout");

namespace {
// Kernels behind the ABI read Merkle layers as 16-byte vectors, FRI fold sources as 8-byte pairs
// and OODS coefficients as 16-byte vectors: misaligned device pointers are refused up front.
inline bool is_aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }
}  // namespace

namespace {

thread_local std::string g_last_error;

int32_t set_error(int32_t code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace

namespace sb {
int32_t set_last_error(int32_t code, const std::string& msg) { return set_error(code, msg); }
}  // namespace sb

namespace {

#define CK_CTX(c)                                                      \
  do {                                                                 \
    if (!(c)) return set_error(STWO_B200_E_INVALID, "null context");   \
    cudaSetDevice((c)->ctx.device);                                    \
  } while (0)

int32_t cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return STWO_B200_OK;
  return set_error(STWO_B200_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

inline sb::QM31 q(stwo_b200_qm31 v) { return sb::qmake(v.a, v.b, v.c, v.d); }
inline cudaStream_t st(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr uint32_t TOWER_LOG = 22;  // domains up to 2^23

sb::ProveRequest to_request(const stwo_b200_wide_fib_request& r) {
  sb::ProveRequest p;
  p.log_n_rows = r.log_n_rows;
  p.sequence_len = r.sequence_len;
  p.config.pow_bits = r.config.pow_bits;
  p.config.log_blowup_factor = r.config.log_blowup_factor;
  p.config.log_last_layer_degree_bound = r.config.log_last_layer_degree_bound;
  p.config.n_queries = r.config.n_queries;
  p.trace_host = r.trace_host;
  p.trace_device = r.trace_device;
  p.trace_kind = (int)r.trace_kind;
  p.trace_seed = r.trace_seed;
  p.has_channel_seed = r.has_channel_seed != 0;
  p.channel_seed = r.channel_seed;
  return p;
}

bool domain_ok(const stwo_b200_context* c, uint32_t log_size) {
  return log_size >= 1 && log_size <= c->ctx.tables.tower_log + 1;
}

}  // namespace

extern "C" {

const char* stwo_b200_last_error(void) { return g_last_error.c_str(); }
const char* stwo_b200_status_string(int32_t s) { return sb::status_string(s); }
const char* stwo_b200_version(void) { return "stwo_b200 0.1 sm_100a"; }

int32_t stwo_b200_telemetry_snapshot(stwo_b200_telemetry* out) {
  if (!out) return set_error(STWO_B200_E_INVALID, "null telemetry output");
  out->kernel_launches = sb::launch_count();
  return STWO_B200_OK;
}

int32_t stwo_b200_context_create(int32_t device, stwo_b200_context** out) {
  if (!out) return set_error(STWO_B200_E_INVALID, "null output");
  *out = nullptr;
  auto* c = new stwo_b200_context();
  int32_t rc = c->ctx.init(device, TOWER_LOG);
  if (rc != STWO_B200_OK) {
    delete c;
    return set_error(rc, std::string("context init failed: ") + sb::status_string(rc));
  }
  *out = c;
  return STWO_B200_OK;
}

int32_t stwo_b200_context_destroy(stwo_b200_context* ctx) {
  if (!ctx) return STWO_B200_OK;
  cudaSetDevice(ctx->ctx.device);
  cudaDeviceSynchronize();
  delete ctx;
  return STWO_B200_OK;
}

int32_t stwo_b200_prove_wide_fibonacci(stwo_b200_context* ctx, const stwo_b200_wide_fib_request* req,
                                       uint8_t* proof_out, size_t proof_cap, size_t* proof_len,
                                       stwo_b200_stage_times* times) {
  CK_CTX(ctx);
  if (!req) return set_error(STWO_B200_E_INVALID, "null request");
  sb::WideFibProver* p = ctx->ctx.acquire();
  if (!p) return set_error(STWO_B200_E_CUDA, "stream creation failed");
  std::string proof;
  sb::StageTimes t;
  int32_t rc = p->prove(to_request(*req), proof, times ? &t : nullptr);
  std::string err = p->error();
  ctx->ctx.release(p);
  if (rc != STWO_B200_OK) return set_error(rc, err);
  if (times) std::memcpy(times, &t, sizeof(t));
  if (proof_len) *proof_len = proof.size();
  if (!proof_out || proof_cap < proof.size()) return set_error(STWO_B200_E_BUFFER_TOO_SMALL, "proof buffer too small");
  std::memcpy(proof_out, proof.data(), proof.size());
  return STWO_B200_OK;
}

int32_t stwo_b200_prove_wide_fibonacci_batch(stwo_b200_context* ctx, const stwo_b200_wide_fib_request* reqs,
                                             size_t n, uint8_t* const* proof_outs, const size_t* proof_caps,
                                             size_t* proof_lens, int32_t* statuses, uint32_t max_in_flight,
                                             stwo_b200_stage_times* times) {
  CK_CTX(ctx);
  if (n == 0) return STWO_B200_OK;
  if (!reqs || !proof_outs || !proof_caps || !proof_lens || !statuses)
    return set_error(STWO_B200_E_INVALID, "null batch argument");
  if (max_in_flight == 0) max_in_flight = 1;
  std::atomic<size_t> next(0);
  std::vector<std::string> errors(n);
  auto worker = [&]() {
    cudaSetDevice(ctx->ctx.device);
    sb::WideFibProver* p = ctx->ctx.acquire();
    for (;;) {
      size_t i = next.fetch_add(1);
      if (i >= n) break;
      if (!p) { statuses[i] = STWO_B200_E_CUDA; continue; }
      std::string proof;
      sb::StageTimes t;
      int32_t rc = p->prove(to_request(reqs[i]), proof, times ? &t : nullptr);
      if (times && rc == STWO_B200_OK) std::memcpy(&times[i], &t, sizeof(t));
      if (rc == STWO_B200_OK) {
        proof_lens[i] = proof.size();
        if (proof_outs[i] && proof_caps[i] >= proof.size()) std::memcpy(proof_outs[i], proof.data(), proof.size());
        else rc = STWO_B200_E_BUFFER_TOO_SMALL;
      } else {
        errors[i] = p->error();
      }
      statuses[i] = rc;
    }
    if (p) ctx->ctx.release(p);
  };
  size_t n_threads = std::min<size_t>(max_in_flight, n);
  std::vector<std::thread> threads;
  for (size_t t = 1; t < n_threads; ++t) threads.emplace_back(worker);
  worker();
  for (auto& t : threads) t.join();
  for (size_t i = 0; i < n; ++i)
    if (statuses[i] != STWO_B200_OK) return set_error(statuses[i], "request " + std::to_string(i) + ": " + errors[i]);
  return STWO_B200_OK;
}

int32_t stwo_b200_interpolate_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, uint32_t* cols,
                                      uint64_t stride, void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, log_size) || (!cols && n_cols)) return set_error(STWO_B200_E_INVALID, "bad interpolate arguments");
  return cuda_status(sb::fft_columns(ctx->ctx.tables, true, log_size, n_cols, cols, stride, st(stream)), "interpolate");
}

int32_t stwo_b200_evaluate_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, uint32_t* cols,
                                   uint64_t stride, void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, log_size) || (!cols && n_cols)) return set_error(STWO_B200_E_INVALID, "bad evaluate arguments");
  return cuda_status(sb::fft_columns(ctx->ctx.tables, false, log_size, n_cols, cols, stride, st(stream)), "evaluate");
}

int32_t stwo_b200_interpolate_and_extend(stwo_b200_context* ctx, uint32_t log_size, uint32_t log_blowup,
                                         uint32_t n_cols, const uint32_t* evals, uint64_t evals_stride,
                                         uint32_t* coeffs, uint64_t coeffs_stride, uint32_t* lde,
                                         uint64_t lde_stride, void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, log_size + log_blowup) || log_blowup == 0 || log_blowup > 4 || (n_cols && (!evals || !coeffs || !lde)))
    return set_error(STWO_B200_E_INVALID, "bad interpolate_and_extend arguments");
  return cuda_status(sb::interpolate_extend(ctx->ctx.tables, log_size, log_blowup, n_cols, evals, evals_stride, coeffs,
                                            coeffs_stride, lde, lde_stride, st(stream)),
                     "interpolate_and_extend");
}

int32_t stwo_b200_extend_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                                 const uint32_t* coeffs, uint64_t coeffs_stride, uint32_t* lde, uint64_t lde_stride,
                                 void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, log_size + log_blowup) || log_blowup == 0 || log_blowup > 4 || (n_cols && (!coeffs || !lde)))
    return set_error(STWO_B200_E_INVALID, "bad extend arguments");
  return cuda_status(sb::extend(ctx->ctx.tables, log_size, log_blowup, n_cols, coeffs, coeffs_stride, lde, lde_stride,
                                st(stream)),
                     "extend");
}

int32_t stwo_b200_eval_at_point(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, const uint32_t* coeffs,
                                uint64_t stride, stwo_b200_qm31 px, stwo_b200_qm31 py, stwo_b200_qm31* out_dev,
                                void* stream) {
  CK_CTX(ctx);
  if (log_size > 28 || n_cols > sb::EVAL_AT_POINT_MAX_COLS || (n_cols && (!coeffs || !out_dev)))
    return set_error(STWO_B200_E_INVALID, "bad eval_at_point arguments");
  if (n_cols == 0) return STWO_B200_OK;
  if (!sb::eval_at_point_aligned(log_size, n_cols, coeffs, stride))
    return set_error(STWO_B200_E_INVALID, "coefficients must be 16-byte aligned with a stride of a multiple of 4");
  size_t parts = sb::eval_at_point_partial_count(log_size, n_cols);
  void* scratch = nullptr;
  cudaError_t e = sb::dev_malloc_async(&scratch, parts * sizeof(sb::QM31), st(stream));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(STWO_B200_E_OOM, std::string("eval_at_point scratch: ") + cudaGetErrorString(e));
  }
  e = sb::eval_at_point(ctx->ctx.tables, log_size, n_cols, coeffs, stride, sb::PointQ{q(px), q(py)}, nullptr,
                        static_cast<sb::QM31*>(scratch), reinterpret_cast<sb::QM31*>(out_dev), st(stream));
  cudaError_t e2 = cudaFreeAsync(scratch, st(stream));
  if (e != cudaSuccess) return cuda_status(e, "eval_at_point");
  return cuda_status(e2, "eval_at_point scratch free");
}

int32_t stwo_b200_merkle_commit(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, const uint32_t* cols,
                                uint64_t stride, uint8_t* layers_dev, uint8_t* root_host, void* stream) {
  CK_CTX(ctx);
  if (log_size > 28 || !layers_dev || (n_cols && !cols)) return set_error(STWO_B200_E_INVALID, "bad merkle arguments");
  if (!is_aligned(layers_dev, 16)) return set_error(STWO_B200_E_INVALID, "layers_dev must be 16-byte aligned");
  if (n_cols == 0) log_size = 0;
  cudaError_t e = sb::merkle_commit(log_size, n_cols, cols, stride, layers_dev, st(stream));
  if (e != cudaSuccess) return cuda_status(e, "merkle_commit");
  if (root_host) {
    uint64_t root_node = (2ull << log_size) - 2;
    e = cudaMemcpyAsync(root_host, layers_dev + root_node * 32, 32, cudaMemcpyDeviceToHost, st(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(st(stream));
    return cuda_status(e, "merkle root readback");
  }
  return STWO_B200_OK;
}

int32_t stwo_b200_merkle_commit_lifted(stwo_b200_context* ctx, uint32_t n_cols, const uint32_t* const* cols,
                                       const uint32_t* log_sizes, uint8_t* layers_dev, uint8_t* root_host,
                                       void* stream) {
  CK_CTX(ctx);
  if (!layers_dev || (n_cols && (!cols || !log_sizes)) || n_cols > 2048)
    return set_error(STWO_B200_E_INVALID, "bad merkle_commit_lifted arguments");
  if (!is_aligned(layers_dev, 16)) return set_error(STWO_B200_E_INVALID, "layers_dev must be 16-byte aligned");
  uint32_t max_log = 0;
  for (uint32_t c = 0; c < n_cols; ++c) {
    if (log_sizes[c] > 28 || !cols[c]) return set_error(STWO_B200_E_INVALID, "bad lifted column");
    max_log = std::max(max_log, log_sizes[c]);
  }
  for (uint32_t c = 0; c < n_cols; ++c)
    if (log_sizes[c] == 0 && max_log > 0) return set_error(STWO_B200_E_INVALID, "lifted columns need log size >= 1");
  // Leaf order: stably sorted by log size ascending.
  std::vector<uint32_t> order(n_cols);
  for (uint32_t c = 0; c < n_cols; ++c) order[c] = c;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return log_sizes[a] < log_sizes[b]; });
  std::vector<uint64_t> staged(n_cols + (n_cols + 1) / 2 + 1, 0);
  uint32_t* logs = reinterpret_cast<uint32_t*>(staged.data() + n_cols);
  for (uint32_t i = 0; i < n_cols; ++i) {
    staged[i] = reinterpret_cast<uint64_t>(cols[order[i]]);
    logs[i] = log_sizes[order[i]];
  }
  cudaStream_t s = st(stream);
  void* dev = nullptr;
  cudaError_t e = cudaSuccess;
  if (n_cols) {
    e = cudaMallocAsync(&dev, staged.size() * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev, staged.data(), staged.size() * 8, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) {
    auto* dptr = static_cast<const uint32_t* const*>(dev);
    auto* dlog = dev ? reinterpret_cast<const uint32_t*>(static_cast<uint64_t*>(dev) + n_cols) : nullptr;
    e = sb::merkle_commit_lifted(max_log, n_cols, dptr, dlog, layers_dev, s);
  }
  // The staging copy above came from pageable memory, so it has completed; the free is stream-ordered.
  if (dev) {
    cudaError_t e2 = cudaFreeAsync(dev, s);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) return cuda_status(e, "merkle_commit_lifted");
  if (root_host) {
    const uint64_t leaves = n_cols ? (1ull << max_log) : 1;
    e = cudaMemcpyAsync(root_host, layers_dev + (2 * leaves - 2) * 32, 32, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "merkle root readback");
  }
  return STWO_B200_OK;
}

int32_t stwo_b200_fold_circle_into_line(stwo_b200_context* ctx, uint32_t src_log, const uint32_t* src,
                                        uint64_t src_stride, stwo_b200_qm31 alpha, uint32_t* dst,
                                        uint64_t dst_stride, int32_t accumulate, void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, src_log) || src_log < 2 || !src || !dst) return set_error(STWO_B200_E_INVALID, "bad fold arguments");
  if (!is_aligned(src, 8) || (src_stride & 1))
    return set_error(STWO_B200_E_INVALID, "fold source must be 8-byte aligned with an even stride");
  return cuda_status(sb::fold_circle_into_line(ctx->ctx.tables, src_log, src, src_stride, q(alpha), dst, dst_stride,
                                               accumulate != 0, st(stream)),
                     "fold_circle_into_line");
}

int32_t stwo_b200_fold_line(stwo_b200_context* ctx, uint32_t src_log, const uint32_t* src, uint64_t src_stride,
                            stwo_b200_qm31 alpha, uint32_t* dst, uint64_t dst_stride, void* stream) {
  CK_CTX(ctx);
  if (src_log < 1 || !domain_ok(ctx, src_log + 1) || !src || !dst) return set_error(STWO_B200_E_INVALID, "bad fold arguments");
  if (!is_aligned(src, 8) || (src_stride & 1))
    return set_error(STWO_B200_E_INVALID, "fold source must be 8-byte aligned with an even stride");
  return cuda_status(sb::fold_line(ctx->ctx.tables, src_log, src, src_stride, q(alpha), dst, dst_stride, st(stream)),
                     "fold_line");
}

namespace {
int32_t read_root(uint8_t* root_host, const uint8_t* layers_dev, uint32_t log_size, cudaStream_t s,
                  const char* what) {
  if (!root_host) return STWO_B200_OK;
  const uint64_t root_node = (2ull << log_size) - 2;
  cudaError_t e = cudaMemcpyAsync(root_host, layers_dev + root_node * 32, 32, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return cuda_status(e, what);
}
}  // namespace

int32_t stwo_b200_fold_and_commit(stwo_b200_context* ctx, int32_t circle, uint32_t src_log, const uint32_t* src,
                                  uint64_t src_stride, stwo_b200_qm31 alpha, uint32_t* dst, uint64_t dst_stride,
                                  uint8_t* layers_dev, uint8_t* root_host, void* stream) {
  CK_CTX(ctx);
  if (src_log < 2 || !domain_ok(ctx, circle ? src_log : src_log + 1) || !src || !dst ||
      (reinterpret_cast<uintptr_t>(src) & 7) || (src_stride & 1) || src_stride < (1ull << src_log) ||
      dst_stride < (1ull << (src_log - 1)) || (root_host && !layers_dev) || (layers_dev && !is_aligned(layers_dev, 16)))
    return set_error(STWO_B200_E_INVALID, "bad fold_and_commit arguments");
  cudaStream_t s = st(stream);
  void* a_dev = nullptr;
  cudaError_t e = cudaMallocAsync(&a_dev, sizeof(sb::QM31), s);
  if (e != cudaSuccess) return cuda_status(e, "fold_and_commit alpha");
  const sb::QM31 a = q(alpha);
  e = cudaMemcpyAsync(a_dev, &a, sizeof(a), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = sb::fri_fold_commit(ctx->ctx.tables, circle != 0, src_log, src, src_stride,
                            static_cast<const sb::QM31*>(a_dev), dst, dst_stride, layers_dev, s);
  cudaError_t e2 = cudaFreeAsync(a_dev, s);
  if (e != cudaSuccess) return cuda_status(e, "fold_and_commit");
  if (e2 != cudaSuccess) return cuda_status(e2, "fold_and_commit alpha free");
  return read_root(root_host, layers_dev, src_log - 1, s, "fold_and_commit root readback");
}

int32_t stwo_b200_commit_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                                 const uint32_t* evals, uint64_t evals_stride, uint32_t* coeffs, uint64_t coeffs_stride,
                                 uint32_t* lde, uint64_t lde_stride, uint8_t* layers_dev, uint8_t* root_host,
                                 void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, log_size + log_blowup) || log_blowup == 0 || log_blowup > 4 || n_cols == 0 || !evals ||
      !coeffs || !lde || !layers_dev || !is_aligned(layers_dev, 16))
    return set_error(STWO_B200_E_INVALID, "bad commit_columns arguments");
  cudaStream_t s = st(stream);
  cudaError_t e = sb::interpolate_extend(ctx->ctx.tables, log_size, log_blowup, n_cols, evals, evals_stride, coeffs,
                                         coeffs_stride, lde, lde_stride, s);
  if (e == cudaSuccess) e = sb::merkle_commit(log_size + log_blowup, n_cols, lde, lde_stride, layers_dev, s);
  if (e != cudaSuccess) return cuda_status(e, "commit_columns");
  return read_root(root_host, layers_dev, log_size + log_blowup, s, "commit_columns root readback");
}

int32_t stwo_b200_interpolate_secure_composition(stwo_b200_context* ctx, uint32_t comp_log, uint32_t* comp,
                                                 uint64_t comp_stride, uint32_t log_blowup, uint32_t* lde,
                                                 uint64_t lde_stride, void* stream) {
  CK_CTX(ctx);
  if (comp_log < 2 || log_blowup == 0 || log_blowup > 4 || !domain_ok(ctx, comp_log - 1 + log_blowup) || !comp ||
      !lde || comp_stride < (1ull << comp_log))
    return set_error(STWO_B200_E_INVALID, "bad interpolate_secure_composition arguments");
  cudaStream_t s = st(stream);
  const sb::DeviceTables& T = ctx->ctx.tables;
  const uint32_t half_log = comp_log - 1;
  cudaError_t e = sb::fft_columns(T, true, comp_log, 4, comp, comp_stride, s);
  if (e == cudaSuccess) e = sb::extend(T, half_log, log_blowup, 4, comp, comp_stride, lde, lde_stride, s);
  if (e == cudaSuccess)
    e = sb::extend(T, half_log, log_blowup, 4, comp + (1ull << half_log), comp_stride, lde + 4 * lde_stride, lde_stride, s);
  return cuda_status(e, "interpolate_secure_composition");
}

int32_t stwo_b200_accumulate_quotients(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols,
                                       const uint32_t* const* col_ptrs_dev, const stwo_b200_qm31* c_dev,
                                       stwo_b200_qm31 px, stwo_b200_qm31 py, stwo_b200_qm31 sum_a,
                                       stwo_b200_qm31 sum_b, uint32_t* out, uint64_t out_stride, void* stream) {
  CK_CTX(ctx);
  if (!domain_ok(ctx, log_size) || n_cols == 0 || n_cols > 1024 || !col_ptrs_dev || !c_dev || !out)
    return set_error(STWO_B200_E_INVALID, "bad quotient arguments");
  sb::QuotientBatchDev hb;
  hb.point = sb::PointQ{q(px), q(py)};
  hb.sum_a = q(sum_a);
  hb.sum_b = q(sum_b);
  hb.first = 0;
  hb.count = n_cols;
  // The column pointers are read back so that 16-byte aligned columns may take the bulk-staged
  // kernel, whose status word sits after the batch descriptor.
  std::vector<const uint32_t*> hptr(n_cols);
  cudaError_t e = cudaMemcpyAsync(hptr.data(), col_ptrs_dev, n_cols * sizeof(void*), cudaMemcpyDeviceToHost, st(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(st(stream));
  if (e != cudaSuccess) return cuda_status(e, "quotient column pointers");
  bool aligned = true;
  for (const uint32_t* p : hptr) aligned = aligned && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
  constexpr size_t STATUS_OFF = (sizeof(sb::QuotientBatchDev) + 15) & ~size_t(15);
  void* dbatch = nullptr;
  e = cudaMallocAsync(&dbatch, STATUS_OFF + 16, st(stream));
  if (e != cudaSuccess) return cuda_status(e, "quotient batch");
  uint32_t* dstatus = reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(dbatch) + STATUS_OFF);
  e = cudaMemcpyAsync(dbatch, &hb, sizeof(hb), cudaMemcpyHostToDevice, st(stream));
  if (e == cudaSuccess) e = cudaMemsetAsync(dstatus, 0, sizeof(uint32_t), st(stream));
  if (e == cudaSuccess)
    e = sb::accumulate_quotients(ctx->ctx.tables, log_size, 1, n_cols, static_cast<sb::QuotientBatchDev*>(dbatch), col_ptrs_dev,
                                 reinterpret_cast<const sb::QM31*>(c_dev), out, out_stride, st(stream),
                                 aligned ? dstatus : nullptr);
  uint32_t status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, dstatus, sizeof(status), cudaMemcpyDeviceToHost, st(stream));
  cudaError_t e2 = cudaStreamSynchronize(st(stream));  // the batch descriptor lives on this host frame
  cudaFreeAsync(dbatch, st(stream));
  if (e != cudaSuccess) return cuda_status(e, "accumulate_quotients");
  if (e2 != cudaSuccess) return cuda_status(e2, "accumulate_quotients sync");
  if (status != 0)
    return set_error(STWO_B200_E_CUDA, (status & sb::QUOT_STATUS_TIMEOUT)
                                           ? "a staged column load of the quotient kernel ran out of time"
                                           : "the quotient batches do not fit the staged kernel's item table");
  return STWO_B200_OK;
}

int32_t stwo_b200_wide_fib_trace(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t sequence_len,
                                 uint32_t trace_kind, uint64_t seed, uint32_t* out, uint64_t stride, void* stream) {
  CK_CTX(ctx);
  if (log_n_rows == 0 || log_n_rows > 28 || sequence_len < 2 || !out || trace_kind > 2)
    return set_error(STWO_B200_E_INVALID, "bad trace arguments");
  return cuda_status(sb::wide_fib_trace(log_n_rows, sequence_len, (int)trace_kind, seed, out, stride, st(stream)),
                     "wide_fib_trace");
}

int32_t stwo_b200_quadratic_recurrence_trace(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t n_cols,
                                             const uint32_t recipe[7], uint32_t* out, uint64_t stride, void* stream) {
  CK_CTX(ctx);
  if (log_n_rows == 0 || log_n_rows > 28 || n_cols < 2 || !recipe || !out || stride < (1ull << log_n_rows))
    return set_error(STWO_B200_E_INVALID, "bad quadratic recurrence arguments");
  return cuda_status(sb::quadratic_trace(log_n_rows, n_cols, recipe, out, stride, st(stream)),
                     "quadratic_recurrence_trace");
}

int32_t stwo_b200_wide_fib_composition(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t sequence_len,
                                       const uint32_t* eval, uint64_t stride, const stwo_b200_qm31* coeffs_dev,
                                       uint32_t den_inv0, uint32_t den_inv1, uint32_t* out, uint64_t out_stride,
                                       void* stream) {
  CK_CTX(ctx);
  if (log_n_rows == 0 || log_n_rows > 27 || sequence_len < 3 || sequence_len > 3000 || !eval || !coeffs_dev || !out)
    return set_error(STWO_B200_E_INVALID, "bad composition arguments");
  return cuda_status(sb::wide_fib_composition(log_n_rows, sequence_len, eval, stride,
                                              reinterpret_cast<const sb::QM31*>(coeffs_dev), den_inv0, den_inv1, out,
                                              out_stride, st(stream)),
                     "wide_fib_composition");
}

int32_t stwo_b200_accumulate(stwo_b200_context* ctx, uint32_t dst_log, uint32_t* dst, uint64_t dst_stride,
                             uint32_t src_log, const uint32_t* src, uint64_t src_stride, stwo_b200_qm31 coeff,
                             void* stream) {
  CK_CTX(ctx);
  if (dst_log > 30 || src_log > dst_log || !dst || !src || dst_stride < (1ull << dst_log) ||
      src_stride < (1ull << src_log))
    return set_error(STWO_B200_E_INVALID, "bad accumulate arguments");
  return cuda_status(sb::accumulate_lifted(dst_log, dst, dst_stride, src_log, src, src_stride, q(coeff), st(stream)),
                     "accumulate");
}

int32_t stwo_b200_pow_grind(stwo_b200_context* ctx, const uint8_t prefix_digest[32], uint32_t n_bits,
                            uint64_t* nonce_out) {
  CK_CTX(ctx);
  if (!prefix_digest || !nonce_out || n_bits > sb::MAX_POW_BITS)
    return set_error(STWO_B200_E_INVALID, "bad pow arguments (n_bits above STWO_B200_MAX_POW_BITS)");
  if (n_bits == 0) { *nonce_out = 0; return STWO_B200_OK; }
  std::lock_guard<std::mutex> g(ctx->ctx.small_mu);
  cudaStream_t s = ctx->ctx.stream;
  uint32_t* res = ctx->ctx.small;
  uint32_t w[8];
  std::memcpy(w, prefix_digest, 32);
  // The prover's search: bounded rounds in nonce order, four per check, at most 2^(bits+16) nonces.
  const uint64_t max_nonce = n_bits >= 48 ? ~0ull : (1ull << (n_bits + 16));
  const uint64_t per_round = sb::pow_round_nonces(ctx->ctx.sm_count);
  cudaError_t e = cudaMemsetAsync(res, 0xff, 8, s);
  uint64_t nonce = ~0ull;
  for (uint64_t base = 0; e == cudaSuccess && base < max_nonce && nonce == ~0ull;) {
    for (int r = 0; r < 4 && base < max_nonce && e == cudaSuccess; ++r, base += per_round)
      e = sb::pow_round(w, n_bits, base, res, ctx->ctx.sm_count, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nonce, res, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) return cuda_status(e, "pow_grind");
  if (nonce == ~0ull) return set_error(STWO_B200_E_TIMEOUT, "proof-of-work search bound reached");
  *nonce_out = nonce;
  return STWO_B200_OK;
}

int32_t stwo_b200_verify_wide_fibonacci(const uint8_t* proof, size_t proof_len, uint32_t log_n_rows,
                                        uint32_t sequence_len, uint32_t has_channel_seed, uint64_t channel_seed) {
  if (!proof) return set_error(STWO_B200_E_INVALID, "null proof");
  std::string err;
  int32_t rc = sb::verify_wide_fib_json(std::string(reinterpret_cast<const char*>(proof), proof_len), log_n_rows,
                                        sequence_len, has_channel_seed != 0, channel_seed, err);
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_verify_logup_xor(const uint8_t* proof, size_t proof_len, uint32_t log_n, uint32_t log_table,
                                   uint32_t has_channel_seed, uint64_t channel_seed) {
  if (!proof) return set_error(STWO_B200_E_INVALID, "null proof");
  std::string err;
  int32_t rc = sb::verify_logup_xor_json(std::string(reinterpret_cast<const char*>(proof), proof_len), log_n,
                                         log_table, has_channel_seed != 0, channel_seed, err);
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_prove_logup_xor(stwo_b200_context* ctx, const stwo_b200_xor_request* req, uint8_t* proof_out,
                                  size_t proof_cap, size_t* proof_len) {
  CK_CTX(ctx);
  if (!req || !proof_len) return set_error(STWO_B200_E_INVALID, "null argument");
  sb::XorRequest r;
  r.log_n = req->log_n;
  r.log_table = req->log_table;
  r.seed = req->seed;
  r.config.pow_bits = req->config.pow_bits;
  r.config.log_blowup_factor = req->config.log_blowup_factor;
  r.config.log_last_layer_degree_bound = req->config.log_last_layer_degree_bound;
  r.config.n_queries = req->config.n_queries;
  r.has_channel_seed = req->has_channel_seed != 0;
  r.channel_seed = req->channel_seed;
  sb::LogupXorProver* p = ctx->ctx.acquire_xor();
  std::string proof;
  int32_t rc = p->prove(r, proof);
  std::string err = p->error();
  ctx->ctx.release_xor(p);
  if (rc != STWO_B200_OK) return set_error(rc, err);
  *proof_len = proof.size();
  if (!proof_out || proof_cap < proof.size()) return set_error(STWO_B200_E_BUFFER_TOO_SMALL, "proof buffer too small");
  std::memcpy(proof_out, proof.data(), proof.size());
  return STWO_B200_OK;
}

struct stwo_b200_server {
  sb::Server* server;
  stwo_b200_context* ctx;
};

int32_t stwo_b200_server_create(stwo_b200_context* ctx, const stwo_b200_server_config* cfg,
                                stwo_b200_server** out) {
  CK_CTX(ctx);
  if (!cfg || !out || cfg->profile > 2 || cfg->slots > 64 || cfg->flags > 3)
    return set_error(STWO_B200_E_INVALID, "bad server config");
  uint64_t budget = cfg->memory_budget;
  if (budget == 0) {
    size_t free_b = 0, total_b = 0;
    cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemGetInfo");
    budget = free_b / 10 * 8;
  }
  auto* s = new stwo_b200_server{new sb::Server(&ctx->ctx, cfg->slots ? cfg->slots : 8, budget, cfg->profile, cfg->flags),
                                ctx};
  int32_t rc = s->server->start();
  if (rc != STWO_B200_OK) {
    delete s->server;
    delete s;
    return set_error(rc, "server start failed");
  }
  *out = s;
  return STWO_B200_OK;
}

int32_t stwo_b200_server_submit(stwo_b200_server* server, const stwo_b200_wide_fib_request* req, uint64_t* ticket) {
  if (!server || !req || !ticket) return set_error(STWO_B200_E_INVALID, "null server argument");
  std::string err;
  int32_t rc = server->server->submit(to_request(*req), ticket, &err);
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_server_submit_xor(stwo_b200_server* server, const stwo_b200_xor_request* req, uint64_t* ticket) {
  if (!server || !req || !ticket) return set_error(STWO_B200_E_INVALID, "null server argument");
  sb::XorRequest r;
  r.log_n = req->log_n;
  r.log_table = req->log_table;
  r.seed = req->seed;
  r.config.pow_bits = req->config.pow_bits;
  r.config.log_blowup_factor = req->config.log_blowup_factor;
  r.config.log_last_layer_degree_bound = req->config.log_last_layer_degree_bound;
  r.config.n_queries = req->config.n_queries;
  r.has_channel_seed = req->has_channel_seed != 0;
  r.channel_seed = req->channel_seed;
  std::string err;
  int32_t rc = server->server->submit_xor(r, ticket, &err);
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_server_wait(stwo_b200_server* server, uint64_t ticket, uint8_t* proof_out, size_t proof_cap,
                              size_t* proof_len, stwo_b200_request_stats* stats) {
  if (!server) return set_error(STWO_B200_E_INVALID, "null server");
  std::string err;
  sb::RequestStats st;
  int32_t rc = server->server->wait(ticket, proof_out, proof_cap, proof_len, &st, &err);
  if (stats) {
    stats->accounted_bytes = st.accounted_bytes;
    stats->workspace_bytes = st.workspace_bytes;
    stats->queued_ms = st.queued_ms;
    stats->run_ms = st.run_ms;
    stats->slot = st.slot;
    static_assert(sizeof(stats->stages) == sizeof(st.stages), "stage times layout");
    std::memcpy(&stats->stages, &st.stages, sizeof(st.stages));
  }
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_server_warmup(stwo_b200_server* server, uint32_t max_log_n_rows, uint32_t max_sequence_len,
                                uint32_t log_blowup, uint32_t max_xor_log_n) {
  if (!server || max_log_n_rows > 22 || max_xor_log_n > 22 || log_blowup < 1 || log_blowup > 4 ||
      (max_log_n_rows && (max_sequence_len < 2 || max_sequence_len > 1000)))
    return set_error(STWO_B200_E_INVALID, "bad warmup arguments");
  std::string err;
  int32_t rc = server->server->warmup(max_log_n_rows, max_sequence_len, log_blowup, max_xor_log_n, &err);
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_server_set_request_timeout(stwo_b200_server* server, uint32_t timeout_ms) {
  if (!server) return set_error(STWO_B200_E_INVALID, "null server");
  server->server->set_request_timeout(timeout_ms);
  return STWO_B200_OK;
}

int32_t stwo_b200_autotune_mode(int32_t mode) {
  if (mode < -1) return set_error(STWO_B200_E_INVALID, "autotune mode is -1 (tune) or a variant index");
  sb::tune_force(mode);
  return STWO_B200_OK;
}

int32_t stwo_b200_autotune_wide_fibonacci(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t sequence_len,
                                          uint32_t log_blowup) {
  CK_CTX(ctx);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_status(e, "autotune: device synchronization");
  sb::ProveRequest r;
  r.log_n_rows = log_n_rows;
  r.sequence_len = sequence_len;
  r.config.pow_bits = 0;  // the grind has no variants
  r.config.log_blowup_factor = log_blowup;
  r.config.log_last_layer_degree_bound = 0;
  r.config.n_queries = 3;
  r.trace_kind = 1;
  r.trace_seed = 1;
  sb::WideFibProver* p = ctx->ctx.acquire();
  if (!p) return set_error(STWO_B200_E_CUDA, "stream creation failed");
  std::string proof;
  int32_t rc = p->prove(r, proof, nullptr);
  std::string err = p->error();
  ctx->ctx.release(p);
  return rc == STWO_B200_OK ? rc : set_error(rc, err);
}

int32_t stwo_b200_autotune_table(stwo_b200_tune_entry* out, size_t cap, size_t* n) {
  if (!n) return set_error(STWO_B200_E_INVALID, "null count");
  std::vector<sb::TuneEntry> t = sb::tune_table();
  *n = t.size();
  if (t.size() > cap || (t.size() && !out)) return set_error(STWO_B200_E_BUFFER_TOO_SMALL, "autotune table buffer too small");
  static_assert(sizeof(sb::TuneEntry) == sizeof(stwo_b200_tune_entry), "tune entry layout");
  if (!t.empty()) std::memcpy(out, t.data(), t.size() * sizeof(sb::TuneEntry));
  return STWO_B200_OK;
}

int32_t stwo_b200_arm_quotient_stage_timeout_for_testing(void) {
  sb::arm_quotient_stage_timeout_for_testing();
  return STWO_B200_OK;
}

int32_t stwo_b200_arm_allocation_failure_for_testing(uint32_t nth) {
  sb::alloc_fail_countdown().store(nth, std::memory_order_relaxed);
  return STWO_B200_OK;
}

int32_t stwo_b200_server_snapshot_get(stwo_b200_server* server, stwo_b200_server_snapshot* out) {
  if (!server || !out) return set_error(STWO_B200_E_INVALID, "null server argument");
  sb::ServerSnapshot s = server->server->snapshot();
  out->submitted = s.submitted;
  out->completed = s.completed;
  out->failed = s.failed;
  out->rejected = s.rejected;
  out->peak_in_flight = s.peak_in_flight;
  out->peak_workspace_bytes = s.peak_workspace_bytes;
  out->budget_bytes = s.budget_bytes;
  return STWO_B200_OK;
}

int32_t stwo_b200_server_destroy(stwo_b200_server* server) {
  if (!server) return STWO_B200_OK;
  cudaSetDevice(server->ctx->ctx.device);
  delete server->server;
  delete server;
  return STWO_B200_OK;
}

int32_t stwo_b200_xor_lookup_trace(stwo_b200_context* ctx, uint32_t log_n, uint64_t seed, uint32_t* main_cols,
                                   uint32_t* table, uint32_t* multiplicity, void* stream) {
  CK_CTX(ctx);
  if (log_n > 28 || !main_cols || !table || !multiplicity)
    return set_error(STWO_B200_E_INVALID, "bad xor_lookup_trace arguments");
  return cuda_status(sb::xor_lookup_trace(log_n, seed, main_cols, table, multiplicity, st(stream)), "xor_lookup_trace");
}

int32_t stwo_b200_batch_inverse(stwo_b200_context* ctx, uint32_t degree, uint64_t n, const uint32_t* src,
                                uint64_t src_stride, uint32_t* dst, uint64_t dst_stride, void* stream) {
  CK_CTX(ctx);
  if ((degree != 1 && degree != 2 && degree != 4) || (n && (!src || !dst)) || n > (1ull << 32) ||
      (degree > 1 && (src_stride < n || dst_stride < n)))
    return set_error(STWO_B200_E_INVALID, "bad batch_inverse arguments");
  if (n == 0) return STWO_B200_OK;
  std::lock_guard<std::mutex> g(ctx->ctx.small_mu);
  uint32_t* flag = ctx->ctx.small;
  cudaStream_t s = st(stream);
  cudaError_t e = cudaMemsetAsync(flag, 0, 4, s);
  if (e == cudaSuccess) e = sb::batch_inverse(degree, n, src, src_stride, dst, dst_stride, flag, s);
  uint32_t host = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&host, flag, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "batch_inverse");
  if (host) return set_error(STWO_B200_E_DIVISION_BY_ZERO, "batch_inverse: zero element");
  return STWO_B200_OK;
}

int32_t stwo_b200_logup_interaction(stwo_b200_context* ctx, uint32_t log_rows, uint32_t n_uses,
                                    const stwo_b200_logup_use* uses, const stwo_b200_qm31* alphas,
                                    stwo_b200_qm31 z, uint32_t batch, uint32_t order, uint32_t* out,
                                    uint64_t out_stride, stwo_b200_qm31* claimed_host, void* stream) {
  CK_CTX(ctx);
  if (log_rows > 28 || n_uses == 0 || n_uses > STWO_B200_LOGUP_MAX_USES || !uses || !out || !claimed_host ||
      (batch != 1 && batch != 2) || order > 1 || out_stride < (1ull << log_rows))
    return set_error(STWO_B200_E_INVALID, "bad logup_interaction arguments");
  sb::LogupParams p{};
  p.log_rows = log_rows;
  p.n_uses = n_uses;
  p.batch = batch;
  p.order = order;
  p.z = q(z);
  uint32_t max_words = 0;
  for (uint32_t u = 0; u < n_uses; ++u) {
    const stwo_b200_logup_use& in = uses[u];
    if (in.n_words == 0 || in.n_words > STWO_B200_LOGUP_MAX_WORDS)
      return set_error(STWO_B200_E_INVALID, "logup use with 0 or more than 8 words");
    max_words = std::max(max_words, in.n_words);
    sb::LogupUse& o = p.uses[u];
    o.n_words = in.n_words;
    o.negate = in.negate != 0;
    for (uint32_t j = 0; j < in.n_words; ++j) {
      o.words[j] = in.words[j];
      o.constants[j] = in.constants[j];
      if (!in.words[j] && in.constants[j] >= sb::P) return set_error(STWO_B200_E_INVALID, "non-canonical constant");
    }
    o.multiplicity = in.multiplicity;
  }
  if (!alphas) return set_error(STWO_B200_E_INVALID, "null alphas");
  for (uint32_t j = 0; j < max_words; ++j) p.alphas[j] = q(alphas[j]);
  cudaStream_t s = st(stream);
  size_t nscratch = sb::logup_scratch_count(log_rows) + 1;  // block sums + claimed
  void* scratch = nullptr;
  cudaError_t e = cudaMallocAsync(&scratch, nscratch * sizeof(sb::QM31), s);
  if (e != cudaSuccess) return cuda_status(e, "logup scratch");
  sb::QM31* claimed_dev = static_cast<sb::QM31*>(scratch);
  std::lock_guard<std::mutex> g(ctx->ctx.small_mu);
  uint32_t* flag = ctx->ctx.small;
  e = cudaMemsetAsync(flag, 0, 4, s);
  if (e == cudaSuccess) e = sb::logup_interaction(p, out, out_stride, claimed_dev, claimed_dev + 1, flag, s);
  uint32_t host[5] = {0, 0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, claimed_dev, 16, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host + 4, flag, 4, cudaMemcpyDeviceToHost, s);
  cudaError_t e2 = cudaFreeAsync(scratch, s);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "logup_interaction");
  if (host[4]) return set_error(STWO_B200_E_DIVISION_BY_ZERO, "logup_interaction: zero denominator");
  *claimed_host = stwo_b200_qm31{host[0], host[1], host[2], host[3]};
  return STWO_B200_OK;
}

}  // extern "C"
