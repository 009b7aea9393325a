// Launch interface of the device kernels. Every launcher enqueues on `stream`
// and returns the launch status; none synchronizes.
//
// Column sets are (base, stride) pairs: column c starts at base + c * stride
// (the reference CPU backend's column view, src/backends/cpu_scalar/mod.zig:185-197).
// Columns hold canonical M31 words in bit-reversed circle-domain order.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "circle.cuh"
#include "field.cuh"

namespace sb {

// Launch counter behind stwo_b200_telemetry_snapshot (the Metal backend's dispatch
// telemetry, src/backends/metal/telemetry.zig:49-336).
void note_launch();
uint64_t launch_count();

// Per-device read-only tables.
struct DeviceTables {
  PointM* points = nullptr;    // point table (circle.cuh)
  uint32_t* tw = nullptr;      // forward twiddle tower
  uint32_t* itw = nullptr;     // inverse twiddle tower
  // Both towers doubled (2t as an integer below 2^32), for the radix-16 butterflies (fft16.cuh);
  // they live in the second halves of the tw / itw allocations.
  uint32_t* tw2 = nullptr;
  uint32_t* itw2 = nullptr;
  uint32_t tower_log = 0;      // R: root half coset halfOdds(R)
  uint32_t sm_count = 148;     // multiprocessors of the device (persistent grid sizes)
  TwiddleView view(uint32_t domain_log, bool inverse) const;
};

// Builds the twiddle towers for root log R on the device (one-time).
cudaError_t build_twiddle_tower(DeviceTables& t, uint32_t root_log, cudaStream_t stream);

// ---- Circle FFT (src/prover/poly/circle/transforms.zig) -------------------
// In-place forward (evaluate) or inverse (interpolate, scaled by 1/n) transform
// of n_cols columns on CanonicCoset(log_size).
cudaError_t fft_columns(const DeviceTables& t, bool inverse, uint32_t log_size, uint32_t n_cols,
                        uint32_t* cols, uint64_t stride, cudaStream_t stream);
// Evaluations on CanonicCoset(log_size) -> coefficients (written to `coeffs`)
// and their evaluations on CanonicCoset(log_size + log_blowup) (written to `lde`).
// `evals` may alias `coeffs`. `coeffs` may be null when the caller only needs `lde`
// (then `scratch` of n_cols * 2^log_size words must be given).
cudaError_t interpolate_extend(const DeviceTables& t, uint32_t log_size, uint32_t log_blowup,
                               uint32_t n_cols, const uint32_t* evals, uint64_t ev_stride,
                               uint32_t* coeffs, uint64_t co_stride, uint32_t* lde,
                               uint64_t lde_stride, cudaStream_t stream);
// Coefficients (2^log_size) -> evaluations on CanonicCoset(log_size + log_blowup).
cudaError_t extend(const DeviceTables& t, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                   const uint32_t* coeffs, uint64_t co_stride, uint32_t* lde, uint64_t lde_stride,
                   cudaStream_t stream);

// ---- Lifted Blake2s Merkle (src/prover/vcs_lifted/leaves.zig, layers.zig) --
// Leaves of n_cols equal-size columns (2^log_size rows) plus all node layers.
// `layers` holds 2^(log_size+1) - 1 hashes: leaves first (2^log_size), then
// each parent layer, the root last. n_cols == 0 gives the empty-tree root.
cudaError_t merkle_commit(uint32_t log_size, uint32_t n_cols, const uint32_t* cols, uint64_t stride,
                          uint8_t* layers, cudaStream_t stream);
// Leaves of columns with mixed log sizes (lifted), columns in leaf order
// (stably sorted by log size ascending), pointers and logs in device memory;
// at most 2048 columns, each of log size >= 1 unless max_log is 0.
cudaError_t merkle_commit_lifted(uint32_t max_log, uint32_t n_cols, const uint32_t* const* col_ptrs,
                                 const uint32_t* col_logs, uint8_t* layers, cudaStream_t stream);
SB_HD uint64_t merkle_layer_offset(uint32_t max_log, uint32_t layer_log) {
  // layer with 2^layer_log nodes starts after the larger layers
  return (1ull << (max_log + 1)) - (1ull << (layer_log + 1));
}

// ---- Lifted accumulation (DomainEvaluationAccumulator, src/prover/air/accumulation.zig:256-347):
// dst (4 coordinate columns of 2^dst_log) += coeff * src (4 coordinate columns of 2^src_log) lifted.
cudaError_t accumulate_lifted(uint32_t dst_log, uint32_t* dst, uint64_t dst_stride, uint32_t src_log,
                              const uint32_t* src, uint64_t src_stride, QM31 coeff, cudaStream_t stream);

// ---- Wide-Fibonacci composition (src/examples/wide_fibonacci/component.zig:138-236)
// out: 4 coordinate columns of 2^(log_n+1). `eval` holds the W trace columns on
// CanonicCoset(log_n + 1). `coeffs` has W-2 QM31 (constraint k uses coeffs[k]).
cudaError_t wide_fib_composition(uint32_t log_n, uint32_t W, const uint32_t* eval, uint64_t stride,
                                 const QM31* coeffs_dev, uint32_t den_inv0, uint32_t den_inv1,
                                 uint32_t* out, uint64_t out_stride, cudaStream_t stream);

// ---- OODS evaluation of coefficient columns at a QM31 point ---------------
// partial: scratch of n_cols * ceil(2^log_size / 4096) QM31; out: n_cols QM31 (device).
cudaError_t eval_at_point(const DeviceTables& t, uint32_t log_size, uint32_t n_cols, const uint32_t* coeffs,
                          uint64_t stride, PointQ p, QM31* factors_dev, QM31* partial, QM31* out,
                          cudaStream_t stream);
// Whether eval_at_point may run on these columns: with 2^log_size >= 16 each thread reads 16
// coefficients as 16-byte vectors, so the base must be 16-byte aligned and the stride a multiple of 4.
inline bool eval_at_point_aligned(uint32_t log_size, uint32_t n_cols, const uint32_t* coeffs, uint64_t stride) {
  if (log_size < 4) return true;
  return (reinterpret_cast<uintptr_t>(coeffs) & 15) == 0 && (n_cols <= 1 || stride % 4 == 0);
}
size_t eval_at_point_partial_count(uint32_t log_size, uint32_t n_cols);
// Columns of one eval_at_point call: one grid row each (the grid's y extent).
constexpr uint32_t EVAL_AT_POINT_MAX_COLS = 65535;

// ---- DEEP quotients (src/core/pcs/quotients/row_evaluation.zig) -----------
struct QuotientBatchDev {
  PointQ point;          // sample point
  QM31 sum_a, sum_b;     // batch linear term
  uint32_t first, count; // range in the column/coefficient lists
};
// Single-size quotient: all columns have log size `log_size` (the lifting size).
// col_ptrs/coeff_c are device arrays of length n_entries; batches device array.
// `status` (device word, may be null): a caller that passes one vouches that every column pointer is
// 16-byte aligned, which makes the bulk-staged kernel one of the tuned variants; that kernel ORs
// QUOT_STATUS_* bits into it when a staged load runs out of time or the batches do not fit its
// item table, and its output is then not valid.
constexpr uint32_t QUOT_STATUS_TIMEOUT = 2, QUOT_STATUS_LAYOUT = 4;
cudaError_t accumulate_quotients(const DeviceTables& t, uint32_t log_size, uint32_t n_batches, uint32_t n_entries,
                                 const QuotientBatchDev* batches, const uint32_t* const* col_ptrs,
                                 const QM31* coeff_c, uint32_t* out, uint64_t out_stride,
                                 cudaStream_t stream, uint32_t* status = nullptr);
// Test hook: the next bulk-staged quotient launch leaves its first stage empty in every CTA, so that
// its bounded waits run out (status QUOT_STATUS_TIMEOUT).
void arm_quotient_stage_timeout_for_testing();

// ---- FRI folds (src/core/fri/folding.zig:352-602) --------------------------
cudaError_t fold_circle_into_line(const DeviceTables& t, uint32_t src_log, const uint32_t* src,
                                  uint64_t src_stride, QM31 alpha, uint32_t* dst, uint64_t dst_stride,
                                  bool accumulate, cudaStream_t stream);
// Line domain of the source: halfOdds(first_line_log) doubled (first_line_log - src_log) times.
cudaError_t fold_line(const DeviceTables& t, uint32_t src_log, const uint32_t* src, uint64_t src_stride,
                      QM31 alpha, uint32_t* dst, uint64_t dst_stride, cudaStream_t stream);

// FRI fold (circle -> line when `circle`, else line -> line with the source line
// domain halfOdds(src_log)) fused with the commitment of the folded layer: when
// `layers` is non-null the folded values are hashed as leaves (4 words each) and
// the whole tree of 2^(src_log-1) leaves is built. `alpha` is device memory (written
// by fri_channel_step earlier on the same stream).
cudaError_t fri_fold_commit(const DeviceTables& t, bool circle, uint32_t src_log, const uint32_t* src,
                            uint64_t src_stride, const QM31* alpha, uint32_t* dst, uint64_t dst_stride,
                            uint8_t* layers, cudaStream_t stream);

// Blake2s Fiat-Shamir channel state on the device for the FRI commit phase
// (src/prover/fri.zig:314-592: per layer mixRoot, then drawSecureFelt for its alpha), so
// the layers follow one another without a host round trip. The host uploads its channel
// state first and replays the same steps from `roots` afterwards.
constexpr uint32_t FRI_MAX_LAYERS = 32;
struct FriChannelDev {
  uint32_t digest[8];
  uint32_t n_draws;
  uint32_t status;  // nonzero: a draw was rejected FRI_DRAW_TRIES times in a row
  uint32_t quot_status;  // QUOT_STATUS_* of the proof's quotient launch (cleared before it)
  uint32_t pad;
  QM31 alpha[FRI_MAX_LAYERS];
  uint32_t roots[FRI_MAX_LAYERS][8];
};
// mixRoot(root) (src/core/vcs_lifted/blake2_merkle.zig:236-247), then drawSecureFelt
// (src/core/channel/blake2s.zig:52-112,260-279) into alpha[slot]; the root is kept in roots[slot].
cudaError_t fri_channel_step(FriChannelDev* c, const uint8_t* root, uint32_t slot, cudaStream_t stream);
// The inner FRI layers from line layer fri_tail_first(L, n_inner) on (at most 2^12 values each) in one
// CTA: per layer the channel step, the fold and the next layer's commitment, in the order and with
// the outputs of fri_channel_step + fri_fold_commit. line[k]: line layer k (4 coordinate columns of
// 2^(L-1-k)); trees[k]: its tree; line[n_inner] receives the last layer.
uint32_t fri_tail_first(uint32_t L, uint32_t n_inner);
cudaError_t fri_tail(const DeviceTables& t, FriChannelDev* c, uint32_t L, uint32_t k0, uint32_t n_inner,
                     uint32_t* const* line, uint8_t* const* trees, cudaStream_t stream);

// ---- Proof of work (src/core/channel/blake2s.zig:135-240) ------------------
// Bounded rounds of the same search (the form the prover uses, so the grind
// never holds every SM slot for the whole search): result_dev[0..1] must start
// at ~0; round r covers nonces [base, base + pow_round_nonces(sm_count)).
uint64_t pow_round_nonces(int sm_count);
cudaError_t pow_round(const uint32_t prefix_words[8], uint32_t n_bits, uint64_t base, uint32_t* result_dev,
                      int sm_count, cudaStream_t stream);

// ---- Trace generation (src/examples/wide_fibonacci/trace.zig:34-162) -------
// Seven-word quadratic recurrence (row seeds r0 + r1 k, r2 + r3 k; next = r4 a^2 + r5 b^2 + r6).
cudaError_t quadratic_trace(uint32_t log_n, uint32_t W, const uint32_t recipe[7], uint32_t* out, uint64_t stride,
                            cudaStream_t stream);
cudaError_t wide_fib_trace(uint32_t log_n, uint32_t W, int kind, uint64_t seed, uint32_t* out,
                           uint64_t stride, cudaStream_t stream);

// ---- Gathers for decommitment ----------------------------------------------
struct GatherItem {
  const uint32_t* src;  // word source (device)
  uint64_t index;       // word index
};
cudaError_t gather_words(const GatherItem* items, uint32_t n, uint32_t* out, cudaStream_t stream);
struct HashGatherItem {
  const uint8_t* layers;  // tree layer buffer
  uint64_t node;          // global node index in the buffer (hash units)
};
cudaError_t gather_hashes(const HashGatherItem* items, uint32_t n, uint8_t* out, cudaStream_t stream);

// ---- Batch inversion (src/core/fields/mod.zig:164-200) ---------------------
// Montgomery batch inverse of n elements of `degree` (1 M31, 2 CM31, 4 QM31)
// coordinate columns. Sets *zero_flag (device) to 1 when an element is zero.
// dst may alias src.
cudaError_t batch_inverse(uint32_t degree, uint64_t n, const uint32_t* src, uint64_t src_stride, uint32_t* dst,
                          uint64_t dst_stride, uint32_t* zero_flag, cudaStream_t stream);

// ---- LogUp interaction columns (a20) ---------------------------------------
// One use of a relation: denominator = sum_j alphas[j] * word_j(row) - z,
// numerator = +/- multiplicity(row) (relation_combine / relation_multiplicity,
// src/backends/metal/shaders/core/relation.metal:54-90).
constexpr uint32_t LOGUP_MAX_WORDS = 8;
constexpr uint32_t LOGUP_MAX_USES = 32;
struct LogupUse {
  uint32_t n_words;
  uint32_t negate;
  const uint32_t* words[LOGUP_MAX_WORDS];  // nullptr: constants[j]
  uint32_t constants[LOGUP_MAX_WORDS];
  const uint32_t* multiplicity;            // nullptr: 1
};
struct LogupParams {
  uint32_t log_rows;
  uint32_t n_uses;
  uint32_t batch;  // uses per interaction column: 1, or 2 (pairs n1 d2 + n2 d1 over d1 d2)
  uint32_t order;  // 0: cumulative sum in storage order; 1: coset order minus total/N per step
  QM31 alphas[LOGUP_MAX_WORDS];
  QM31 z;
  LogupUse uses[LOGUP_MAX_USES];
};
SB_HD uint32_t logup_n_cols(uint32_t n_uses, uint32_t batch) { return (n_uses + batch - 1) / batch; }
// Scratch entries (QM31) logup_interaction needs for 2^log_rows rows.
size_t logup_scratch_count(uint32_t log_rows);
// out: n_cols interaction columns of 4 coordinate columns each (column c, coordinate k at
// out + (4c + k) * out_stride). Column c holds, per row, the running sum over columns 0..c of
// the row's fractions; the last column is then scanned over rows. claimed (device QM31) gets
// the total. *zero_flag (device) is set to 1 when a denominator is zero.
cudaError_t logup_interaction(const LogupParams& p, uint32_t* out, uint64_t out_stride, QM31* claimed,
                              QM31* scratch, uint32_t* zero_flag, cudaStream_t stream);

// XOR-lookup trace of 2^log_n rows (3 columns a, b, a ^ b, stride 2^log_n; a, b seeded
// uniform u8), the 2^16-row XOR table (3 columns, row a * 256 + b) and the table-row
// multiplicities (65536 words).
cudaError_t xor_lookup_trace(uint32_t log_n, uint64_t seed, uint32_t* main_cols, uint32_t* table, uint32_t* mult,
                             cudaStream_t stream);

}  // namespace sb
