/*
 * stwo_b200: C ABI of the B200 (sm_100a) backend for the stwo-zig circle-STARK
 * prover. A Zig backend type (or any FFI caller) binds these functions the way
 * src/backends/cuda/ffi.zig binds the stwo-cuda prototypes (an `extern fn`
 * per entry point, slices passed as pointer + length).
 *
 * Conventions
 *  - Every function returns int32_t status: 0 = STWO_B200_OK, negative = error.
 *    stwo_b200_last_error() returns a message for the calling thread's last error.
 *    (The stwo-cuda precedent returns void, src/backends/cuda/ffi.zig:43-70.)
 *  - M31 columns are uint32_t canonical values in bit-reversed circle-domain
 *    order. A column set is (base, stride): column c starts at base + c * stride
 *    (src/backends/cpu_scalar/mod.zig:185-197).
 *  - QM31 values are stwo_b200_qm31 {a, b, c, d} = (c0.a, c0.b, c1.a, c1.b),
 *    the layout of CudaQM31 (src/backends/cuda/ffi.zig:12-21).
 *  - Secure (QM31) columns are 4 coordinate columns (SecureColumnByCoords,
 *    src/backend/secure_column.zig).
 *  - Hashes are 32 bytes. Merkle layer buffers hold 2^(L+1)-1 hashes: the 2^L
 *    leaves first, then each parent layer, the root last.
 *  - Op-level functions take DEVICE pointers and a cudaStream_t (as void*); they
 *    enqueue work and return without synchronizing unless stated.
 *  - Handles are released only by their *_destroy function; no function frees
 *    caller buffers (ownership rules of src/prover/engine.zig:28-31).
 */
#ifndef STWO_B200_H
#define STWO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STWO_B200_OK 0
#define STWO_B200_E_INVALID (-1)
#define STWO_B200_E_OOM (-2)
#define STWO_B200_E_CUDA (-3)
#define STWO_B200_E_TIMEOUT (-4)
#define STWO_B200_E_CONSTRAINTS (-5)
#define STWO_B200_E_BUFFER_TOO_SMALL (-6)
#define STWO_B200_E_FALLBACK (-7)
#define STWO_B200_E_NO_DEVICE (-8)
#define STWO_B200_E_DIVISION_BY_ZERO (-9) /* Error.DivisionByZero / ZeroDenominator of the reference */
#define STWO_B200_E_REJECTED (-10)         /* admission refused (CommittedCellBudgetExceeded, memory budget) */

typedef struct stwo_b200_context stwo_b200_context;

typedef struct {
  uint32_t a, b, c, d;
} stwo_b200_qm31;

/* PcsConfig (src/core/pcs/mod.zig:23-52) with FriConfig fold_step 1 and no lifting override. */
typedef struct {
  uint32_t pow_bits;
  uint32_t log_blowup_factor;
  uint32_t log_last_layer_degree_bound;
  uint32_t n_queries;
} stwo_b200_pcs_config;

/* Wide-Fibonacci proving request: the Statement (src/examples/wide_fibonacci/trace.zig:18-21)
 * plus the prepared trace. Exactly one trace source is used, in this order: trace_device,
 * trace_host, generated (trace_kind 0 = the reference's (1, row) seeds, 1 = seeded uniform
 * col0/col1 in [0, p-1)). With trace_kind 2 (STWO_B200_TRACE_FIRST_COLUMNS) trace_device or
 * trace_host holds only col0 then col1 (2 x 2^log_n_rows canonical words, bit-reversed circle
 * order) and the device derives col_k = col_{k-2}^2 + col_{k-1}^2: the deferred quadratic-
 * recurrence column source the Metal backend materialises on the device
 * (src/examples/wide_fibonacci/trace.zig:221-265, materializeColumnSource at
 * src/prover/pcs/scheme.zig:271-278). has_channel_seed mixes channel_seed (mixU64) right after
 * the statement; 0 keeps the reference transcript. */
#define STWO_B200_TRACE_REFERENCE 0
#define STWO_B200_TRACE_SEEDED 1
#define STWO_B200_TRACE_FIRST_COLUMNS 2
typedef struct {
  uint32_t log_n_rows;
  uint32_t sequence_len;
  stwo_b200_pcs_config config;
  const uint32_t* trace_host;
  const uint32_t* trace_device;
  uint32_t trace_kind;
  uint32_t has_channel_seed;
  uint64_t trace_seed;
  uint64_t channel_seed;
} stwo_b200_wide_fib_request;

/* Device time per proving stage, in milliseconds; host_encode is the host time after the last device
 * stage (JSON wire encoding and the OODS self-check); host_gaps the host time between the transcript's
 * stream synchronizations and the next device work (for a proof that runs alone, the device idles
 * then: total - host_gaps bounds the proof's device work). */
typedef struct {
  float upload, trace, main_commit, composition, composition_commit, oods, quotients, fri, pow, decommit, total;
  float host_encode, host_gaps;
} stwo_b200_stage_times;

/* Device pointers: Merkle layer buffers must be 16-byte aligned, FRI fold sources 8-byte aligned with
 * an even stride, OODS coefficient columns (2^log_size >= 16) 16-byte aligned with a stride that is a
 * multiple of 4; other pointers need the alignment of their element type. Calls that break this
 * return STWO_B200_E_INVALID without launching anything. */

/* ---- Runtime --------------------------------------------------------------------------------- */

/* Creates a context on `device`: point tables and twiddle towers for domains up to 2^23
 * (M31TwiddleTower, src/prover/poly/twiddle_tower.zig:29-81; Metal initializeRuntime,
 * src/backends/metal/commit_backend.zig). */
int32_t stwo_b200_context_create(int32_t device, stwo_b200_context** out);
int32_t stwo_b200_context_destroy(stwo_b200_context* ctx);
const char* stwo_b200_last_error(void);
const char* stwo_b200_status_string(int32_t status);
/* Library version string (build identity). */
const char* stwo_b200_version(void);

/* Process-wide counters (Metal's telemetrySnapshot / TelemetrySnapshot,
 * src/backends/metal/telemetry.zig:49-336): kernels launched by this library. */
typedef struct {
  uint64_t kernel_launches;
} stwo_b200_telemetry;
int32_t stwo_b200_telemetry_snapshot(stwo_b200_telemetry* out);

/* ---- Engine level ------------------------------------------------------------------------------ */

/* One proof; writes the JSON wire bytes (src/interop/proof_wire.zig:19-77). Replaces
 * ProverEngine(B,...).prove for the wide-Fibonacci AIR (src/prover/engine.zig:163-181 via
 * src/examples/wide_fibonacci.zig:200-220 provePreparedWithEngine). If `proof_cap` is too small
 * the call returns STWO_B200_E_BUFFER_TOO_SMALL with *proof_len set. `times` may be NULL. */
int32_t stwo_b200_prove_wide_fibonacci(stwo_b200_context* ctx, const stwo_b200_wide_fib_request* req,
                                       uint8_t* proof_out, size_t proof_cap, size_t* proof_len,
                                       stwo_b200_stage_times* times);

/* Batched proving: n independent requests, up to `max_in_flight` proofs resident and
 * overlapping on the device (one stream and workspace each). statuses[i], proof_lens[i] and
 * times[i] (nullable array) are per request; the call returns STWO_B200_OK when every request
 * succeeded. No reference counterpart: the reference proves one statement per call. */
int32_t stwo_b200_prove_wide_fibonacci_batch(stwo_b200_context* ctx, const stwo_b200_wide_fib_request* reqs,
                                             size_t n, uint8_t* const* proof_outs, const size_t* proof_caps,
                                             size_t* proof_lens, int32_t* statuses, uint32_t max_in_flight,
                                             stwo_b200_stage_times* times);

/* LogUp XOR-lookup AIR request: 2^log_n lookups of seeded w-bit operand pairs (w = log_table / 2;
 * log_table 16 for u8 pairs, 8 for 4-bit pairs) into the 2^log_table-row XOR table. No reference
 * AIR exists; the proof uses the reference's lifted PCS, FRI, channel and wire layout, with the
 * lookups (2^log_n rows) and the table (2^log_table rows) at their own sizes, four trees
 * (preprocessed table at its size; main trace and multiplicities, LogUp interaction: lifted trees
 * over both sizes; composition) and the two LogUp claimed sums, which the verifier requires to
 * cancel. */
typedef struct {
  uint32_t log_n;
  uint32_t log_table;
  stwo_b200_pcs_config config;
  uint64_t seed;
  uint32_t has_channel_seed;
  uint32_t reserved;
  uint64_t channel_seed;
} stwo_b200_xor_request;

/* Proves the LogUp XOR-lookup AIR; proof bytes as for stwo_b200_prove_wide_fibonacci. */
int32_t stwo_b200_prove_logup_xor(stwo_b200_context* ctx, const stwo_b200_xor_request* req, uint8_t* proof_out,
                                  size_t proof_cap, size_t* proof_len);

/* ---- Verifier (host) ------------------------------------------------------------------------------ */

/* Verifies a proof from its bytes on the calling host thread (no device use): the reference verifier
 * (src/examples/wide_fibonacci.zig:360-433, src/core/verifier.zig, src/core/pcs/verifier.zig,
 * src/core/fri.zig, src/core/vcs_lifted/verifier.zig). STWO_B200_OK, or STWO_B200_E_CONSTRAINTS with
 * the failed check in stwo_b200_last_error(). has_channel_seed mirrors the prover's optional mix. */
int32_t stwo_b200_verify_wide_fibonacci(const uint8_t* proof, size_t proof_len, uint32_t log_n_rows,
                                        uint32_t sequence_len, uint32_t has_channel_seed, uint64_t channel_seed);
/* The same for LogUp XOR-lookup AIR proofs (additionally: the claimed sums cancel). */
int32_t stwo_b200_verify_logup_xor(const uint8_t* proof, size_t proof_len, uint32_t log_n, uint32_t log_table,
                                   uint32_t has_channel_seed, uint64_t channel_seed);

/* ---- Serving loop ------------------------------------------------------------------------------- */

/* Continuous batching of wide-Fibonacci proofs on one device: `slots` proofs in flight (each a host
 * thread and a stream), admitted first-in first-out as a slot is free and the in-flight device
 * workspace stays within memory_budget bytes (0 = 80% of the device memory free at creation). Each
 * request must also pass the reference's resource-profile admission (profile 0 standard, 1 large,
 * 2 extreme; 16 accounted bytes per committed cell, src/prover/native/resource_admission.zig:5-19,
 * :147-161), else submit returns STWO_B200_E_REJECTED. Proof bytes equal those of
 * stwo_b200_prove_wide_fibonacci for the same request. The reference has no serving loop; the
 * admission limits are its resource profiles. */
typedef struct stwo_b200_server stwo_b200_server;
#define STWO_B200_SERVER_VERIFY 2u /* every proof is verified on its slot's host thread before it is returned */
#define STWO_B200_SERVER_PERSISTENT_WORKSPACES 1u /* slots keep their workspace between proofs (counted
                                                  * against the budget while held) instead of taking it
                                                  * from the stream-ordered pool per proof */
typedef struct {
  uint32_t slots;
  uint32_t profile;
  uint64_t memory_budget;
  uint32_t flags;
} stwo_b200_server_config;
typedef struct {
  uint64_t accounted_bytes; /* 16 B per committed cell */
  uint64_t workspace_bytes; /* device workspace the proof used */
  double queued_ms;         /* submit -> admitted (host steady clock) */
  double run_ms;            /* admitted -> proof bytes */
  uint32_t slot;
  stwo_b200_stage_times stages;
} stwo_b200_request_stats;
typedef struct {
  uint64_t submitted, completed, failed, rejected;
  uint64_t peak_in_flight, peak_workspace_bytes, budget_bytes;
} stwo_b200_server_snapshot;

int32_t stwo_b200_server_create(stwo_b200_context* ctx, const stwo_b200_server_config* cfg,
                                stwo_b200_server** out);
/* Queues a request and returns at once; host/device trace buffers must stay valid until wait returns. */
int32_t stwo_b200_server_submit(stwo_b200_server* server, const stwo_b200_wide_fib_request* req, uint64_t* ticket);
/* Queues a LogUp XOR-lookup AIR request (committed cells: 16 columns of 2^max(log_n, log_table) rows). */
int32_t stwo_b200_server_submit_xor(stwo_b200_server* server, const stwo_b200_xor_request* req, uint64_t* ticket);
/* Blocks until the request is done and returns its status; STWO_B200_E_BUFFER_TOO_SMALL sets
 * *proof_len and keeps the result for another call. */
int32_t stwo_b200_server_wait(stwo_b200_server* server, uint64_t ticket, uint8_t* proof_out, size_t proof_cap,
                              size_t* proof_len, stwo_b200_request_stats* stats);
/* Sizes every slot for the largest shapes it will serve (the reference's warmup / initializeRuntime
 * hooks, src/prover/engine.zig): persistent workspaces grow to 2^max_log_n_rows x max_sequence_len
 * (within the memory budget), and the stream-ordered pool is pre-grown for transient workspaces and
 * XOR-lookup proofs of up to 2^max_xor_log_n rows (0: none), whose provers' page-locked staging is
 * allocated now. Call while the server is idle. */
int32_t stwo_b200_server_warmup(stwo_b200_server* server, uint32_t max_log_n_rows, uint32_t max_sequence_len,
                                uint32_t log_blowup, uint32_t max_xor_log_n);
int32_t stwo_b200_server_snapshot_get(stwo_b200_server* server, stwo_b200_server_snapshot* out);
/* Time limit of every request submitted from now on, counted from its submission (0: none, the
 * default). A request still queued at its deadline ends with STWO_B200_E_TIMEOUT without running; a
 * running proof checks it between stages and between proof-of-work rounds and ends with
 * STWO_B200_E_TIMEOUT, its slot free for the next request. The reference has no serving loop; its
 * provers run to completion. */
int32_t stwo_b200_server_set_request_timeout(stwo_b200_server* server, uint32_t timeout_ms);
/* Finishes every queued and running request, then releases the slots. */
int32_t stwo_b200_server_destroy(stwo_b200_server* server);

/* ---- PolyOps (src/backend/poly_ops.zig:12-24) --------------------------------------------------- */

/* In-place interpolation (evaluations -> coefficients) of n_cols columns on CanonicCoset(log_size).
 * Replaces interpolateCircleBuffers (src/prover/pcs/columns/circle_transforms.zig:212) and
 * ntt_b2n_column (src/backends/cuda/ffi.zig:52). */
int32_t stwo_b200_interpolate_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, uint32_t* cols,
                                      uint64_t stride, void* stream);
/* In-place evaluation (coefficients -> evaluations) on CanonicCoset(log_size). Replaces
 * evaluateCircleBuffers (circle_transforms.zig:248) and ntt_n2b_columns (ffi.zig:51). */
int32_t stwo_b200_evaluate_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, uint32_t* cols,
                                   uint64_t stride, void* stream);
/* Evaluations on CanonicCoset(log_size) -> coefficients and evaluations on
 * CanonicCoset(log_size + log_blowup), fused. Replaces interpolateAndEvaluateCircleBuffers
 * (src/backends/cpu_scalar/mod.zig:185-266, src/prover/pcs/columns/preparation.zig:212-352). */
int32_t stwo_b200_interpolate_and_extend(stwo_b200_context* ctx, uint32_t log_size, uint32_t log_blowup,
                                         uint32_t n_cols, const uint32_t* evals, uint64_t evals_stride,
                                         uint32_t* coeffs, uint64_t coeffs_stride, uint32_t* lde,
                                         uint64_t lde_stride, void* stream);
/* Coefficients -> evaluations on CanonicCoset(log_size + log_blowup) (evaluateExtensionBufferWithTwiddles,
 * src/prover/poly/circle/transforms.zig:132-147; extendCoefficientColumnsByGroupForBackend,
 * src/prover/pcs/commit_polys.zig:33). */
int32_t stwo_b200_extend_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                                 const uint32_t* coeffs, uint64_t coeffs_stride, uint32_t* lde, uint64_t lde_stride,
                                 void* stream);
/* Value of each coefficient column at a QM31 circle point (CircleCoefficients.evalAtPoint,
 * src/prover/poly/circle/poly.zig:62-230; evaluateCoefficientPlans hook,
 * src/prover/pcs/sampled_values.zig:68; eval_at_point / batch_eval_at_points, ffi.zig:55,:89).
 * out_dev: n_cols QM31 on the device, n_cols <= STWO_B200_EVAL_AT_POINT_MAX_COLS. Allocates its
 * scratch from the stream's pool (STWO_B200_E_OOM when that fails). */
#define STWO_B200_EVAL_AT_POINT_MAX_COLS 65535
int32_t stwo_b200_eval_at_point(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, const uint32_t* coeffs,
                                uint64_t stride, stwo_b200_qm31 px, stwo_b200_qm31 py, stwo_b200_qm31* out_dev,
                                void* stream);

/* Same result as stwo_b200_eval_at_point, but it allocates nothing: no reference counterpart (the
 * reference evaluates on the host). For callers that cannot allocate device memory when they need
 * this value, e.g. a serving loop bound to an admitted device-memory budget, an embedder whose arena
 * owns all device memory, or code where CUDA allocation calls are not allowed. The per-chunk partial
 * sums live in one fixed device array of STWO_B200_NOALLOC_EVAL_SCRATCH 16-byte entries (1 MiB, kept
 * on every GPU that loads the library until exit): n_cols * max(1, 2^(log_size-12)) must not exceed
 * it, and n_cols must not exceed STWO_B200_EVAL_AT_POINT_MAX_COLS, else STWO_B200_E_INVALID. All
 * calls on a device share the array, so calls whose work overlaps on the GPU race: serialize them.
 * The first call on each device looks up the array's address; make it before any stream capture.
 * The address is cached for the process: do not call this again after resetting the device. */
#define STWO_B200_NOALLOC_EVAL_SCRATCH 65536
int32_t stwo_b200_eval_at_point_noalloc(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols,
                                        const uint32_t* coeffs, uint64_t stride, stwo_b200_qm31 px,
                                        stwo_b200_qm31 py, stwo_b200_qm31* out_dev, void* stream);

/* ---- MerkleOps (src/backend/merkle_ops.zig:20-56) ------------------------------------------------ */

/* Blake2s lifted Merkle commitment of n_cols columns of 2^log_size rows ("leaf"/"node" prefixed
 * hasher, src/core/vcs_lifted/blake2_merkle.zig). layers_dev: 2^(log_size+1)-1 hashes. root_host
 * (nullable) receives the root after the stream synchronizes. Replaces commitMerkle
 * (merkle_ops.zig:20-56, src/prover/vcs_lifted/prover.zig:61-70) and commit_on_first_layer_in_gpu /
 * commit_on_layer_in_gpu (ffi.zig:69-70). */
int32_t stwo_b200_merkle_commit(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols, const uint32_t* cols,
                                uint64_t stride, uint8_t* layers_dev, uint8_t* root_host, void* stream);

/* Lifted Blake2s Merkle commitment of columns of mixed log sizes (the interaction and preprocessed
 * trees of AIRs with several component sizes). cols: host array of n_cols device column pointers,
 * log_sizes: host array of their log sizes (each >= 1 unless all are 0; at most 2048 columns).
 * Columns are hashed in the reference's leaf order, stably sorted by log size ascending, each at its
 * lifted index ((pos >> (max_log - log + 1)) << 1) + (pos & 1) (src/prover/vcs_lifted/leaves.zig:
 * 104-115, decommit.zig:88). layers_dev: 2^(max_log+1)-1 hashes, leaves first. Synchronous when
 * root_host is set. Replaces commitMerkle for mixed-size column sets (merkle_ops.zig:20-56). */
int32_t stwo_b200_merkle_commit_lifted(stwo_b200_context* ctx, uint32_t n_cols, const uint32_t* const* cols,
                                       const uint32_t* log_sizes, uint8_t* layers_dev, uint8_t* root_host,
                                       void* stream);

/* ---- FriOps (src/backend/fri_ops.zig:19-37) ------------------------------------------------------ */

/* dst = dst * alpha^2 + fold(src) when accumulate, else fold(src); src 4 coordinate columns of
 * 2^src_log on CanonicCoset(src_log), dst 4 columns of 2^(src_log-1). Replaces foldCircleIntoLine
 * (src/core/fri/folding.zig:558-602; fold_circle_into_line, ffi.zig:62). */
int32_t stwo_b200_fold_circle_into_line(stwo_b200_context* ctx, uint32_t src_log, const uint32_t* src,
                                        uint64_t src_stride, stwo_b200_qm31 alpha, uint32_t* dst,
                                        uint64_t dst_stride, int32_t accumulate, void* stream);
/* One fold of a line evaluation of 2^src_log on the line domain halfOdds(src_log) (the FRI
 * inner-layer tower). Replaces foldLine (folding.zig:352-384; fold_line, ffi.zig:61). */
int32_t stwo_b200_fold_line(stwo_b200_context* ctx, uint32_t src_log, const uint32_t* src, uint64_t src_stride,
                            stwo_b200_qm31 alpha, uint32_t* dst, uint64_t dst_stride, void* stream);

/* ---- QuotientOps (src/backend/quotient_ops.zig:10-16) ------------------------------------------- */

/* DEEP quotient of columns sampled at one point, on CanonicCoset(log_size) in bit-reversed order:
 * out(row) = (sum_i c_i v_i(row) - (sum_a y + sum_b)) / ((Re Px - x) Im Py - (Re Py - y) Im Px).
 * col_ptrs_dev: device array of n_cols device pointers; c_dev: n_cols QM31 line coefficients c
 * (random-coefficient scaled), sum_a / sum_b the batch's summed a and b line coefficients
 * (src/core/pcs/quotients/row_evaluation.zig:71-101,400-521). Replaces accumulateQuotients and
 * accumulate_quotients (ffi.zig:94). */
/* One FRI fold fused with the commitment of the folded layer (foldLineAndCommitNext and the first
 * layer's fold, src/prover/fri.zig:314-592; Metal foldLineAndCommitNext / commitFriLayers): circle != 0
 * folds a circle evaluation of 2^src_log values into a line (foldCircleIntoLine without accumulation),
 * else a line of 2^src_log values into its half (foldLine). src: 4 coordinate columns, 8-byte aligned,
 * even stride; dst: 4 columns of 2^(src_log-1). layers_dev (nullable: fold only) receives the folded
 * layer's Merkle tree (2^src_log - 1 hashes, leaf = the 4 coordinates); root_host (nullable) its root
 * after the stream synchronizes. */
int32_t stwo_b200_fold_and_commit(stwo_b200_context* ctx, int32_t circle, uint32_t src_log, const uint32_t* src,
                                  uint64_t src_stride, stwo_b200_qm31 alpha, uint32_t* dst, uint64_t dst_stride,
                                  uint8_t* layers_dev, uint8_t* root_host, void* stream);
/* Interpolate, extend by 2^log_blowup and commit the extension (prepareAndCommitPolys /
 * prepareAndCommitOwned, src/backends/metal/commit_backend.zig; src/prover/pcs/commit_polys.zig:10-67):
 * stwo_b200_interpolate_and_extend followed by stwo_b200_merkle_commit of the n_cols LDE columns. */
int32_t stwo_b200_commit_columns(stwo_b200_context* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                                 const uint32_t* evals, uint64_t evals_stride, uint32_t* coeffs, uint64_t coeffs_stride,
                                 uint32_t* lde, uint64_t lde_stride, uint8_t* layers_dev, uint8_t* root_host,
                                 void* stream);
/* The composition polynomial's interpolation, split and extension (interpolateSecureComposition,
 * src/prover/poly/circle/secure_poly.zig:77-105,164-226): comp holds the 4 coordinate columns of its
 * evaluations on CanonicCoset(comp_log) and receives their coefficients; lde receives 8 columns of
 * 2^(comp_log-1+log_blowup): the extensions of the 4 left halves (first 2^(comp_log-1) coefficients),
 * then of the 4 right halves. */
int32_t stwo_b200_interpolate_secure_composition(stwo_b200_context* ctx, uint32_t comp_log, uint32_t* comp,
                                                 uint64_t comp_stride, uint32_t log_blowup, uint32_t* lde,
                                                 uint64_t lde_stride, void* stream);
int32_t stwo_b200_accumulate_quotients(stwo_b200_context* ctx, uint32_t log_size, uint32_t n_cols,
                                       const uint32_t* const* col_ptrs_dev, const stwo_b200_qm31* c_dev,
                                       stwo_b200_qm31 px, stwo_b200_qm31 py, stwo_b200_qm31 sum_a,
                                       stwo_b200_qm31 sum_b, uint32_t* out, uint64_t out_stride, void* stream);

/* ---- AccumulationOps (src/backend/accumulation_ops.zig) -------------------------------------------- */

/* Lifted accumulation of secure columns: dst (4 coordinate columns of 2^dst_log, stride dst_stride)
 * += coeff * src (4 coordinate columns of 2^src_log <= 2^dst_log), where row i of dst reads src at
 * ((i >> (dst_log - src_log + 1)) << 1) + (i & 1), or at i for equal sizes: the accumulate hook and
 * DomainEvaluationAccumulator.accumulateColumn + finalize (src/prover/air/accumulation.zig:256-347,
 * liftedValueAt :336-347). Device pointers, async on `stream`. */
int32_t stwo_b200_accumulate(stwo_b200_context* ctx, uint32_t dst_log, uint32_t* dst, uint64_t dst_stride,
                             uint32_t src_log, const uint32_t* src, uint64_t src_stride, stwo_b200_qm31 coeff,
                             void* stream);

/* ---- Wide-Fibonacci AIR -------------------------------------------------------------------------- */

/* Trace generation in bit-reversed circle order (fillQuadraticRecurrenceTrace hook,
 * src/examples/wide_fibonacci/trace.zig:63-74; generate_wide_fibonacci_trace, ffi.zig:263).
 * trace_kind 2 derives columns 2.. from the col0/col1 already in `out`. */
int32_t stwo_b200_wide_fib_trace(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t sequence_len,
                                 uint32_t trace_kind, uint64_t seed, uint32_t* out, uint64_t stride, void* stream);
/* Trace of a seven-word quadratic recurrence in bit-reversed circle order (the
 * fillQuadraticRecurrenceTrace hook and its recipe ABI, src/examples/wide_fibonacci/trace.zig:13-16,
 * 63-74): for logical (coset-order) row k, col0 = r0 + r1 k, col1 = r2 + r3 k and
 * col_j = r4 col_{j-2}^2 + r5 col_{j-1}^2 + r6 in M31. The wide-Fibonacci recipe is
 * {1, 0, 0, 1, 1, 1, 0}. n_cols >= 2 columns of `stride` words at `out` (device). */
int32_t stwo_b200_quadratic_recurrence_trace(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t n_cols,
                                             const uint32_t recipe[7], uint32_t* out, uint64_t stride, void* stream);
/* Composition evaluation on CanonicCoset(log_n_rows+1): out (4 columns) = sum_k coeffs[k] *
 * (c_k - a_k^2 - b_k^2) * den_inv[row >> log_n_rows] (computeCompositionEvaluation hook,
 * src/prover/air/component_prover.zig:269; src/examples/wide_fibonacci/component.zig:138-236). */
int32_t stwo_b200_wide_fib_composition(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t sequence_len,
                                       const uint32_t* eval, uint64_t stride, const stwo_b200_qm31* coeffs_dev,
                                       uint32_t den_inv0, uint32_t den_inv1, uint32_t* out, uint64_t out_stride,
                                       void* stream);

/* ---- FieldOps (src/backend/field_ops.zig:9-15) -------------------------------------------------- */

/* Montgomery batch inverse of n elements of `degree` 1 (M31), 2 (CM31) or 4 (QM31); an element is
 * `degree` coordinate columns (column k at base + k * stride). dst may alias src. Synchronous: returns
 * STWO_B200_E_DIVISION_BY_ZERO when an element is zero, as batchInverse does (dst is then
 * unspecified). Replaces batchInverse (src/core/fields/mod.zig:164-200). */
int32_t stwo_b200_batch_inverse(stwo_b200_context* ctx, uint32_t degree, uint64_t n, const uint32_t* src,
                                uint64_t src_stride, uint32_t* dst, uint64_t dst_stride, void* stream);

/* ---- LogUp interaction columns ------------------------------------------------------------------- */

/* One use of a relation at every row: denominator = sum_j alphas[j] * word_j(row) - z, numerator =
 * multiplicity(row) (1 when NULL), negated when `negate`. words[j] is a device M31 column of
 * 2^log_rows rows, or NULL for the constant constants[j] (relation_combine / relation_multiplicity,
 * src/backends/metal/shaders/core/relation.metal:54-90). */
#define STWO_B200_LOGUP_MAX_WORDS 8
#define STWO_B200_LOGUP_MAX_USES 32
typedef struct {
  uint32_t n_words;
  uint32_t negate;
  const uint32_t* words[STWO_B200_LOGUP_MAX_WORDS];
  uint32_t constants[STWO_B200_LOGUP_MAX_WORDS];
  const uint32_t* multiplicity;
} stwo_b200_logup_use;

/* Interaction columns of n_uses uses (host array), `batch` (1 or 2) uses per column: a column of two
 * uses is (n_a d_b + n_b d_a) / (d_a d_b). Column c (4 coordinate columns at out + (4c + k) * out_stride)
 * holds per row the running sum of the row's fractions over columns 0..c; the last column is then the
 * cumulative sum over rows: order 1 visits rows in coset order (scan index s -> circle index s/2 or
 * N-1-s/2, stored at its bit reverse) and subtracts total (s+1)/N (relation.metal:160-237, law of
 * src/tests/metal/backend/commitment_test.zig:73-154); order 0 sums in storage order without shift
 * (cumulativeColumn, src/frontends/riscv/air/logup.zig:83-105). claimed_host receives the total.
 * alphas: host array of max n_words QM31. Synchronous; STWO_B200_E_DIVISION_BY_ZERO when a
 * denominator is zero. */
int32_t stwo_b200_logup_interaction(stwo_b200_context* ctx, uint32_t log_rows, uint32_t n_uses,
                                    const stwo_b200_logup_use* uses, const stwo_b200_qm31* alphas,
                                    stwo_b200_qm31 z, uint32_t batch, uint32_t order, uint32_t* out,
                                    uint64_t out_stride, stwo_b200_qm31* claimed_host, void* stream);

/* XOR-lookup trace for a LogUp lookup AIR (no reference AIR; the table follows the reference's
 * bitwise table, src/frontends/riscv/air/preprocessed/bitwise.zig:17-35): main_cols receives 3
 * columns of 2^log_n rows (a, b seeded uniform u8 - SplitMix64 of seed ^ (0xD6E8FEB86659FD93 *
 * (row + 1)), a = low byte, b = next byte - and a XOR b), table 3 columns of 65536 rows (row
 * a * 256 + b holds a, b, a XOR b), multiplicity 65536 words: how often each table row occurs. */
int32_t stwo_b200_xor_lookup_trace(stwo_b200_context* ctx, uint32_t log_n, uint64_t seed, uint32_t* main_cols,
                                   uint32_t* table, uint32_t* multiplicity, void* stream);

/* ---- Channel proof of work ---------------------------------------------------------------------- */

/* Lowest nonce whose Blake2s(prefix_digest || LE64 nonce) has >= n_bits trailing zero bits in its
 * first 16 bytes (src/core/channel/blake2s.zig:135-240). Synchronous. n_bits <= STWO_B200_MAX_POW_BITS,
 * the limit every prover applies to pow_bits too (the reference accepts any u32; a search of 2^n_bits
 * expected nonces holds the device for that long, about 40 s at 40 bits on one B200). */
#define STWO_B200_MAX_POW_BITS 40
int32_t stwo_b200_pow_grind(stwo_b200_context* ctx, const uint8_t prefix_digest[32], uint32_t n_bits,
                            uint64_t* nonce_out);

/* ---- Autotuner ----------------------------------------------------------------------------------- */

/* Launch-shape autotuner of the kernels that come in variants writing the same bits (op 0: the
 * interpolate + blow-up-2 high pass, fused or generic; op 1: the Merkle leaf kernel at 5, 6 or 4 CTAs
 * per SM; op 2: the DEEP quotient kernel at 6, 3 or 9 loads in flight, and, for callers whose
 * columns are 16-byte aligned (the provers, and the op-level call after it reads the column pointers
 * back), the bulk-staged kernel that streams column chunks into shared memory with bulk async
 * copies), keyed by (op, log_size, n_cols) for the process. A key's first call times every variant on its own inputs with CUDA events
 * and keeps the fastest; later calls run it. The north star's autotuner cached per
 * (log_size, n_columns); the reference has none (its Metal backend fixes its launch shapes).
 * mode -1 (the default) tunes; mode v >= 0 runs variant v of every op (the last one where an op has
 * fewer) and tunes nothing. */
typedef struct {
  uint32_t op, log_size, n_cols;
  int32_t variant;
  float ms[4]; /* measured milliseconds of each variant on the key's first call (0: none) */
} stwo_b200_tune_entry;
int32_t stwo_b200_autotune_mode(int32_t mode);
/* Tunes every key of one wide-Fibonacci proof shape: waits for the device, then proves one throwaway
 * proof of that shape (no proof of work) on the calling thread, whose first calls of each op tune it.
 * Call it while nothing else runs on the device (timings taken beside other work pick worse
 * variants); keys met later for the first time tune inside whatever call meets them. */
int32_t stwo_b200_autotune_wide_fibonacci(stwo_b200_context* ctx, uint32_t log_n_rows, uint32_t sequence_len,
                                          uint32_t log_blowup);
/* Copies the tuned keys into out[0..cap); *n receives their count (STWO_B200_E_BUFFER_TOO_SMALL when
 * cap is smaller). */
int32_t stwo_b200_autotune_table(stwo_b200_tune_entry* out, size_t cap, size_t* n);

/* ---- Testing ------------------------------------------------------------------------------------- */

/* Makes the nth device or pinned-host allocation of the library from now on fail as if out of memory
 * (0 disarms): the failure paths return STWO_B200_E_OOM, free what the call had taken and leave the
 * context usable. Host-side injection only, as the reference's armed failures
 * (armOwnershipTransferFailureForTesting, src/backends/metal/commit_backend.zig:69-71). */
int32_t stwo_b200_arm_allocation_failure_for_testing(uint32_t nth);

/* Makes the next launch of the bulk-staged DEEP quotient kernel (the quotient variant that copies
 * column chunks into shared memory with bulk async copies) leave its first stage empty in every CTA:
 * each bounded wait on it runs out after about a second, the kernel sets its timeout status and
 * returns, and the proof (or the op) ends with STWO_B200_E_CUDA and a message saying so. No copy
 * faults and no wait is unbounded; the context stays usable. */
int32_t stwo_b200_arm_quotient_stage_timeout_for_testing(void);

#ifdef __cplusplus
}
#endif
#endif /* STWO_B200_H */
