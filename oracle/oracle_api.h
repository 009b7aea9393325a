/*
 * C entry points of the CPU oracle: a plain C++ restatement of the reference
 * prover's algorithm for the wide-Fibonacci circle-STARK path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker or the timed CPU baseline. The product (libstwo_b200)
 * never links or calls it.
 *
 * Every function returns 0 on success and a negative value on bad arguments.
 * Column buffers are canonical M31 words (uint32 in [0, 2^31-1)).
 */
#ifndef STWO_ORACLE_API_H
#define STWO_ORACLE_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Protocol parameters, the reference's PcsConfig (src/core/pcs/mod.zig:23-52). */
typedef struct {
  uint32_t pow_bits;
  uint32_t log_blowup_factor;
  uint32_t log_last_layer_degree_bound;
  uint32_t n_queries;
} oracle_pcs_config;

/* Trace kinds: 0 = the reference's (1, row) seeds (src/examples/wide_fibonacci/trace.zig:16),
 * 1 = seeded uniform col0/col1 in [0, p-1) (SplitMix64 with rejection, per (seed, column, row)). */
int oracle_gen_trace(uint32_t log_n_rows, uint32_t sequence_len, int trace_kind, uint64_t seed,
                     uint32_t* out /* sequence_len * 2^log_n_rows, column-major */);

/* Full proof. `trace` may be NULL (then generated from trace_kind/seed). The proof is the
 * reference's JSON wire encoding (src/interop/proof_wire.zig:19-77). */
int oracle_prove_wide_fib(uint32_t log_n_rows, uint32_t sequence_len, const oracle_pcs_config* cfg,
                          const uint32_t* trace, int trace_kind, uint64_t trace_seed,
                          int has_channel_seed, uint64_t channel_seed, int n_threads,
                          uint8_t* out, size_t out_cap, size_t* out_len);

/* LogUp XOR-lookup AIR proof (2^log_n lookups of seeded (log_table/2)-bit pairs into the
 * 2^log_table-row XOR table, both components at their own sizes under the lifted PCS); the JSON
 * layout of the wide-Fibonacci proof plus "statement" and "claimed_sums". Returns -5 on a zero LogUp
 * denominator, -4 when a self-check fails, -2 when out_cap is too small (out_len set). */
int oracle_prove_logup_xor(uint32_t log_n, uint32_t log_table, const oracle_pcs_config* cfg, uint64_t seed,
                           int has_channel_seed, uint64_t channel_seed, int n_threads, uint8_t* out,
                           size_t out_cap, size_t* out_len);

/* Seconds the calling thread's last oracle proof spent in its proof-of-work grind. */
double oracle_last_pow_seconds(void);

/* Op-level checkers (all host buffers). */
int oracle_interpolate(uint32_t log_size, uint32_t* values /* in: evals, out: coeffs */);
int oracle_evaluate(uint32_t log_size, uint32_t* values /* in: coeffs, out: evals */);
/* coeffs of log_size extended to log_size+log_blowup evaluations. */
int oracle_extend(uint32_t log_size, uint32_t log_blowup, const uint32_t* coeffs, uint32_t* evals);
int oracle_merkle_root(uint32_t n_cols, const uint32_t* log_sizes, const uint32_t* const* cols,
                       uint8_t root[32]);
/* Full layer dump: layers[k] for k = max_log..0 concatenated, 32 bytes per node. */
int oracle_merkle_layers(uint32_t n_cols, const uint32_t* log_sizes, const uint32_t* const* cols,
                         uint8_t* out_layers);
int oracle_fold_circle_into_line(uint32_t src_log_size, const uint32_t* src /* 4 coord cols */,
                                 const uint32_t alpha[4], uint32_t* dst /* 4 coord cols, accumulated */);
/* line_coset_log_size is the log size of the source line evaluation; the line domain is
 * halfOdds(line_coset_log_size) doubled `n_doubles` times (the FRI inner-layer tower). */
int oracle_fold_line(uint32_t src_log_size, uint32_t first_line_log_size, const uint32_t* src,
                     const uint32_t alpha[4], uint32_t* dst);
int oracle_eval_at_point(uint32_t log_size, const uint32_t* coeffs, const uint32_t px[4],
                         const uint32_t py[4], uint32_t out[4]);
int oracle_blake2s(const uint8_t* data, size_t len, uint8_t out[32]);
int oracle_pow_grind(const uint8_t digest[32], uint32_t n_bits, int n_threads, uint64_t* nonce);

/* Batch inverse of n elements of degree 1, 2 or 4 (degree coordinate planes of n words).
 * Returns -2 when an element is zero. */
int oracle_batch_inverse(uint32_t degree, uint64_t n, const uint32_t* src, uint32_t* dst);

/* One LogUp use (host columns of 2^log_rows words; NULL word = constant, NULL multiplicity = 1). */
typedef struct {
  uint32_t n_words;
  uint32_t negate;
  const uint32_t* words[8];
  uint32_t constants[8];
  const uint32_t* multiplicity;
} oracle_logup_use;
/* Interaction columns (4 planes per column, 2^log_rows words each) and the claimed sum.
 * alphas: n_words x 4 words. Returns -2 on a zero denominator. */
int oracle_logup_interaction(uint32_t log_rows, uint32_t n_uses, const oracle_logup_use* uses,
                             const uint32_t* alphas, const uint32_t z[4], uint32_t batch, uint32_t order,
                             uint32_t* out, uint32_t claimed[4]);

/* XOR-lookup trace: main 3 x 2^log_n (a, b, a ^ b), table 3 x 65536, mult 65536. */
int oracle_xor_lookup_trace(uint32_t log_n, uint64_t seed, uint32_t* main_cols, uint32_t* table, uint32_t* mult);

#ifdef __cplusplus
}
#endif
#endif
