// LogUp interaction columns: per-row fractions of a relation's uses, running
// sums across a row's columns, and the row scan of the last column.
//
// Reference behaviour:
//  - fractions and the per-row accumulation across columns: stwo_zig_relation_fused,
//    src/backends/metal/shaders/core/relation.metal:131-158 (a column with two uses is
//    (n_a d_b + n_b d_a) / (d_a d_b), relation.metal:77-90; the pair batching of
//    src/frontends/riscv/air/logup.zig:76-105);
//  - coset-order scan with the total/N shift: relation.metal:160-237, scalar law
//    src/tests/metal/backend/commitment_test.zig:73-154 (scan index s visits circle index
//    s/2 for even s and N-1-s/2 for odd s, stored at its bit reverse; value(s) =
//    sum_{s' <= s} v(s') - total (s+1)/N; claimed = total);
//  - storage-order scan without shift: cumulativeColumn, src/frontends/riscv/air/logup.zig:83-105.
//
// Kernels: k_logup_fractions (one thread per row, one QM31 inversion per row by
// the suffix-product trick), then a three-pass scan over 1024-position blocks:
// block sums, a one-CTA scan of the block sums (which also writes the claimed
// sum), and the finalising rescan that writes the last column in place.
#include <algorithm>

#include "kernels.cuh"

namespace sb {

namespace {

constexpr int LU_THREADS = 256;
constexpr int SCAN_PER_THREAD = 4;
constexpr int SCAN_BLOCK = LU_THREADS * SCAN_PER_THREAD;  // positions per scan block

__device__ __forceinline__ QM31 use_denominator(const LogupParams& p, const LogupUse& u, uint64_t row) {
  QM31 acc = qneg(p.z);
  for (uint32_t j = 0; j < u.n_words; ++j) {
    uint32_t w = u.words[j] ? u.words[j][row] : u.constants[j];
    acc = qadd(acc, qmulm(p.alphas[j], w));
  }
  return acc;
}

__device__ __forceinline__ uint32_t use_numerator(const LogupUse& u, uint64_t row) {
  uint32_t m = u.multiplicity ? u.multiplicity[row] : 1u;
  return u.negate ? mneg(m) : m;
}

// Numerator and denominator of interaction column c at `row`.
__device__ __forceinline__ void column_fraction(const LogupParams& p, uint32_t c, uint64_t row, QM31& num,
                                                QM31& den) {
  uint32_t u0 = c * p.batch;
  QM31 da = use_denominator(p, p.uses[u0], row);
  uint32_t ma = use_numerator(p.uses[u0], row);
  if (p.batch == 2 && u0 + 1 < p.n_uses) {
    QM31 db = use_denominator(p, p.uses[u0 + 1], row);
    uint32_t mb = use_numerator(p.uses[u0 + 1], row);
    num = qadd(qmulm(da, mb), qmulm(db, ma));
    den = qmul(da, db);
  } else {
    num = qbase(ma);
    den = da;
  }
}

__device__ __forceinline__ QM31 col_load(const uint32_t* out, uint64_t stride, uint32_t c, uint64_t row) {
  const uint32_t* b = out + 4ull * c * stride + row;
  return qmake(b[0], b[stride], b[2 * stride], b[3 * stride]);
}
__device__ __forceinline__ void col_store(uint32_t* out, uint64_t stride, uint32_t c, uint64_t row, QM31 v) {
  uint32_t* b = out + 4ull * c * stride + row;
  b[0] = v.c0.a;
  b[stride] = v.c0.b;
  b[2 * stride] = v.c1.a;
  b[3 * stride] = v.c1.b;
}

__global__ void __launch_bounds__(LU_THREADS) k_logup_fractions(const __grid_constant__ LogupParams p, uint32_t* out,
                                                                uint64_t stride, uint32_t* zero_flag) {
  uint64_t row = (uint64_t)blockIdx.x * LU_THREADS + threadIdx.x;
  if (row >= (1ull << p.log_rows)) return;
  const uint32_t n_cols = logup_n_cols(p.n_uses, p.batch);
  // Backward: out[c] = n_c * prod_{c' > c} d_c', suffix = prod of all denominators.
  QM31 suffix = qone();
  for (uint32_t c = n_cols; c-- > 0;) {
    QM31 num, den;
    column_fraction(p, c, row, num, den);
    col_store(out, stride, c, row, qmul(num, suffix));
    suffix = qmul(suffix, den);
  }
  if (qiszero(suffix)) {
    atomicOr(zero_flag, 1u);
    return;
  }
  // Forward: running = (prod_{c' < c} d_c') / prod_all, so out[c] * running = n_c / d_c.
  QM31 running = qinv(suffix), acc = qzero();
  for (uint32_t c = 0; c < n_cols; ++c) {
    QM31 num, den;
    column_fraction(p, c, row, num, den);
    acc = qadd(acc, qmul(col_load(out, stride, c, row), running));
    col_store(out, stride, c, row, acc);
    running = qmul(running, den);
  }
}

__device__ __forceinline__ uint64_t scan_row(uint64_t s, uint32_t log_rows, uint32_t order) {
  if (order == 0 || log_rows == 0) return s;
  uint64_t rows = 1ull << log_rows;
  uint64_t ci = (s & 1) == 0 ? s >> 1 : rows - 1 - (s >> 1);
  return __brevll(ci) >> (64 - log_rows);
}

__device__ __forceinline__ QM31 shfl_up_q(QM31 v, int d) {
  return qmake(__shfl_up_sync(0xffffffffu, v.c0.a, d), __shfl_up_sync(0xffffffffu, v.c0.b, d),
               __shfl_up_sync(0xffffffffu, v.c1.a, d), __shfl_up_sync(0xffffffffu, v.c1.b, d));
}

// Inclusive scan of one QM31 per thread over a CTA of LU_THREADS threads; also returns the CTA total.
__device__ __forceinline__ QM31 block_inclusive_scan(QM31 v, QM31& total) {
  __shared__ QM31 warp_sums[LU_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    QM31 o = shfl_up_q(v, d);
    if (lane >= d) v = qadd(v, o);
  }
  if (lane == 31) warp_sums[warp] = v;
  __syncthreads();
  if (warp == 0) {
    QM31 w = lane < LU_THREADS / 32 ? warp_sums[lane] : qzero();
#pragma unroll
    for (int d = 1; d < LU_THREADS / 32; d <<= 1) {
      QM31 o = shfl_up_q(w, d);
      if (lane >= d) w = qadd(w, o);
    }
    if (lane < LU_THREADS / 32) warp_sums[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v = qadd(v, warp_sums[warp - 1]);
  total = warp_sums[LU_THREADS / 32 - 1];
  return v;
}

__global__ void __launch_bounds__(LU_THREADS) k_logup_block_sums(const uint32_t* col, uint64_t stride,
                                                                 uint32_t log_rows, uint32_t order, QM31* block_sums) {
  const uint64_t rows = 1ull << log_rows;
  const uint64_t s0 = (uint64_t)blockIdx.x * SCAN_BLOCK + (uint64_t)threadIdx.x * SCAN_PER_THREAD;
  QM31 sum = qzero();
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; ++k)
    if (s0 + k < rows) sum = qadd(sum, col_load(col, stride, 0, scan_row(s0 + k, log_rows, order)));
  QM31 total;
  block_inclusive_scan(sum, total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// One CTA: block_sums[b] <- sum of blocks before b; *claimed <- sum of all.
__global__ void __launch_bounds__(LU_THREADS) k_logup_scan_blocks(QM31* block_sums, uint32_t n_blocks,
                                                                  QM31* claimed) {
  const uint32_t per = (n_blocks + LU_THREADS - 1) / LU_THREADS;
  const uint32_t b0 = threadIdx.x * per;
  QM31 sum = qzero();
  for (uint32_t i = 0; i < per; ++i)
    if (b0 + i < n_blocks) sum = qadd(sum, block_sums[b0 + i]);
  QM31 total;
  QM31 incl = block_inclusive_scan(sum, total);
  QM31 run = qsub(incl, sum);  // exclusive prefix of this thread's chunk
  for (uint32_t i = 0; i < per; ++i) {
    if (b0 + i >= n_blocks) break;
    QM31 v = block_sums[b0 + i];
    block_sums[b0 + i] = run;
    run = qadd(run, v);
  }
  if (threadIdx.x == 0) *claimed = total;
}

__global__ void __launch_bounds__(LU_THREADS) k_logup_finalize(uint32_t* col, uint64_t stride, uint32_t log_rows,
                                                               uint32_t order, const QM31* block_prefix,
                                                               const QM31* claimed) {
  const uint64_t rows = 1ull << log_rows;
  const uint64_t s0 = (uint64_t)blockIdx.x * SCAN_BLOCK + (uint64_t)threadIdx.x * SCAN_PER_THREAD;
  QM31 v[SCAN_PER_THREAD];
  QM31 sum = qzero();
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; ++k) {
    v[k] = s0 + k < rows ? col_load(col, stride, 0, scan_row(s0 + k, log_rows, order)) : qzero();
    sum = qadd(sum, v[k]);
  }
  QM31 total_block;
  QM31 incl = block_inclusive_scan(sum, total_block);
  QM31 run = qadd(block_prefix[blockIdx.x], qsub(incl, sum));
  const QM31 total = *claimed;
  // 1/N = 2^(31 - log_rows) in M31 (2^31 = 1).
  const uint32_t inv_rows = log_rows == 0 ? 1u : (1u << (31 - log_rows)) % P;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; ++k) {
    uint64_t s = s0 + k;
    if (s >= rows) break;
    run = qadd(run, v[k]);
    QM31 out = run;
    if (order == 1) out = qsub(out, qmulm(total, mmul(inv_rows, (uint32_t)((s + 1) % P))));
    col_store(col, stride, 0, scan_row(s, log_rows, order), out);
  }
}

uint32_t scan_blocks(uint32_t log_rows) {
  uint64_t rows = 1ull << log_rows;
  return (uint32_t)((rows + SCAN_BLOCK - 1) / SCAN_BLOCK);
}

// XOR-lookup trace: seeded uniform u8 pairs, their XOR, the 2^16-row XOR table
// in the layout of the reference's bitwise table (row a * 256 + b holds (a, b, a ^ b),
// src/frontends/riscv/air/preprocessed/bitwise.zig:17-35) and the multiplicity of
// every table row in the trace.
__device__ __forceinline__ uint64_t xor_splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_xor_trace(uint32_t log_n, uint64_t seed, uint32_t* main_cols, uint32_t* mult) {
  const uint64_t rows = 1ull << log_n;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t x = xor_splitmix(seed ^ (0xD6E8FEB86659FD93ull * (r + 1)));
    uint32_t a = (uint32_t)x & 255u, b = (uint32_t)(x >> 8) & 255u;
    main_cols[r] = a;
    main_cols[rows + r] = b;
    main_cols[2 * rows + r] = a ^ b;
    atomicAdd(mult + (a << 8 | b), 1u);
  }
}

__global__ void k_xor_table(uint32_t* table) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 65536) return;
  const uint32_t a = i >> 8, b = i & 255u;
  table[i] = a;
  table[65536 + i] = b;
  table[2 * 65536 + i] = a ^ b;
}

}  // namespace

size_t logup_scratch_count(uint32_t log_rows) { return scan_blocks(log_rows); }

cudaError_t logup_interaction(const LogupParams& p, uint32_t* out, uint64_t out_stride, QM31* claimed,
                              QM31* scratch, uint32_t* zero_flag, cudaStream_t stream) {
  if (p.n_uses == 0 || p.n_uses > LOGUP_MAX_USES || (p.batch != 1 && p.batch != 2) || p.log_rows > 28 ||
      p.order > 1)
    return cudaErrorInvalidValue;
  const uint64_t rows = 1ull << p.log_rows;
  const uint32_t n_cols = logup_n_cols(p.n_uses, p.batch);
  k_logup_fractions<<<(unsigned)((rows + LU_THREADS - 1) / LU_THREADS), LU_THREADS, 0, stream>>>(p, out, out_stride,
                                                                                               zero_flag);
  note_launch();
  uint32_t* last = out + 4ull * (n_cols - 1) * out_stride;
  const uint32_t nb = scan_blocks(p.log_rows);
  k_logup_block_sums<<<nb, LU_THREADS, 0, stream>>>(last, out_stride, p.log_rows, p.order, scratch);
  note_launch();
  k_logup_scan_blocks<<<1, LU_THREADS, 0, stream>>>(scratch, nb, claimed);
  note_launch();
  k_logup_finalize<<<nb, LU_THREADS, 0, stream>>>(last, out_stride, p.log_rows, p.order, scratch, claimed);
  note_launch();
  return cudaGetLastError();
}

cudaError_t xor_lookup_trace(uint32_t log_n, uint64_t seed, uint32_t* main_cols, uint32_t* table, uint32_t* mult,
                             cudaStream_t stream) {
  if (log_n > 28) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(mult, 0, 65536 * 4, stream);
  if (e != cudaSuccess) return e;
  const uint64_t rows = 1ull << log_n;
  const uint32_t grid = (uint32_t)std::min<uint64_t>((rows + 255) / 256, 148 * 16);
  k_xor_trace<<<grid, 256, 0, stream>>>(log_n, seed, main_cols, mult);
  note_launch();
  k_xor_table<<<256, 256, 0, stream>>>(table);
  note_launch();
  return cudaGetLastError();
}

}  // namespace sb
