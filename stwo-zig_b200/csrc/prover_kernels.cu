// Per-stage kernels of the wide-Fibonacci proof: trace generation, constraint
// (composition) evaluation, OODS point evaluation, DEEP quotients, FRI folds and
// decommitment gathers.
//
// Sums of QM31 x M31 products are accumulated lazily per coordinate in 64-bit
// registers (each product < 2^62, folded every third term) and reduced once,
// which gives the same canonical result as the reference's term-by-term adds.
#include "blake2s.cuh"
#include "kernels.cuh"

namespace sb {

namespace {

// ---------------------------------------------------------------------------
// Trace generation (src/examples/wide_fibonacci/trace.zig:34-162). Storage
// position s holds logical row circleDomainIndexToCosetIndex(bitReverse(s)).
// kind 0: (1, row) seeds of the reference; kind 1: seeded uniform col0/col1 in
// [0, p-1): SplitMix64 keyed by seed ^ (0xD1B54A32D192ED03 * (2 row + col + 1)),
// top 31 bits, values >= p-1 rejected.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix64(uint64_t& state) {
  state += 0x9E3779B97F4A7C15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ uint32_t seeded_value(uint64_t seed, uint32_t column, uint64_t row) {
  uint64_t state = seed ^ (0xD1B54A32D192ED03ull * (2 * row + column + 1));
  for (int guard = 0; guard < 64; ++guard) {
    uint32_t v = (uint32_t)(splitmix64(state) >> 33);
    if (v < P - 1) return v;
  }
  return 0;  // probability 2^-1984: unreachable in practice
}

__global__ void k_wide_fib_trace(uint32_t log_n, uint32_t W, int kind, uint64_t seed, uint32_t* out, uint64_t stride) {
  const uint32_t n = 1u << log_n;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    uint32_t ci = bitrev(s, log_n);
    uint32_t row = ci < n / 2 ? ci * 2 : (n - 1 - ci) * 2 + 1;
    uint32_t a, b;
    if (kind == 0) { a = 1; b = row % P; }
    else { a = seeded_value(seed, 0, row); b = seeded_value(seed, 1, row); }
    out[s] = a;
    out[stride + s] = b;
    for (uint32_t k = 2; k < W; ++k) {
      uint32_t c = madd(mmul(a, a), mmul(b, b));
      out[k * stride + s] = c;
      a = b; b = c;
    }
  }
}

// ---------------------------------------------------------------------------
// Composition (src/examples/wide_fibonacci/component.zig:138-236): per row of
// CanonicCoset(n+1), sum_k coeff_k * (c_k - a_k^2 - b_k^2), times the inverse
// coset vanishing value den_inv[row >> n]. coeff_k = random_coeff^(W-3-k).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_composition(uint32_t log_n, uint32_t W, const uint32_t* __restrict__ eval,
                                                     uint64_t stride, const QM31* __restrict__ coeffs,
                                                     uint32_t den0, uint32_t den1, uint32_t* out, uint64_t out_stride) {
  extern __shared__ uint32_t sco[];  // (W-2) * 4 words
  const uint32_t n_cons = W - 2;
  for (uint32_t i = threadIdx.x; i < n_cons; i += blockDim.x) qstore4(coeffs[i], sco + 4 * i);
  __syncthreads();
  const uint32_t rows = 2u << log_n;
  for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    uint32_t a = __ldg(eval + row), b = __ldg(eval + stride + row);
    uint64_t acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
    for (uint32_t k = 0; k < n_cons; ++k) {
      uint32_t c = __ldg(eval + (uint64_t)(k + 2) * stride + row);
      uint32_t cons = msub(c, madd(mmul(a, a), mmul(b, b)));
      const uint32_t* q = sco + 4 * k;
      acc0 += (uint64_t)q[0] * cons; acc1 += (uint64_t)q[1] * cons;
      acc2 += (uint64_t)q[2] * cons; acc3 += (uint64_t)q[3] * cons;
      if (k % 3 == 2) { acc0 = mfold64(acc0); acc1 = mfold64(acc1); acc2 = mfold64(acc2); acc3 = mfold64(acc3); }
      a = b; b = c;
    }
    uint32_t d = (row >> log_n) ? den1 : den0;
    out[row] = mmul(mreduce64(acc0), d);
    out[out_stride + row] = mmul(mreduce64(acc1), d);
    out[2 * out_stride + row] = mmul(mreduce64(acc2), d);
    out[3 * out_stride + row] = mmul(mreduce64(acc3), d);
  }
}

// ---------------------------------------------------------------------------
// OODS evaluation (src/prover/poly/circle/poly.zig:62-230): value = sum_j c_j *
// prod_{bit b of j} F_b with F_0 = y, F_1 = x, F_b = pi^{b-1}(x). A CTA reduces
// a chunk of 4096 coefficients: 16 per thread against the subset products of
// F_0..F_3 (lazy 64-bit sums), then two radix-16 levels with F_4..F_7 and
// F_8..F_11, times the chunk's product of F_12.. .
// ---------------------------------------------------------------------------
constexpr uint32_t OODS_CHUNK_BITS = 12;
constexpr uint32_t OODS_THREADS = 256;

struct OodsFactors { QM31 f[32]; uint32_t log_size; };

__device__ QM31 subset_product(const OodsFactors& F, uint32_t bits, uint32_t first) {
  QM31 r = qone();
  for (uint32_t b = 0; bits; ++b, bits >>= 1)
    if (bits & 1) r = qmul(r, F.f[first + b]);
  return r;
}

__global__ void __launch_bounds__(OODS_THREADS) k_oods_chunks(OodsFactors F, const uint32_t* __restrict__ coeffs,
                                                              uint64_t stride, QM31* partial, uint32_t n_chunks) {
  __shared__ QM31 b4[3][16];
  __shared__ QM31 s1[OODS_THREADS];
  __shared__ QM31 s2[16];
  const uint32_t chunk = blockIdx.x, col = blockIdx.y;
  const uint32_t L = F.log_size;
  const uint32_t chunk_bits = L < OODS_CHUNK_BITS ? L : OODS_CHUNK_BITS;
  if (threadIdx.x < 48) {
    uint32_t lvl = threadIdx.x / 16, r = threadIdx.x % 16;
    // factors beyond log_size do not exist; mask them out
    uint32_t first = 4 * lvl;
    uint32_t valid_bits = first >= chunk_bits ? 0 : (chunk_bits - first >= 4 ? 4 : chunk_bits - first);
    b4[lvl][r] = (r >> valid_bits) ? qzero() : subset_product(F, r, first);
  }
  __syncthreads();
  const uint32_t n_in = 1u << chunk_bits;
  const uint32_t* c = coeffs + col * stride + ((uint64_t)chunk << chunk_bits);
  // level 0: thread t sums coefficients 16t .. 16t+15
  QM31 v = qzero();
  if (16 * threadIdx.x < n_in) {
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    const uint4* c4 = reinterpret_cast<const uint4*>(c + 16 * threadIdx.x);
    uint32_t w[16];
    uint32_t nw = n_in - 16 * threadIdx.x < 16 ? n_in - 16 * threadIdx.x : 16;
    if (nw == 16) {
#pragma unroll
      for (int q = 0; q < 4; ++q) { uint4 x = __ldg(c4 + q); w[4 * q] = x.x; w[4 * q + 1] = x.y; w[4 * q + 2] = x.z; w[4 * q + 3] = x.w; }
    } else {
      for (uint32_t r = 0; r < 16; ++r) w[r] = r < nw ? c[16 * threadIdx.x + r] : 0u;
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      QM31 bb = b4[0][r];
      a0 += (uint64_t)bb.c0.a * w[r]; a1 += (uint64_t)bb.c0.b * w[r];
      a2 += (uint64_t)bb.c1.a * w[r]; a3 += (uint64_t)bb.c1.b * w[r];
      if (r % 3 == 2) { a0 = mfold64(a0); a1 = mfold64(a1); a2 = mfold64(a2); a3 = mfold64(a3); }
    }
    v = qmake(mreduce64(a0), mreduce64(a1), mreduce64(a2), mreduce64(a3));
  }
  s1[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < 16) {
    QM31 acc = qzero();
    for (int r = 0; r < 16; ++r) acc = qadd(acc, qmul(s1[16 * threadIdx.x + r], b4[1][r]));
    s2[threadIdx.x] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    QM31 acc = qzero();
    for (int r = 0; r < 16; ++r) acc = qadd(acc, qmul(s2[r], b4[2][r]));
    // chunk index bits b correspond to factors chunk_bits + b
    QM31 hi = qone();
    uint32_t bits = chunk;
    for (uint32_t b = 0; bits; ++b, bits >>= 1)
      if (bits & 1) hi = qmul(hi, F.f[chunk_bits + b]);
    partial[(uint64_t)col * n_chunks + chunk] = qmul(acc, hi);
  }
}

__global__ void k_oods_sum(const QM31* partial, uint32_t n_chunks, uint32_t n_cols, QM31* out) {
  uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n_cols) return;
  QM31 acc = qzero();
  for (uint32_t i = 0; i < n_chunks; ++i) acc = qadd(acc, partial[(uint64_t)col * n_chunks + i]);
  out[col] = acc;
}

// ---------------------------------------------------------------------------
// DEEP quotients (src/core/pcs/quotients/row_evaluation.zig:101-140,400-521):
// row value = sum_batches (sum_i c_i v_i(row) - (sum_a * y + sum_b)) / den,
// den = (Re(Px) - x) Im(Py) - (Re(Py) - y) Im(Px) at the lifting-domain point of
// the row (bit-reversed circle-domain order).
// ---------------------------------------------------------------------------
constexpr uint32_t QUOT_MAX_ENTRIES = 1024;

__global__ void __launch_bounds__(256) k_quotients(PointTable pts, uint32_t log_size, uint32_t n_batches,
                                                   const QuotientBatchDev* __restrict__ batches,
                                                   const uint32_t* const* __restrict__ col_ptrs,
                                                   const QM31* __restrict__ coeff_c, uint32_t* out, uint64_t out_stride) {
  extern __shared__ uint32_t sq[];  // 4 words per entry
  uint32_t n_entries = 0;
  for (uint32_t b = 0; b < n_batches; ++b) n_entries = max(n_entries, batches[b].first + batches[b].count);
  for (uint32_t i = threadIdx.x; i < n_entries; i += blockDim.x) qstore4(coeff_c[i], sq + 4 * i);
  __syncthreads();
  const uint32_t rows = 1u << log_size;
  const CircleDomain dom = canonic_domain(log_size);
  for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    PointM dp = pts.at(dom.index_at(bitrev(row, log_size)));
    QM31 acc = qzero();
    for (uint32_t b = 0; b < n_batches; ++b) {
      const QuotientBatchDev bt = batches[b];
      uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
      for (uint32_t i = 0; i < bt.count; ++i) {
        uint32_t e = bt.first + i;
        uint32_t v = __ldg(col_ptrs[e] + row);
        const uint32_t* q = sq + 4 * e;
        a0 += (uint64_t)q[0] * v; a1 += (uint64_t)q[1] * v;
        a2 += (uint64_t)q[2] * v; a3 += (uint64_t)q[3] * v;
        if (i % 3 == 2) { a0 = mfold64(a0); a1 = mfold64(a1); a2 = mfold64(a2); a3 = mfold64(a3); }
      }
      QM31 num = qmake(mreduce64(a0), mreduce64(a1), mreduce64(a2), mreduce64(a3));
      num = qsub(num, qadd(qmulm(bt.sum_a, dp.y), bt.sum_b));
      CM31 prx = bt.point.x.c0, pry = bt.point.y.c0, pix = bt.point.x.c1, piy = bt.point.y.c1;
      CM31 den = csub(cmul(csub(prx, CM31{dp.x, 0}), piy), cmul(csub(pry, CM31{dp.y, 0}), pix));
      acc = qadd(acc, qmulc(num, cinv(den)));
    }
    out[row] = acc.c0.a;
    out[out_stride + row] = acc.c0.b;
    out[2 * out_stride + row] = acc.c1.a;
    out[3 * out_stride + row] = acc.c1.b;
  }
}

// ---------------------------------------------------------------------------
// FRI folds (src/core/fri/folding.zig:352-384, 558-602). The inverse twiddles
// of the fold are the inverse FFT twiddles of the source domain: 1/py of the
// circle layer for fold_circle_into_line, 1/x of line layer 0 for fold_line.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void qibfly(QM31& f0, QM31& f1, uint32_t it) {
  QM31 a = f0;
  f0 = qadd(a, f1);
  f1 = qmulm(qsub(a, f1), it);
}

__global__ void k_fold_circle(TwiddleView itv, uint32_t dst_log, const uint32_t* __restrict__ src, uint64_t ss,
                              QM31 alpha, QM31 alpha_sq, uint32_t* dst, uint64_t ds, int accumulate) {
  const uint32_t n = 1u << dst_log;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint2 w0 = *reinterpret_cast<const uint2*>(src + 2 * i);
    uint2 w1 = *reinterpret_cast<const uint2*>(src + ss + 2 * i);
    uint2 w2 = *reinterpret_cast<const uint2*>(src + 2 * ss + 2 * i);
    uint2 w3 = *reinterpret_cast<const uint2*>(src + 3 * ss + 2 * i);
    QM31 f0 = qmake(w0.x, w1.x, w2.x, w3.x), f1 = qmake(w0.y, w1.y, w2.y, w3.y);
    qibfly(f0, f1, itv.circ(i));
    QM31 r = qadd(qmul(alpha, f1), f0);
    if (accumulate) r = qadd(qmul(qmake(dst[i], dst[ds + i], dst[2 * ds + i], dst[3 * ds + i]), alpha_sq), r);
    dst[i] = r.c0.a; dst[ds + i] = r.c0.b; dst[2 * ds + i] = r.c1.a; dst[3 * ds + i] = r.c1.b;
  }
}

__global__ void k_fold_line(TwiddleView itv, uint32_t dst_log, const uint32_t* __restrict__ src, uint64_t ss,
                            QM31 alpha, uint32_t* dst, uint64_t ds) {
  const uint32_t n = 1u << dst_log;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint2 w0 = *reinterpret_cast<const uint2*>(src + 2 * i);
    uint2 w1 = *reinterpret_cast<const uint2*>(src + ss + 2 * i);
    uint2 w2 = *reinterpret_cast<const uint2*>(src + 2 * ss + 2 * i);
    uint2 w3 = *reinterpret_cast<const uint2*>(src + 3 * ss + 2 * i);
    QM31 f0 = qmake(w0.x, w1.x, w2.x, w3.x), f1 = qmake(w0.y, w1.y, w2.y, w3.y);
    qibfly(f0, f1, itv.line(1, i));
    QM31 r = qadd(f0, qmul(alpha, f1));
    dst[i] = r.c0.a; dst[ds + i] = r.c0.b; dst[2 * ds + i] = r.c1.a; dst[3 * ds + i] = r.c1.b;
  }
}

__global__ void k_gather_words(const GatherItem* items, uint32_t n, uint32_t* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = items[i].src[items[i].index];
}

__global__ void k_gather_hashes(const HashGatherItem* items, uint32_t n, uint8_t* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4* s = reinterpret_cast<const uint4*>(items[i].layers + items[i].node * 32);
  uint4* d = reinterpret_cast<uint4*>(out + (uint64_t)i * 32);
  d[0] = s[0];
  d[1] = s[1];
}

inline uint32_t grid_for(uint64_t n, uint32_t threads, uint32_t cap = 148 * 32) {
  uint64_t g = (n + threads - 1) / threads;
  if (g > cap) g = cap;
  return g == 0 ? 1 : (uint32_t)g;
}

}  // namespace

cudaError_t wide_fib_trace(uint32_t log_n, uint32_t W, int kind, uint64_t seed, uint32_t* out, uint64_t stride,
                           cudaStream_t stream) {
  k_wide_fib_trace<<<grid_for(1ull << log_n, 256), 256, 0, stream>>>(log_n, W, kind, seed, out, stride); note_launch();
  return cudaGetLastError();
}

cudaError_t wide_fib_composition(uint32_t log_n, uint32_t W, const uint32_t* eval, uint64_t stride,
                                 const QM31* coeffs_dev, uint32_t den_inv0, uint32_t den_inv1, uint32_t* out,
                                 uint64_t out_stride, cudaStream_t stream) {
  size_t smem = (size_t)(W - 2) * 16;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_composition, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_composition<<<grid_for(2ull << log_n, 256), 256, smem, stream>>>(log_n, W, eval, stride, coeffs_dev, den_inv0,
                                                                     den_inv1, out, out_stride); note_launch();
  return cudaGetLastError();
}

size_t eval_at_point_partial_count(uint32_t log_size, uint32_t n_cols) {
  uint32_t chunk_bits = log_size < OODS_CHUNK_BITS ? log_size : OODS_CHUNK_BITS;
  return (size_t)n_cols << (log_size - chunk_bits);
}

cudaError_t eval_at_point(const DeviceTables&, uint32_t log_size, uint32_t n_cols, const uint32_t* coeffs,
                          uint64_t stride, PointQ p, QM31*, QM31* partial, QM31* out, cudaStream_t stream) {
  if (log_size > 31) return cudaErrorInvalidValue;
  OodsFactors F{};
  F.log_size = log_size;
  if (log_size > 0) {
    F.f[0] = p.y;
    QM31 x = p.x;
    for (uint32_t b = 1; b < log_size; ++b) { F.f[b] = x; x = qdouble_x(x); }
  }
  uint32_t chunk_bits = log_size < OODS_CHUNK_BITS ? log_size : OODS_CHUNK_BITS;
  uint32_t n_chunks = 1u << (log_size - chunk_bits);
  dim3 grid(n_chunks, n_cols);
  k_oods_chunks<<<grid, OODS_THREADS, 0, stream>>>(F, coeffs, stride, partial, n_chunks); note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_oods_sum<<<(n_cols + 127) / 128, 128, 0, stream>>>(partial, n_chunks, n_cols, out); note_launch();
  return cudaGetLastError();
}

cudaError_t accumulate_quotients(const DeviceTables& t, uint32_t log_size, uint32_t n_batches,
                                 const QuotientBatchDev* batches, const uint32_t* const* col_ptrs, const QM31* coeff_c,
                                 uint32_t* out, uint64_t out_stride, cudaStream_t stream) {
  size_t smem = QUOT_MAX_ENTRIES * 16;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_quotients, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  k_quotients<<<grid_for(1ull << log_size, 256), 256, smem, stream>>>(PointTable{t.points}, log_size, n_batches,
                                                                      batches, col_ptrs, coeff_c, out, out_stride); note_launch();
  return cudaGetLastError();
}

cudaError_t fold_circle_into_line(const DeviceTables& t, uint32_t src_log, const uint32_t* src, uint64_t src_stride,
                                  QM31 alpha, uint32_t* dst, uint64_t dst_stride, bool accumulate,
                                  cudaStream_t stream) {
  TwiddleView itv = t.view(src_log, true);
  k_fold_circle<<<grid_for(1ull << (src_log - 1), 256), 256, 0, stream>>>(itv, src_log - 1, src, src_stride, alpha,
                                                                          qsq(alpha), dst, dst_stride, accumulate); note_launch();
  return cudaGetLastError();
}

cudaError_t fold_line(const DeviceTables& t, uint32_t src_log, const uint32_t* src, uint64_t src_stride, QM31 alpha,
                      uint32_t* dst, uint64_t dst_stride, cudaStream_t stream) {
  // Source line domain halfOdds(src_log): its tower layer is the line layer 0 of
  // the circle domain of log src_log + 1.
  TwiddleView itv = t.view(src_log + 1, true);
  k_fold_line<<<grid_for(1ull << (src_log - 1), 256), 256, 0, stream>>>(itv, src_log - 1, src, src_stride, alpha, dst,
                                                                        dst_stride); note_launch();
  return cudaGetLastError();
}

cudaError_t gather_words(const GatherItem* items, uint32_t n, uint32_t* out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_gather_words<<<(n + 255) / 256, 256, 0, stream>>>(items, n, out); note_launch();
  return cudaGetLastError();
}

cudaError_t gather_hashes(const HashGatherItem* items, uint32_t n, uint8_t* out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_gather_hashes<<<(n + 255) / 256, 256, 0, stream>>>(items, n, out); note_launch();
  return cudaGetLastError();
}

}  // namespace sb
