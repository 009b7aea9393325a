// Per-stage kernels of the wide-Fibonacci proof: trace generation, constraint
// (composition) evaluation, OODS point evaluation, DEEP quotients, FRI folds and
// decommitment gathers.
//
// Sums of QM31 x M31 products are accumulated lazily per coordinate in 64-bit
// registers (each product < 2^62, folded every third term) and reduced once,
// which gives the same canonical result as the reference's term-by-term adds.
#include <atomic>

#include "blake2s.cuh"
#include "kernels.cuh"
#include "tuner.hpp"

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

// Wide-Fibonacci trace in bit-reversed circle order: col0/col1 are the reference's (1, row) for
// kind 0, seeded uniform for kind 1, or already in `out` for kind 2; col_k = col_{k-2}^2 + col_{k-1}^2.
__global__ void k_wide_fib_trace(uint32_t log_n, uint32_t W, int kind, uint64_t seed, uint32_t* out, uint64_t stride) {
  const uint32_t n = 1u << log_n;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    uint32_t ci = bitrev(s, log_n);
    uint32_t row = ci < n / 2 ? ci * 2 : (n - 1 - ci) * 2 + 1;
    uint32_t a, b;
    if (kind == 2) {  // the first two columns are given: derive the rest
      a = out[s];
      b = out[stride + s];
    } else {
      if (kind == 0) { a = 1; b = row % P; }
      else { a = seeded_value(seed, 0, row); b = seeded_value(seed, 1, row); }
      out[s] = a;
      out[stride + s] = b;
    }
    for (uint32_t k = 2; k < W; ++k) {
      uint32_t c = madd(mmul(a, a), mmul(b, b));
      out[k * stride + s] = c;
      a = b; b = c;
    }
  }
}

// Quadratic-recurrence trace of a seven-word recipe (the fillQuadraticRecurrenceTrace column
// source, src/examples/wide_fibonacci/trace.zig:13-16): for the logical row k of each storage
// position, col0 = r0 + r1 k, col1 = r2 + r3 k, col_j = r4 col_{j-2}^2 + r5 col_{j-1}^2 + r6 (M31).
struct QuadRecipe { uint32_t r[7]; };
__global__ void k_quadratic_trace(uint32_t log_n, uint32_t W, QuadRecipe q, uint32_t* out, uint64_t stride) {
  const uint32_t n = 1u << log_n;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const uint32_t ci = bitrev(s, log_n);
    const uint32_t row = ci < n / 2 ? ci * 2 : (n - 1 - ci) * 2 + 1;
    uint32_t a = madd(q.r[0], mmul(q.r[1], row)), b = madd(q.r[2], mmul(q.r[3], row));
    out[s] = a;
    out[stride + s] = b;
    for (uint32_t k = 2; k < W; ++k) {
      const uint32_t c = madd(madd(mmul(q.r[4], mmul(a, a)), mmul(q.r[5], mmul(b, b))), q.r[6]);
      out[k * stride + s] = c;
      a = b;
      b = c;
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

// R consecutive rows per thread (RowVec<R>; R = 2 with 8-byte loads measured best:
// more warps and more loads in flight than 4 rows with 16-byte loads), the column
// loop unrolled by U (a multiple of 3: U loads in flight before their use, a
// 64-bit fold per three terms) and each column's square computed once (it is b^2
// of one constraint and a^2 of the next). Needs columns and output aligned to R
// words (eval, stride, out, out_stride) and 2^(log_n+1) >= R.
template <int R>
struct RowVec;
template <>
struct RowVec<2> {
  uint2 v;
  __device__ __forceinline__ static RowVec load(const uint32_t* p) { return {__ldg(reinterpret_cast<const uint2*>(p))}; }
  __device__ __forceinline__ static RowVec load_words(const uint32_t* p) { return {make_uint2(__ldg(p), __ldg(p + 1))}; }
  __device__ __forceinline__ uint32_t operator[](int j) const { return j == 0 ? v.x : v.y; }
  __device__ __forceinline__ static void store(uint32_t* p, const uint32_t* w) {
    *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
  }
};

// Rows per thread and unroll depth of the vectorized composition and quotient kernels.
constexpr int COMP_R = 2, COMP_U = 6, QUOT_R = 2, QUOT_U = 6;

template <int R, int U>
__global__ void __launch_bounds__(256, 4) k_composition_v(uint32_t log_n, uint32_t W, const uint32_t* __restrict__ eval,
                                                          uint64_t stride, const QM31* __restrict__ coeffs,
                                                          uint32_t den0, uint32_t den1, uint32_t* out,
                                                          uint64_t out_stride) {
  static_assert(U % 3 == 0, "fold every three terms");
  using V = RowVec<R>;
  extern __shared__ uint4 scq[];  // W-2 coefficients
  const uint32_t n_cons = W - 2;
  for (uint32_t i = threadIdx.x; i < n_cons; i += blockDim.x) {
    QM31 c = coeffs[i];
    scq[i] = make_uint4(c.c0.a, c.c0.b, c.c1.a, c.c1.b);
  }
  __syncthreads();
  const uint32_t groups = (2u << log_n) / R;
  for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < groups; gi += gridDim.x * blockDim.x) {
    const uint32_t row0 = gi * R;
    const uint32_t* base = eval + row0;
    V A = V::load(base), B = V::load(base + stride);
    uint32_t sa[R], sb[R];
#pragma unroll
    for (int j = 0; j < R; ++j) { sa[j] = mmul(A[j], A[j]); sb[j] = mmul(B[j], B[j]); }
    uint64_t acc[R][4];
#pragma unroll
    for (int j = 0; j < R; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[j][c] = 0;
    auto step = [&](const V& C, const uint4& q) {
#pragma unroll
      for (int j = 0; j < R; ++j) {
        uint32_t cj = C[j];
        uint32_t cons = msub(cj, madd(sa[j], sb[j]));
        sa[j] = sb[j];
        sb[j] = mmul(cj, cj);
        acc[j][0] += (uint64_t)q.x * cons;
        acc[j][1] += (uint64_t)q.y * cons;
        acc[j][2] += (uint64_t)q.z * cons;
        acc[j][3] += (uint64_t)q.w * cons;
      }
    };
    auto fold = [&]() {
#pragma unroll
      for (int j = 0; j < R; ++j)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[j][c] = mfold64(acc[j][c]);
    };
    uint32_t k = 0;
    for (; k + U <= n_cons; k += U) {
      V C[U];
#pragma unroll
      for (int u = 0; u < U; ++u) C[u] = V::load(base + (uint64_t)(k + 2 + u) * stride);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        step(C[u], scq[k + u]);
        if (u % 3 == 2) fold();
      }
    }
    for (uint32_t t = 0; k < n_cons; ++k, ++t) {
      step(V::load(base + (uint64_t)(k + 2) * stride), scq[k]);
      if (t % 3 == 2) fold();
    }
    const uint32_t d = (row0 >> log_n) ? den1 : den0;  // the R rows share row >> log_n
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t w[R];
#pragma unroll
      for (int j = 0; j < R; ++j) w[j] = mmul(mreduce64(acc[j][c]), d);
      V::store(out + (uint64_t)c * out_stride + row0, w);
    }
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

// A CTA owns one column and a strided set of its 4096-coefficient chunks: chunk = blockIdx.x +
// k * gridDim.x with gridDim.x a power of two, so a chunk's product of F_12.. splits over disjoint
// bits into the CTA's part (the bits of blockIdx.x, multiplied in once at the end) and k's part
// (a table hk[k] in shared memory, each entry a direct product computed by one thread: one barrier).
// Thread t sums its 16 coefficients of a chunk against the subset products of F_0..F_3, multiplies
// by hk[k] and accumulates; at the end it multiplies by the CTA's factor and its own (F_4..F_11
// subset selected by t), and the CTA reduces with warp shuffles to one partial.
constexpr uint32_t OODS_SMEM_CHUNKS = 1024;  // per-CTA chunk-factor table entries kept in shared memory

__device__ __forceinline__ QM31 shfl_down_q(QM31 v, int d) {
  return qmake(__shfl_down_sync(0xffffffffu, v.c0.a, d), __shfl_down_sync(0xffffffffu, v.c0.b, d),
               __shfl_down_sync(0xffffffffu, v.c1.a, d), __shfl_down_sync(0xffffffffu, v.c1.b, d));
}

__global__ void __launch_bounds__(OODS_THREADS) k_oods_chunks(OodsFactors F, const uint32_t* __restrict__ coeffs,
                                                              uint64_t stride, QM31* partial, uint32_t n_chunks) {
  __shared__ QM31 b4[3][16];
  __shared__ QM31 hk[OODS_SMEM_CHUNKS];
  __shared__ QM31 wsum[OODS_THREADS / 32];
  const uint32_t col = blockIdx.y;
  const uint32_t L = F.log_size;
  const uint32_t chunk_bits = L < OODS_CHUNK_BITS ? L : OODS_CHUNK_BITS;
  const uint32_t g_bits = __ffs(gridDim.x) - 1;  // gridDim.x = 2^g_bits
  const uint32_t k_first = chunk_bits + g_bits;   // factor index of k's bit 0
  if (threadIdx.x < 48) {
    uint32_t lvl = threadIdx.x / 16, r = threadIdx.x % 16;
    // factors beyond log_size do not exist; mask them out
    uint32_t first = 4 * lvl;
    uint32_t valid_bits = first >= chunk_bits ? 0 : (chunk_bits - first >= 4 ? 4 : chunk_bits - first);
    b4[lvl][r] = (r >> valid_bits) ? qzero() : subset_product(F, r, first);
  }
  const uint32_t n_k = blockIdx.x < n_chunks ? (n_chunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t n_tab = n_k < OODS_SMEM_CHUNKS ? n_k : OODS_SMEM_CHUNKS;
  for (uint32_t k = threadIdx.x; k < n_tab; k += blockDim.x) hk[k] = subset_product(F, k, k_first);
  __syncthreads();
  const uint32_t n_in = 1u << chunk_bits;
  const uint32_t t = threadIdx.x;
  const bool active = 16 * t < n_in;
  const uint32_t nw = active ? (n_in - 16 * t < 16 ? n_in - 16 * t : 16) : 0;
  QM31 acc = qzero();
  for (uint32_t k = 0; k < n_k && active; ++k) {
    const uint32_t chunk = blockIdx.x + k * gridDim.x;
    const uint32_t* c = coeffs + col * stride + ((uint64_t)chunk << chunk_bits) + 16 * t;
    uint32_t w[16];
    if (nw == 16) {
      const uint4* c4 = reinterpret_cast<const uint4*>(c);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint4 x = __ldg(c4 + q);
        w[4 * q] = x.x; w[4 * q + 1] = x.y; w[4 * q + 2] = x.z; w[4 * q + 3] = x.w;
      }
    } else {
      for (uint32_t r = 0; r < 16; ++r) w[r] = r < nw ? c[r] : 0u;
    }
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      QM31 bb = b4[0][r];
      a0 += (uint64_t)bb.c0.a * w[r]; a1 += (uint64_t)bb.c0.b * w[r];
      a2 += (uint64_t)bb.c1.a * w[r]; a3 += (uint64_t)bb.c1.b * w[r];
      if (r % 3 == 2) { a0 = mfold64(a0); a1 = mfold64(a1); a2 = mfold64(a2); a3 = mfold64(a3); }
    }
    QM31 v = qmake(mreduce64(a0), mreduce64(a1), mreduce64(a2), mreduce64(a3));
    QM31 h;
    if (k < OODS_SMEM_CHUNKS) {
      h = hk[k];
    } else {  // beyond the table: its low bits from the table, the rest multiplied in
      h = hk[k & (OODS_SMEM_CHUNKS - 1)];
      uint32_t bits = k >> 10;
      for (uint32_t b = k_first + 10; bits; ++b, bits >>= 1)
        if (bits & 1) h = qmul(h, F.f[b]);
    }
    acc = qadd(acc, qmul(v, h));
  }
  // the CTA's factor (bits of blockIdx.x), then the thread's own: subset of F_4..F_7 by bits 0-3
  // of t, of F_8..F_11 by bits 4-7
  acc = qmul(acc, subset_product(F, blockIdx.x, chunk_bits));
  acc = qmul(acc, qmul(b4[1][t & 15], b4[2][t >> 4]));
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) acc = qadd(acc, shfl_down_q(acc, d));
  if ((t & 31) == 0) wsum[t >> 5] = acc;
  __syncthreads();
  if (t == 0) {
    QM31 sum = qzero();
    for (int i = 0; i < OODS_THREADS / 32; ++i) sum = qadd(sum, wsum[i]);
    partial[(uint64_t)col * gridDim.x + blockIdx.x] = sum;
  }
}

// One warp per column: the lanes sum every 32nd partial, then a shuffle
// reduction (M31 addition is associative and commutative, so the order does not
// change the value). A thread per column summing up to 1184 partials in turn
// took 18-33 us for the few-column evaluations.
__global__ void k_oods_sum(const QM31* partial, uint32_t n_chunks, uint32_t n_cols, QM31* out) {
  const uint32_t col = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (col >= n_cols) return;  // warp-uniform
  const QM31* p = partial + (uint64_t)col * n_chunks;
  QM31 acc = qzero();
  for (uint32_t i = lane; i < n_chunks; i += 32) acc = qadd(acc, p[i]);
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) acc = qadd(acc, shfl_down_q(acc, d));
  if (lane == 0) out[col] = acc;
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

// Adds one batch's quotient to R rows: the numerators accumulated in `a` (lazy 64-bit sums of
// c_i v_i(row)) minus the batch's linear term, times the inverse denominators, the R rows'
// denominators inverted together.
template <int R>
__device__ __forceinline__ void quot_batch_finish(const QuotientBatchDev& bt, const PointM (&dp)[R],
                                                  const uint64_t (&a)[R][4], QM31 (&acc)[R]) {
  CM31 prx = bt.point.x.c0, pry = bt.point.y.c0, pix = bt.point.x.c1, piy = bt.point.y.c1;
  CM31 den[R], pre[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    den[j] = csub(cmul(csub(prx, CM31{dp[j].x, 0}), piy), cmul(csub(pry, CM31{dp[j].y, 0}), pix));
    pre[j] = j == 0 ? den[0] : cmul(pre[j - 1], den[j]);
  }
  CM31 inv[R];
  if (pre[R - 1].a == 0 && pre[R - 1].b == 0) {
#pragma unroll
    for (int j = 0; j < R; ++j) inv[j] = cinv(den[j]);
  } else {
    CM31 t = cinv(pre[R - 1]);
#pragma unroll
    for (int j = R - 1; j >= 1; --j) {
      inv[j] = cmul(t, pre[j - 1]);
      t = cmul(t, den[j]);
    }
    inv[0] = t;
  }
#pragma unroll
  for (int j = 0; j < R; ++j) {
    QM31 num = qmake(mreduce64(a[j][0]), mreduce64(a[j][1]), mreduce64(a[j][2]), mreduce64(a[j][3]));
    num = qsub(num, qadd(qmulm(bt.sum_a, dp[j].y), bt.sum_b));
    acc[j] = qadd(acc[j], qmulc(num, inv[j]));
  }
}

// R consecutive rows per thread: 8- or 16-byte loads of every column, entries
// unrolled by U (U loads in flight), and the R rows' denominators inverted
// together (one CM31 inversion per R rows, Montgomery's trick; a zero product
// falls back to per-row inversion so a zero denominator gives the same zero as
// the one-row kernel). Needs an output aligned to R words and 2^log_size >= R; a
// CTA that finds a column pointer off the vector alignment loads word by word.
template <int R, int U, int MINB>
__global__ void __launch_bounds__(256, MINB) k_quotients_v(PointTable pts, uint32_t log_size, uint32_t n_batches,
                                                        const QuotientBatchDev* __restrict__ batches,
                                                        const uint32_t* const* __restrict__ col_ptrs,
                                                        const QM31* __restrict__ coeff_c, uint32_t* out,
                                                        uint64_t out_stride) {
  static_assert(U % 3 == 0, "fold every three terms");
  using V = RowVec<R>;
  extern __shared__ uint4 sqe[];  // QUOT_MAX_ENTRIES coefficients, then the column pointers
  const uint32_t** sptr = reinterpret_cast<const uint32_t**>(sqe + QUOT_MAX_ENTRIES);
  __shared__ int s_bad;
  uint32_t n_entries = 0;
  for (uint32_t b = 0; b < n_batches; ++b) n_entries = max(n_entries, batches[b].first + batches[b].count);
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n_entries; i += blockDim.x) {
    QM31 c = coeff_c[i];
    sqe[i] = make_uint4(c.c0.a, c.c0.b, c.c1.a, c.c1.b);
    const uint32_t* p = col_ptrs[i];
    sptr[i] = p;
    if (reinterpret_cast<uintptr_t>(p) & (4 * R - 1)) s_bad = 1;
  }
  __syncthreads();
  const bool aligned = !s_bad;
  auto load = [&](const uint32_t* p) { return aligned ? V::load(p) : V::load_words(p); };
  const uint32_t groups = (1u << log_size) / R;
  const CircleDomain dom = canonic_domain(log_size);
  for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < groups; gi += gridDim.x * blockDim.x) {
    const uint32_t row0 = gi * R;
    PointM dp[R];
#pragma unroll
    for (int j = 0; j < R; ++j) dp[j] = pts.at(dom.index_at(bitrev(row0 + j, log_size)));
    QM31 acc[R];
#pragma unroll
    for (int j = 0; j < R; ++j) acc[j] = qzero();
    for (uint32_t b = 0; b < n_batches; ++b) {
      const QuotientBatchDev bt = batches[b];
      uint64_t a[R][4];
#pragma unroll
      for (int j = 0; j < R; ++j)
#pragma unroll
        for (int c = 0; c < 4; ++c) a[j][c] = 0;
      auto step = [&](const V& v, const uint4& q) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
          uint32_t vj = v[j];
          a[j][0] += (uint64_t)q.x * vj;
          a[j][1] += (uint64_t)q.y * vj;
          a[j][2] += (uint64_t)q.z * vj;
          a[j][3] += (uint64_t)q.w * vj;
        }
      };
      auto fold = [&]() {
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
          for (int c = 0; c < 4; ++c) a[j][c] = mfold64(a[j][c]);
      };
      uint32_t i = 0;
      const uint32_t e0 = bt.first;
      for (; i + U <= bt.count; i += U) {
        V v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = load(sptr[e0 + i + u] + row0);
#pragma unroll
        for (int u = 0; u < U; ++u) {
          step(v[u], sqe[e0 + i + u]);
          if (u % 3 == 2) fold();
        }
      }
      for (uint32_t t = 0; i < bt.count; ++i, ++t) {
        step(load(sptr[e0 + i] + row0), sqe[e0 + i]);
        if (t % 3 == 2) fold();
      }
      quot_batch_finish<R>(bt, dp, a, acc);
    }
    uint32_t w[R];
#pragma unroll
    for (int j = 0; j < R; ++j) w[j] = acc[j].c0.a;
    V::store(out + row0, w);
#pragma unroll
    for (int j = 0; j < R; ++j) w[j] = acc[j].c0.b;
    V::store(out + out_stride + row0, w);
#pragma unroll
    for (int j = 0; j < R; ++j) w[j] = acc[j].c1.a;
    V::store(out + 2 * out_stride + row0, w);
#pragma unroll
    for (int j = 0; j < R; ++j) w[j] = acc[j].c1.b;
    V::store(out + 3 * out_stride + row0, w);
  }
}

// ---- Quotients with the column words staged in shared memory by bulk async copies ----------
// Warp-specialized: eight consumer warps own a tile of QB_ROWS rows (two per thread); a ninth,
// producer warp streams the tile's column chunks (2 KB each) into a ring of QB_STAGES stages of
// QB_GROUP columns with 1-D bulk copies (cp.async.bulk global -> shared, one chunk per lane,
// completing on the stage's `full` mbarrier with the stage's byte count). A consumer warp waits on
// `full`, reads its threads' two words of each column, and arrives on the stage's `empty` mbarrier;
// the producer refills a stage once all eight consumer warps have arrived. The loads of the stages
// ahead stay in flight while one is consumed, without the registers the register kernel's loads in
// flight take, and the producer never holds the consumers at a block barrier. Items run batch by
// batch (a batch's entries in groups of at most QB_GROUP); the last group of a batch adds the
// batch's quotient. Each wait is bounded (about a second of the global timer): a side that runs out
// sets QUOT_STATUS_TIMEOUT in *status and a shared abort flag that ends the other side's loop; the
// producer then waits (again bounded) for the copies it issued. Batches that reach past the
// n_entries columns, or more groups than the item table holds, set QUOT_STATUS_LAYOUT before any
// copy is issued.
constexpr uint32_t QB_ROWS = 512, QB_GROUP = 8, QB_STAGES = 4, QB_MAX_BATCHES = 64;
constexpr uint32_t QB_CONSUMER_WARPS = QB_ROWS / 2 / 32, QB_THREADS = (QB_CONSUMER_WARPS + 1) * 32;
constexpr uint64_t QB_WAIT_NS = 1000000000ull;
// A test hook: the next bulk quotient launch issues no copy for its first item, so that every wait
// on that stage runs out.
std::atomic<bool> g_quot_skip_first_item{false};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) into this CTA's shared
// memory; its completion counts against the barrier's expected bytes.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// Waits for the completion of phase `parity` of the barrier for at most QB_WAIT_NS, or until *abort
// is set; false unless the phase completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int* abort) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
    // The clock and the abort flag are looked at every 64th try only (try_wait itself suspends).
    if ((it & 63) == 63 && ((abort && *abort) || global_ns() - t0 > QB_WAIT_NS)) return false;
  }
}

struct QbItem {
  uint32_t e0;     // first entry of the group
  uint16_t ne;     // entries in the group (0 .. QB_GROUP; 0 only for a batch without entries)
  uint16_t batch;  // 1 + the batch index when the group is its batch's last, else 0
};

template <int MINB>
__global__ void __launch_bounds__(QB_THREADS, MINB) k_quotients_bulk(PointTable pts, uint32_t log_size,
                                                                     uint32_t n_batches,
                                                                     const QuotientBatchDev* __restrict__ batches,
                                                                     const uint32_t* const* __restrict__ col_ptrs,
                                                                     const QM31* __restrict__ coeff_c,
                                                                     uint32_t n_entries, uint32_t item_cap,
                                                                     uint32_t* out, uint64_t out_stride,
                                                                     uint32_t* status, int skip_first_item) {
  constexpr int R = 2;
  extern __shared__ __align__(16) uint8_t qsm[];
  uint32_t* ring = reinterpret_cast<uint32_t*>(qsm);                     // QB_STAGES x QB_GROUP x QB_ROWS words
  uint4* sq = reinterpret_cast<uint4*>(ring + QB_STAGES * QB_GROUP * QB_ROWS);  // n_entries coefficients
  const uint32_t** sptr = reinterpret_cast<const uint32_t**>(sq + n_entries);  // n_entries column pointers
  QbItem* items = reinterpret_cast<QbItem*>(sptr + n_entries);                 // item_cap groups of one tile
  __shared__ uint64_t full[QB_STAGES], empty[QB_STAGES];
  __shared__ QuotientBatchDev sbt[QB_MAX_BATCHES];
  __shared__ int s_abort;
  __shared__ uint32_t s_items;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (uint32_t i = tid; i < n_entries; i += blockDim.x) {
    const QM31 c = coeff_c[i];
    sq[i] = make_uint4(c.c0.a, c.c0.b, c.c1.a, c.c1.b);
    sptr[i] = col_ptrs[i];
  }
  for (uint32_t b = tid; b < n_batches; b += blockDim.x) sbt[b] = batches[b];
  if (tid == 0) {
    uint32_t k = 0;
    bool bad = n_batches > QB_MAX_BATCHES;
    for (uint32_t b = 0; b < n_batches && !bad; ++b) {
      const uint32_t first = batches[b].first, count = batches[b].count;
      if (first > n_entries || count > n_entries - first) {
        bad = true;
        break;
      }
      // A batch without entries still adds its linear term: one empty group.
      for (uint32_t g = 0; g < count || (count == 0 && g == 0); g += QB_GROUP) {
        if (k == item_cap) {
          bad = true;
          break;
        }
        const uint32_t ne = min(QB_GROUP, count - g);
        items[k++] = QbItem{first + g, (uint16_t)ne, (uint16_t)(g + ne == count ? b + 1 : 0)};
      }
    }
    for (uint32_t s = 0; s < QB_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], QB_CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_items = k;
    s_abort = bad ? 1 : 0;
    if (bad) atomicOr(status, QUOT_STATUS_LAYOUT);
  }
  __syncthreads();
  if (s_abort) return;  // nothing issued
  const uint32_t n_items = s_items;
  const uint32_t n_tiles = (1u << log_size) / QB_ROWS;
  const uint32_t my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t total = (uint64_t)my_tiles * n_items;
  volatile int* abort = &s_abort;

  if (warp == QB_CONSUMER_WARPS) {
    // Producer warp: item i (tile-major, groups minor) into stage i % QB_STAGES, lane k copying the
    // group's k-th column chunk.
    uint64_t i = 0;
    bool ok = true;
    for (; i < total; ++i) {
      const uint32_t s = (uint32_t)(i % QB_STAGES);
      // Every lane waits (each acquires the consumers' release); the warp decides together.
      const bool got = i < QB_STAGES || mbar_wait_bounded(&empty[s], (uint32_t)(i / QB_STAGES - 1) & 1, abort);
      if (!__all_sync(0xffffffffu, got)) {
        ok = false;
        break;
      }
      if (skip_first_item && i == 0) continue;
      const uint32_t tile = blockIdx.x + (uint32_t)(i / n_items) * gridDim.x;
      const QbItem it = items[i % n_items];
      uint32_t* dst = ring + s * (QB_GROUP * QB_ROWS);
      // The stage's words were last read through the generic proxy; every lane that issues a copy
      // orders those reads before the async-proxy writes of its refill.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (lane == 0) mbar_arrive_expect_tx(&full[s], it.ne * QB_ROWS * 4);
      __syncwarp();
      if (lane < it.ne)
        bulk_load(dst + lane * QB_ROWS, sptr[it.e0 + lane] + (uint64_t)tile * QB_ROWS, QB_ROWS * 4, &full[s]);
    }
    if (lane == 0) {
      if (!ok) {
        *abort = 1;
        atomicOr(status, QUOT_STATUS_TIMEOUT);
      }
      // Items i - QB_STAGES .. i - 1 are the last ones issued (earlier ones were consumed before
      // their stages were refilled): let their copies land before the CTA's shared memory is
      // released, also when the consumers stopped early (bounded, the abort flag ignored).
      const uint64_t from = i > QB_STAGES ? i - QB_STAGES : 0;
      for (uint64_t j = from; j < i; ++j)
        if (!(skip_first_item && j == 0)) mbar_wait_bounded(&full[j % QB_STAGES], (uint32_t)(j / QB_STAGES) & 1, nullptr);
    }
  } else {
    const CircleDomain dom = canonic_domain(log_size);
    uint64_t item = 0;
    bool ok = true;
    for (uint32_t q = 0; q < my_tiles && ok; ++q) {
      const uint32_t row0 = (blockIdx.x + q * gridDim.x) * QB_ROWS + R * tid;
      PointM dp[R];
#pragma unroll
      for (int j = 0; j < R; ++j) dp[j] = pts.at(dom.index_at(bitrev(row0 + j, log_size)));
      QM31 acc[R];
#pragma unroll
      for (int j = 0; j < R; ++j) acc[j] = qzero();
      uint64_t a[R][4];
#pragma unroll
      for (int j = 0; j < R; ++j)
#pragma unroll
        for (int c = 0; c < 4; ++c) a[j][c] = 0;
      for (uint32_t g = 0; g < n_items; ++g, ++item) {
        const uint32_t s = (uint32_t)(item % QB_STAGES);
        // Every lane waits (each acquires the copies' completion); the warp decides together.
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[s], (uint32_t)(item / QB_STAGES) & 1, abort))) {
          ok = false;
          break;
        }
        const QbItem it = items[g];
        const uint32_t* col = ring + s * (QB_GROUP * QB_ROWS) + R * tid;
        const uint4* cq = sq + it.e0;
        // Terms of a group are folded after its entries 2, 5 and 7 (and after its last): at most
        // three products (< 2^62 each) on top of a folded value (< 2^34) between folds.
        auto term = [&](uint32_t k) {
          const uint2 v = *reinterpret_cast<const uint2*>(col + k * QB_ROWS);
          const uint4 c = cq[k];
          a[0][0] += (uint64_t)c.x * v.x; a[0][1] += (uint64_t)c.y * v.x;
          a[0][2] += (uint64_t)c.z * v.x; a[0][3] += (uint64_t)c.w * v.x;
          a[1][0] += (uint64_t)c.x * v.y; a[1][1] += (uint64_t)c.y * v.y;
          a[1][2] += (uint64_t)c.z * v.y; a[1][3] += (uint64_t)c.w * v.y;
        };
        auto fold = [&]() {
#pragma unroll
          for (int j = 0; j < R; ++j)
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) a[j][c4] = mfold64(a[j][c4]);
        };
        if (it.ne == QB_GROUP) {
#pragma unroll
          for (uint32_t k = 0; k < QB_GROUP; ++k) {
            term(k);
            if (k == 2 || k == 5 || k == 7) fold();
          }
        } else {
          for (uint32_t k = 0; k < it.ne; ++k) {
            term(k);
            if (k == 2 || k == 5 || k + 1 == it.ne) fold();
          }
        }
        // This warp is done with the stage's words.
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (it.batch) {
          quot_batch_finish<R>(sbt[it.batch - 1], dp, a, acc);
#pragma unroll
          for (int j = 0; j < R; ++j)
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) a[j][c4] = 0;
        }
      }
      if (!ok) break;
      const uint32_t w0[4] = {acc[0].c0.a, acc[0].c0.b, acc[0].c1.a, acc[0].c1.b};
      const uint32_t w1[4] = {acc[1].c0.a, acc[1].c0.b, acc[1].c1.a, acc[1].c1.b};
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4)
        *reinterpret_cast<uint2*>(out + c4 * out_stride + row0) = make_uint2(w0[c4], w1[c4]);
    }
    if (!ok) {
      *abort = 1;
      if (lane == 0) atomicOr(status, QUOT_STATUS_TIMEOUT);
    }
  }
  // The producer's bounded wait for its own copies ends before any thread of the CTA exits.
  __syncthreads();
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

cudaError_t quadratic_trace(uint32_t log_n, uint32_t W, const uint32_t recipe[7], uint32_t* out, uint64_t stride,
                            cudaStream_t stream) {
  QuadRecipe q;
  for (int i = 0; i < 7; ++i) q.r[i] = recipe[i] % P;
  k_quadratic_trace<<<grid_for(1ull << log_n, 256), 256, 0, stream>>>(log_n, W, q, out, stride); note_launch();
  return cudaGetLastError();
}

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
  const bool vec = ((reinterpret_cast<uintptr_t>(eval) | reinterpret_cast<uintptr_t>(out)) & (4 * COMP_R - 1)) == 0 &&
                   stride % COMP_R == 0 && out_stride % COMP_R == 0 && (2ull << log_n) >= COMP_R;
  if (vec) {
    k_composition_v<COMP_R, COMP_U><<<grid_for(2ull << log_n, 256 * COMP_R), 256, smem, stream>>>(
        log_n, W, eval, stride, coeffs_dev, den_inv0, den_inv1, out, out_stride);
  } else {
    k_composition<<<grid_for(2ull << log_n, 256), 256, smem, stream>>>(log_n, W, eval, stride, coeffs_dev, den_inv0,
                                                                       den_inv1, out, out_stride);
  }
  note_launch();
  return cudaGetLastError();
}

namespace {
// dst[i] += coeff * src[lifted i] over 4 coordinate columns (src of 2^src_log <= 2^dst_log rows).
__global__ void k_accumulate_lifted(uint32_t dst_log, uint32_t* dst, uint64_t ds, uint32_t src_log,
                                    const uint32_t* __restrict__ src, uint64_t ss, QM31 coeff) {
  const uint64_t n = 1ull << dst_log;
  const uint32_t sh = dst_log - src_log + 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = src_log == dst_log ? i : (((i >> sh) << 1) | (i & 1));
    const QM31 v = qmul(coeff, qmake(src[j], src[ss + j], src[2 * ss + j], src[3 * ss + j]));
    dst[i] = madd(dst[i], v.c0.a);
    dst[ds + i] = madd(dst[ds + i], v.c0.b);
    dst[2 * ds + i] = madd(dst[2 * ds + i], v.c1.a);
    dst[3 * ds + i] = madd(dst[3 * ds + i], v.c1.b);
  }
}

}  // namespace

cudaError_t accumulate_lifted(uint32_t dst_log, uint32_t* dst, uint64_t dst_stride, uint32_t src_log,
                              const uint32_t* src, uint64_t src_stride, QM31 coeff, cudaStream_t stream) {
  if (src_log > dst_log) return cudaErrorInvalidValue;
  k_accumulate_lifted<<<grid_for(1ull << dst_log, 256), 256, 0, stream>>>(dst_log, dst, dst_stride, src_log, src,
                                                                           src_stride, coeff);
  note_launch();
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
  // A power of two of CTAs per column (the chunk factor splits over the CTA's bits): about four
  // waves of five CTAs per SM over all columns, never more CTAs per column than chunks.
  uint32_t per_col = 1;
  while (per_col < n_chunks && (uint64_t)per_col * n_cols < 148ull * 5 * 4) per_col <<= 1;
  dim3 grid(per_col, n_cols);
  k_oods_chunks<<<grid, OODS_THREADS, 0, stream>>>(F, coeffs, stride, partial, n_chunks); note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_oods_sum<<<(n_cols + 3) / 4, 128, 0, stream>>>(partial, per_col, n_cols, out); note_launch();
  return cudaGetLastError();
}

template <int R, int U, int MINB>
static void quotients_smem_attr(size_t smem_v) {
  cudaFuncSetAttribute(k_quotients_v<R, U, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_v);
}

void arm_quotient_stage_timeout_for_testing() { g_quot_skip_first_item.store(true); }

cudaError_t accumulate_quotients(const DeviceTables& t, uint32_t log_size, uint32_t n_batches, uint32_t n_entries,
                                 const QuotientBatchDev* batches, const uint32_t* const* col_ptrs, const QM31* coeff_c,
                                 uint32_t* out, uint64_t out_stride, cudaStream_t stream, uint32_t* status) {
  size_t smem = QUOT_MAX_ENTRIES * 16;
  size_t smem_v = QUOT_MAX_ENTRIES * (16 + sizeof(void*));
  // Bulk-staged kernel: the ring, the coefficients and pointers, and the item table (every batch
  // adds at most one partial group).
  const uint32_t item_cap = (n_entries + QB_GROUP - 1) / QB_GROUP + n_batches;
  const size_t smem_b = (size_t)QB_STAGES * QB_GROUP * QB_ROWS * 4 + (size_t)n_entries * (16 + sizeof(void*)) +
                        (size_t)item_cap * sizeof(QbItem);
  constexpr size_t SMEM_B_MAX = (size_t)QB_STAGES * QB_GROUP * QB_ROWS * 4 +
                                (size_t)QUOT_MAX_ENTRIES * (16 + sizeof(void*)) +
                                (size_t)(QUOT_MAX_ENTRIES / QB_GROUP + QB_MAX_BATCHES) * sizeof(QbItem);
  static const bool attr = [&] {  // once per process (thread-safe static initialisation)
    cudaFuncSetAttribute(k_quotients, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    quotients_smem_attr<QUOT_R, QUOT_U, 3>(smem_v);
    quotients_smem_attr<QUOT_R, 3, 4>(smem_v);
    quotients_smem_attr<QUOT_R, 9, 2>(smem_v);
    cudaFuncSetAttribute(k_quotients_bulk<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_B_MAX);
    cudaFuncSetAttribute(k_quotients_bulk<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_B_MAX);
    return true;
  }();
  (void)attr;
  const bool vec = (reinterpret_cast<uintptr_t>(out) & (4 * QUOT_R - 1)) == 0 && out_stride % QUOT_R == 0 &&
                   (1ull << log_size) >= QUOT_R;
  if (!vec) {
    k_quotients<<<grid_for(1ull << log_size, 256), 256, smem, stream>>>(PointTable{t.points}, log_size, n_batches,
                                                                        batches, col_ptrs, coeff_c, out, out_stride);
    note_launch();
    return cudaGetLastError();
  }
  // The bulk-staged kernel takes whole 512-row tiles of 16-byte aligned columns (the caller vouches
  // for the pointers by passing `status`).
  const bool bulk = status != nullptr && log_size >= 16 && n_batches <= QB_MAX_BATCHES &&
                    n_entries <= QUOT_MAX_ENTRIES;
  // Variants: 6 loads in flight per thread at 3 CTAs per SM, 3 at 4, 9 at 2; bulk-staged.
  auto run = [&](int variant) -> cudaError_t {
    if (variant == 3 && !bulk) variant = 0;  // a key tuned by a caller that could take it
    const dim3 grid(grid_for(1ull << log_size, 256 * QUOT_R));
    const PointTable pts{t.points};
    if (variant == 1)
      k_quotients_v<QUOT_R, 3, 4><<<grid, 256, smem_v, stream>>>(pts, log_size, n_batches, batches, col_ptrs, coeff_c,
                                                                   out, out_stride);
    else if (variant == 2)
      k_quotients_v<QUOT_R, 9, 2><<<grid, 256, smem_v, stream>>>(pts, log_size, n_batches, batches, col_ptrs, coeff_c,
                                                                   out, out_stride);
    else if (variant == 3) {
      // Persistent: as many CTAs as stay resident (three per SM while the shared memory allows).
      const int minb = smem_b <= 70 * 1024 ? 3 : 2;
      const uint32_t n_tiles = (uint32_t)((1ull << log_size) / QB_ROWS);
      const uint32_t g = std::min<uint32_t>(n_tiles, t.sm_count * (uint32_t)minb);
      const int skip = g_quot_skip_first_item.exchange(false) ? 1 : 0;
      if (minb == 3)
        k_quotients_bulk<3><<<g, QB_THREADS, smem_b, stream>>>(pts, log_size, n_batches, batches, col_ptrs, coeff_c, n_entries,
                                                        item_cap, out, out_stride, status, skip);
      else
        k_quotients_bulk<2><<<g, QB_THREADS, smem_b, stream>>>(pts, log_size, n_batches, batches, col_ptrs, coeff_c, n_entries,
                                                        item_cap, out, out_stride, status, skip);
    } else
      k_quotients_v<QUOT_R, QUOT_U, 3><<<grid, 256, smem_v, stream>>>(pts, log_size, n_batches, batches, col_ptrs,
                                                                      coeff_c, out, out_stride);
    note_launch();
    return cudaGetLastError();
  };
  // Reads the columns, writes `out`: re-runnable. Keyed by the committed columns read per row.
  return tuned_run(TUNE_QUOTIENTS, log_size, n_entries, log_size >= 16 ? (bulk ? 4 : 3) : 1, true, stream, run);
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
