// LogUp XOR-lookup AIR prover on one device stream.
//
// The reference has no such AIR (its LogUp machinery is the relation graph of
// src/backends/metal/shaders/core/relation.metal and cumulativeColumn of
// src/frontends/riscv/air/logup.zig); this AIR is built from the same pieces and
// the same PCS, with every stage on the device:
//
//   rows      2^L, L = max(log_n, log_table); logical row k (coset order) is stored
//             at bitrev(circle index of k), as in src/examples/wide_fibonacci/trace.zig:159-162
//   tree 0    preprocessed: ta, tb, tc = ta ^ tb (row k holds table row k mod 2^log_table,
//             a * 2^w + b for operands of w = log_table / 2 bits, the layout of
//             src/frontends/riscv/air/preprocessed/bitwise.zig:17-35), sel = [k < 2^log_n]
//   tree 1    main: a, b (seeded uniform w-bit values for k < 2^log_n, else 0), c = a ^ b,
//             m = multiplicity of table row k among the first 2^log_n rows (0 for k >= 2^log_table)
//   draw      z, alpha; alphas = (1, alpha, alpha^2)
//   tree 2    interaction: S_main, S_table (QM31, 4 columns each), the coset-order cumulative
//             sums with the total/N shift of sel / (a + alpha b + alpha^2 c - z) and of
//             -m / (ta + alpha tb + alpha^2 tc - z); their totals are the claimed sums
//   mix       both claimed sums; the verifier requires them to add to zero
//   tree 3    composition: (rc * C_main + C_table) / Z_trace on CanonicCoset(L+1), split in
//             halves, with C = (S(x) - S(x g^-1) + claimed / N) * d(x) - numerator(x)
//   samples   every column at the OODS point P; tree 2 also at P - g (the previous row)
//   quotients samples with random powers and point batches as in the reference's
//             buildSamplesWithRandomnessAndPeriodicity / buildColumnSampleBatchesFromParallelInputs
//             (src/core/pcs/quotients/samples.zig:163-300): a two-sample column adds a
//             periodicity sample at P plus the lifting generator doubled to the column's log
//             size, here the identity, so at P with the current value
//   tail      FRI, proof of work, queries and decommitment as for wide-Fibonacci.
#include <algorithm>
#include <cstring>

#include "prover_common.hpp"

namespace sb {

namespace {

__device__ __forceinline__ uint32_t coset_row_of(uint32_t s, uint32_t log) {
  uint32_t n = 1u << log;
  uint32_t ci = bitrev(s, log);
  return ci < n / 2 ? ci * 2 : (n - 1 - ci) * 2 + 1;
}
__device__ __forceinline__ uint32_t storage_of(uint32_t k, uint32_t log) {
  uint32_t n = 1u << log;
  uint32_t ci = (k & 1) == 0 ? k / 2 : n - 1 - (k >> 1);
  return bitrev(ci, log);
}

__device__ __forceinline__ uint64_t xor_mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Trace columns at storage position s; counts table-row hits for the multiplicities.
__global__ void k_xor_air_trace(uint32_t L, uint32_t log_n, uint32_t log_table, uint64_t seed, uint32_t* pre,
                                uint32_t* main_cols, uint32_t* hist) {
  const uint32_t N = 1u << L, w = log_table / 2, wmask = (1u << w) - 1, tmask = (1u << log_table) - 1;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const uint32_t k = coset_row_of(s, L);
    const uint32_t t = k & tmask;
    const uint32_t ta = t >> w, tb = t & wmask;
    pre[s] = ta;
    pre[N + s] = tb;
    pre[2 * N + s] = ta ^ tb;
    const bool live = k < (1u << log_n);
    pre[3 * N + s] = live ? 1u : 0u;
    uint32_t a = 0, b = 0;
    if (live) {
      uint64_t x = xor_mix(seed ^ (0xD6E8FEB86659FD93ull * ((uint64_t)k + 1)));
      a = (uint32_t)x & wmask;
      b = (uint32_t)(x >> 8) & wmask;
      atomicAdd(hist + (a << w | b), 1u);
    }
    main_cols[s] = a;
    main_cols[N + s] = b;
    main_cols[2 * N + s] = a ^ b;
  }
}

__global__ void k_xor_air_mult(uint32_t L, uint32_t log_table, const uint32_t* hist, uint32_t* m) {
  const uint32_t N = 1u << L;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const uint32_t k = coset_row_of(s, L);
    m[s] = k < (1u << log_table) ? hist[k] : 0u;
  }
}

struct XorCompParams {
  QM31 alpha1, alpha2, z, rc, shift_main, shift_table;
  uint32_t den0, den1;
  uint32_t L, CL;
};

__device__ __forceinline__ QM31 ld_q(const uint32_t* c, uint64_t stride, uint32_t r) {
  return qmake(c[r], c[stride + r], c[2 * stride + r], c[3 * stride + r]);
}

// Composition on CanonicCoset(L+1): cols = 16 columns (tree 0, tree 1, tree 2) of 2^CL, stride.
__global__ void __launch_bounds__(256) k_xor_composition(const __grid_constant__ XorCompParams p,
                                                         const uint32_t* __restrict__ cols, uint64_t stride,
                                                         uint32_t* out, uint64_t out_stride) {
  const uint32_t NC = 1u << p.CL;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < NC; r += gridDim.x * blockDim.x) {
    // x g^-1 is two steps back on the doubled coset.
    const uint32_t j = coset_row_of(r, p.CL);
    const uint32_t rp = storage_of((j + NC - 2) & (NC - 1), p.CL);
    const uint32_t ta = cols[r], tb = cols[stride + r], tc = cols[2 * stride + r], sel = cols[3 * stride + r];
    const uint32_t a = cols[4 * stride + r], b = cols[5 * stride + r], c = cols[6 * stride + r],
                   m = cols[7 * stride + r];
    const QM31 sm = ld_q(cols + 8 * stride, stride, r), sm_prev = ld_q(cols + 8 * stride, stride, rp);
    const QM31 st = ld_q(cols + 12 * stride, stride, r), st_prev = ld_q(cols + 12 * stride, stride, rp);
    const QM31 d_main = qsub(qadd(qadd(qbase(a), qmulm(p.alpha1, b)), qmulm(p.alpha2, c)), p.z);
    const QM31 d_table = qsub(qadd(qadd(qbase(ta), qmulm(p.alpha1, tb)), qmulm(p.alpha2, tc)), p.z);
    const QM31 c_main = qsub(qmul(qadd(qsub(sm, sm_prev), p.shift_main), d_main), qbase(sel));
    const QM31 c_table = qadd(qmul(qadd(qsub(st, st_prev), p.shift_table), d_table), qbase(m));
    const QM31 q = qmulm(qadd(qmul(p.rc, c_main), c_table), (r >> p.L) ? p.den1 : p.den0);
    out[r] = q.c0.a;
    out[out_stride + r] = q.c0.b;
    out[2 * out_stride + r] = q.c1.a;
    out[3 * out_stride + r] = q.c1.b;
  }
}

struct XorShape {
  uint32_t L, B, log_table, n_inner;
};
struct XorBufs {
  uint32_t *vals, *coeffs, *lde, *eval_c, *comp, *comp_lde, *quot, *hist;
  uint8_t *tree[4], *tree_q, *scratch;
  std::vector<uint32_t*> line;
  std::vector<uint8_t*> line_tree;
  QM31 *oods_partial, *oods_out, *quot_c, *claimed, *logup_scratch;
  const uint32_t** col_ptrs;
  QuotientBatchDev* batch;
  uint32_t *pow_result, *zero_flag;
  FriChannelDev* chan;
};
XorBufs xor_carve(Arena& a, const XorShape& sh) {
  const uint64_t N = 1ull << sh.L, NL = N << sh.B, NC = N << 1;
  const uint32_t LDE = sh.L + sh.B;
  XorBufs b{};
  b.vals = a.take<uint32_t>(16 * N);  // tree 0 (4), tree 1 (4), tree 2 (8) values
  b.coeffs = a.take<uint32_t>(16 * N);
  b.lde = a.take<uint32_t>(16 * NL);
  b.eval_c = sh.B == 1 ? b.lde : a.take<uint32_t>(16 * NC);
  b.comp = a.take<uint32_t>(4 * NC);
  b.comp_lde = a.take<uint32_t>(8 * NL);
  b.quot = a.take<uint32_t>(4 * NL);
  b.hist = a.take<uint32_t>(1u << sh.log_table);
  for (int t = 0; t < 4; ++t) b.tree[t] = a.take<uint8_t>((2 * NL - 1) * 32);
  b.tree_q = a.take<uint8_t>((2 * NL - 1) * 32);
  for (uint32_t k = 0; k <= sh.n_inner; ++k) {
    size_t sz = 1ull << (LDE - 1 - k);
    b.line.push_back(a.take<uint32_t>(4 * sz));
    b.line_tree.push_back(k < sh.n_inner ? a.take<uint8_t>((2 * sz - 1) * 32) : nullptr);
  }
  b.oods_partial = a.take<QM31>(eval_at_point_partial_count(sh.L, 16));
  b.oods_out = a.take<QM31>(40);
  b.quot_c = a.take<QM31>(64);
  b.col_ptrs = a.take<const uint32_t*>(64);
  b.batch = a.take<QuotientBatchDev>(2);
  b.claimed = a.take<QM31>(2);
  b.logup_scratch = a.take<QM31>(logup_scratch_count(sh.L));
  b.pow_result = a.take<uint32_t>(4);
  b.chan = a.take<FriChannelDev>(1);
  b.zero_flag = a.take<uint32_t>(4);
  b.scratch = a.take<uint8_t>(GATHER_SCRATCH);
  return b;
}
size_t xor_workspace_bytes(const XorShape& sh) {
  Arena a{nullptr, 0, SIZE_MAX};
  xor_carve(a, sh);
  return a.off + 256;
}

inline uint32_t grid_of(uint64_t n) { return (uint32_t)std::min<uint64_t>((n + 255) / 256, 148 * 16); }

#define SB_CK(expr)                                                                                    \
  do {                                                                                                 \
    cudaError_t _e = (expr);                                                                           \
    if (_e != cudaSuccess) return fail(E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

}  // namespace

size_t LogupXorProver::workspace_bytes(uint32_t log_n, uint32_t log_table, uint32_t log_blowup,
                                       uint32_t log_last_layer) {
  const uint32_t L = std::max(log_n, log_table);
  const uint32_t last_log = log_last_layer + log_blowup;
  const uint32_t LDE = L + log_blowup;
  if (last_log + 1 > LDE) return 0;
  return xor_workspace_bytes(XorShape{L, log_blowup, log_table, (LDE - 1) - last_log});
}

LogupXorProver::LogupXorProver(Context* ctx) : ctx_(ctx) {
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, least);
  cudaStreamCreateWithPriority(&fast_, cudaStreamNonBlocking, greatest);
  cudaMallocHost(&pinned_, PINNED_BYTES);
}

LogupXorProver::~LogupXorProver() {
  if (pinned_) cudaFreeHost(pinned_);
  if (fast_) cudaStreamDestroy(fast_);
  if (stream_) cudaStreamDestroy(stream_);
}

int32_t LogupXorProver::prove(const XorRequest& req, std::string& out) {
  const PcsConfig& cfg = req.config;
  const uint32_t B = cfg.log_blowup_factor;
  if (req.log_n < 1 || req.log_n > 22 || (req.log_table != 8 && req.log_table != 16) || B < 1 || B > 4 ||
      cfg.n_queries == 0 || cfg.n_queries > 4096 || cfg.pow_bits > 64)
    return fail(E_INVALID, "unsupported XOR-lookup shape or configuration");
  const uint32_t L = std::max(req.log_n, req.log_table), LDE = L + B, CL = L + 1;
  if (LDE > ctx_->tables.tower_log + 1 || cfg.log_last_layer_degree_bound + B + 1 > LDE)
    return fail(E_INVALID, "domain too large for the context or last layer too large");
  if (!pinned_ || !stream_ || !fast_) return fail(E_OOM, "stream or pinned staging allocation failed");
  cudaSetDevice(ctx_->device);
  const uint64_t N = 1ull << L, NL = 1ull << LDE, NC = 1ull << CL;
  const uint32_t last_log = cfg.log_last_layer_degree_bound + B;
  const uint32_t n_inner = (LDE - 1) - last_log;
  const DeviceTables& T = ctx_->tables;
  cudaStream_t s = stream_, fs = fast_;
  uint8_t* pin = pinned_;

  // Workspace from the stream-ordered pool, returned on every exit path.
  XorShape shape{L, B, req.log_table, n_inner};
  const size_t need = xor_workspace_bytes(shape);
  uint8_t* arena_mem = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&arena_mem), need, s) != cudaSuccess) {
    cudaGetLastError();
    return fail(E_OOM, "device workspace allocation failed");
  }
  struct Release {
    uint8_t* p;
    cudaStream_t s, fs;
    ~Release() {
      cudaStreamSynchronize(fs);
      cudaFreeAsync(p, s);
    }
  } release{arena_mem, s, fs};
  Arena arena{arena_mem, 0, need};
  XorBufs b = xor_carve(arena, shape);
  uint32_t* pre = b.vals;
  uint32_t* mainc = b.vals + 4 * N;
  uint32_t* inter = b.vals + 8 * N;

  Channel ch;
  {
    QM31 c = qmake(cfg.pow_bits, B, cfg.n_queries, cfg.log_last_layer_degree_bound);
    ch.mix_felts(&c, 1);
  }
  // Trees 0 and 1.
  SB_CK(cudaMemsetAsync(b.hist, 0, 4ull << req.log_table, s));
  k_xor_air_trace<<<grid_of(N), 256, 0, s>>>(L, req.log_n, req.log_table, req.seed, pre, mainc, b.hist);
  note_launch();
  k_xor_air_mult<<<grid_of(N), 256, 0, s>>>(L, req.log_table, b.hist, mainc + 3 * N);
  note_launch();
  SB_CK(cudaGetLastError());
  uint8_t roots[4][32];
  auto commit = [&](int t, uint32_t first_col, uint32_t n_cols) -> int32_t {
    SB_CK(interpolate_extend(T, L, B, n_cols, b.vals + first_col * N, N, b.coeffs + first_col * N, N,
                             b.lde + first_col * NL, NL, s));
    SB_CK(merkle_commit(LDE, n_cols, b.lde + first_col * NL, NL, b.tree[t], s));
    SB_CK(cudaMemcpyAsync(pin, b.tree[t] + (2 * NL - 2) * 32, 32, cudaMemcpyDeviceToHost, s));
    SB_CK(cudaStreamSynchronize(s));
    std::memcpy(roots[t], pin, 32);
    ch.mix_root(roots[t]);
    return OK;
  };
  int32_t rc = commit(0, 0, 4);
  if (rc != OK) return rc;
  if ((rc = commit(1, 4, 4)) != OK) return rc;
  {
    uint32_t st[2] = {req.log_n, req.log_table};
    ch.mix_words(st, 2);
  }
  if (req.has_channel_seed) ch.mix_u64(req.channel_seed);

  // Interaction: LogUp columns of both uses (the a20 kernels), tree 2.
  const QM31 z = ch.draw_secure_felt();
  const QM31 alpha = ch.draw_secure_felt();
  const QM31 alpha2 = qsq(alpha);
  QM31 claimed[2];
  {
    LogupParams lp{};
    lp.log_rows = L;
    lp.n_uses = 1;
    lp.batch = 1;
    lp.order = 1;
    lp.alphas[0] = qone();
    lp.alphas[1] = alpha;
    lp.alphas[2] = alpha2;
    lp.z = z;
    LogupUse& u = lp.uses[0];
    u.n_words = 3;
    SB_CK(cudaMemsetAsync(b.zero_flag, 0, 4, s));
    u.words[0] = mainc; u.words[1] = mainc + N; u.words[2] = mainc + 2 * N;
    u.multiplicity = pre + 3 * N;
    u.negate = 0;
    SB_CK(logup_interaction(lp, inter, N, b.claimed, b.logup_scratch, b.zero_flag, s));
    u.words[0] = pre; u.words[1] = pre + N; u.words[2] = pre + 2 * N;
    u.multiplicity = mainc + 3 * N;
    u.negate = 1;
    SB_CK(logup_interaction(lp, inter + 4 * N, N, b.claimed + 1, b.logup_scratch, b.zero_flag, s));
    SB_CK(cudaMemcpyAsync(pin, b.claimed, 2 * sizeof(QM31), cudaMemcpyDeviceToHost, s));
    SB_CK(cudaMemcpyAsync(pin + 64, b.zero_flag, 4, cudaMemcpyDeviceToHost, s));
    SB_CK(cudaStreamSynchronize(s));
    std::memcpy(claimed, pin, 2 * sizeof(QM31));
    uint32_t zf;
    std::memcpy(&zf, pin + 64, 4);
    if (zf) return fail(E_DIVISION_BY_ZERO, "LogUp denominator is zero (retry with another channel seed)");
  }
  if ((rc = commit(2, 8, 8)) != OK) return rc;
  ch.mix_felts(claimed, 2);

  // Composition on CanonicCoset(L+1).
  const QM31 random_coeff = ch.draw_secure_felt();
  if (B != 1) SB_CK(extend(T, L, 1, 16, b.coeffs, N, b.eval_c, NC, s));
  {
    XorCompParams p{};
    p.alpha1 = alpha;
    p.alpha2 = alpha2;
    p.z = z;
    p.rc = random_coeff;
    const uint32_t inv_n = minv((uint32_t)(N % P));
    p.shift_main = qmulm(claimed[0], inv_n);
    p.shift_table = qmulm(claimed[1], inv_n);
    const PointTable& pt = host_points();
    CircleDomain cd = canonic_domain(CL);
    Coset trace_coset = coset_odds(L);
    p.den0 = minv(coset_vanishing_m(pt, trace_coset, pt.at(cd.index_at(0))));
    p.den1 = minv(coset_vanishing_m(pt, trace_coset, pt.at(cd.index_at(1))));
    p.L = L;
    p.CL = CL;
    k_xor_composition<<<grid_of(NC), 256, 0, s>>>(p, b.eval_c, B == 1 ? NL : NC, b.comp, NC);
    note_launch();
    SB_CK(cudaGetLastError());
  }
  SB_CK(fft_columns(T, true, CL, 4, b.comp, NC, s));
  SB_CK(extend(T, L, B, 4, b.comp, NC, b.comp_lde, NL, s));
  SB_CK(extend(T, L, B, 4, b.comp + N, NC, b.comp_lde + 4 * NL, NL, s));
  SB_CK(merkle_commit(LDE, 8, b.comp_lde, NL, b.tree[3], s));
  SB_CK(cudaMemcpyAsync(pin, b.tree[3] + (2 * NL - 2) * 32, 32, cudaMemcpyDeviceToHost, s));
  SB_CK(cudaStreamSynchronize(s));
  std::memcpy(roots[3], pin, 32);
  ch.mix_root(roots[3]);

  // OODS samples: P for every column, P - g (previous row) for tree 2.
  const PointQ oods = random_secure_point(ch);
  PointQ prev;
  {
    const PointTable& pt = host_points();
    PointM g = pt.at(coset_odds(L).step);
    prev = qpadd(oods, PointQ{qbase(g.x), qneg(qbase(g.y))});
  }
  // oods_out: [0..16) the 16 trace-tree columns at P, [16..24) tree 2 at P - g, [24..32) composition.
  SB_CK(eval_at_point(T, L, 16, b.coeffs, N, oods, nullptr, b.oods_partial, b.oods_out, fs));
  SB_CK(eval_at_point(T, L, 8, b.coeffs + 8 * N, N, prev, nullptr, b.oods_partial, b.oods_out + 16, fs));
  SB_CK(eval_at_point(T, L, 4, b.comp, NC, oods, nullptr, b.oods_partial, b.oods_out + 24, fs));
  SB_CK(eval_at_point(T, L, 4, b.comp + N, NC, oods, nullptr, b.oods_partial, b.oods_out + 28, fs));
  SB_CK(cudaMemcpyAsync(pin, b.oods_out, 32 * sizeof(QM31), cudaMemcpyDeviceToHost, fs));
  SB_CK(cudaStreamSynchronize(fs));
  std::vector<QM31> at_p(32);
  std::memcpy(at_p.data(), pin, 32 * sizeof(QM31));
  // Mix order: tree by tree, column by column, a column's samples in mask order (previous, current).
  {
    std::vector<QM31> flat;
    for (int c = 0; c < 8; ++c) flat.push_back(at_p[c]);
    for (int c = 0; c < 8; ++c) { flat.push_back(at_p[16 + c]); flat.push_back(at_p[8 + c]); }
    for (int c = 0; c < 8; ++c) flat.push_back(at_p[24 + c]);
    ch.mix_felts(flat.data(), flat.size());
  }
  const QM31 quot_coeff = ch.draw_secure_felt();

  // Quotient batches. Random powers run over (tree, column, sample) with a two-sample column's
  // periodicity sample first; batch 0 is the point P, batch 1 the point P - g.
  {
    struct Entry { const uint32_t* col; QM31 v; QM31 rp; };
    std::vector<Entry> b0, b1;
    QM31 rp = qone();
    auto next = [&]() { QM31 r = rp; rp = qmul(rp, quot_coeff); return r; };
    for (int c = 0; c < 8; ++c) b0.push_back({b.lde + (size_t)c * NL, at_p[c], next()});
    for (int c = 0; c < 8; ++c) {
      const uint32_t* col = b.lde + (size_t)(8 + c) * NL;
      b0.push_back({col, at_p[8 + c], next()});        // periodicity sample at P
      b1.push_back({col, at_p[16 + c], next()});       // P - g
      b0.push_back({col, at_p[8 + c], next()});        // P
    }
    for (int c = 0; c < 8; ++c) b0.push_back({b.comp_lde + (size_t)c * NL, at_p[24 + c], next()});
    QM31* hc = reinterpret_cast<QM31*>(pin);
    const uint32_t** hp = reinterpret_cast<const uint32_t**>(pin + 16 * 1024);
    QuotientBatchDev* hb = reinterpret_cast<QuotientBatchDev*>(pin + 32 * 1024);
    uint32_t at = 0;
    int bi = 0;
    for (const std::vector<Entry>* bv : {&b0, &b1}) {
      const PointQ& pnt = bi == 0 ? oods : prev;
      QM31 cy = qsub(qconj(pnt.y), pnt.y);
      QM31 sum_a = qzero(), sum_b = qzero();
      for (const Entry& e : *bv) {
        QM31 a = qsub(qconj(e.v), e.v);
        QM31 bb = qsub(qmul(e.v, cy), qmul(a, pnt.y));
        hc[at] = qmul(e.rp, cy);
        hp[at] = e.col;
        sum_a = qadd(sum_a, qmul(e.rp, a));
        sum_b = qadd(sum_b, qmul(e.rp, bb));
        ++at;
      }
      hb[bi].point = pnt;
      hb[bi].sum_a = sum_a;
      hb[bi].sum_b = sum_b;
      hb[bi].first = at - (uint32_t)bv->size();
      hb[bi].count = (uint32_t)bv->size();
      ++bi;
    }
    SB_CK(cudaMemcpyAsync(b.quot_c, hc, at * sizeof(QM31), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.col_ptrs, hp, at * sizeof(void*), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.batch, hb, 2 * sizeof(QuotientBatchDev), cudaMemcpyHostToDevice, fs));
    SB_CK(accumulate_quotients(T, LDE, 2, b.batch, b.col_ptrs, b.quot_c, b.quot, NL, fs));
  }

  // Tail: FRI, proof of work, queries, decommitment.
  FriBuffers fbuf{b.quot, b.tree_q, b.line, b.line_tree, b.pow_result, b.chan};
  FriResult fr;
  {
    std::string ferr;
    int32_t frc = fri_pow_queries(T, ctx_->sm_count, ch, cfg, LDE, n_inner, last_log, fbuf, pin, s, fs, nullptr,
                                  nullptr, fr, ferr);
    if (frc != OK) return fail(frc, ferr);
  }
  DecommitPlan plan;
  {
    for (int t = 0; t < 4; ++t) {
      std::vector<const uint32_t*> cols;
      const uint32_t ncols = t == 0 || t == 1 ? 4 : 8;
      const uint32_t* base = t == 3 ? b.comp_lde : b.lde + (size_t)(t == 0 ? 0 : t == 1 ? 4 : 8) * NL;
      for (uint32_t c = 0; c < ncols; ++c) cols.push_back(base + (size_t)c * NL);
      plan.add_tree(b.tree[t], LDE, cols, fr.queries);
    }
    plan.add_fri(fbuf, LDE, n_inner, fr.queries);
    std::string gerr;
    int32_t grc = plan.gather(b.scratch, GATHER_SCRATCH, pin, PINNED_BYTES, fs, nullptr, gerr);
    if (grc != OK) return fail(grc, gerr);
  }

  // Wire encoding: the wide-Fibonacci proof layout with four trees, claimed sums and the
  // statement (log_n, log_table).
  Json j;
  j.reserve(3 << 20);
  j.lit("{\"config\":{\"pow_bits\":"); j.u(cfg.pow_bits);
  j.lit(",\"fri_config\":{\"log_blowup_factor\":"); j.u(B);
  j.lit(",\"log_last_layer_degree_bound\":"); j.u(cfg.log_last_layer_degree_bound);
  j.lit(",\"n_queries\":"); j.u(cfg.n_queries);
  j.lit(",\"fold_step\":1},\"lifting_log_size\":null},\"statement\":{\"log_n\":"); j.u(req.log_n);
  j.lit(",\"log_table\":"); j.u(req.log_table);
  j.lit("},\"commitments\":[");
  for (int t = 0; t < 4; ++t) { if (t) j.ch(','); j.hash(roots[t]); }
  j.lit("],\"claimed_sums\":["); j.qm(claimed[0]); j.ch(','); j.qm(claimed[1]);
  j.lit("],\"sampled_values\":[[");
  for (int c = 0; c < 4; ++c) { if (c) j.ch(','); j.ch('['); j.qm(at_p[c]); j.ch(']'); }
  j.lit("],[");
  for (int c = 0; c < 4; ++c) { if (c) j.ch(','); j.ch('['); j.qm(at_p[4 + c]); j.ch(']'); }
  j.lit("],[");
  for (int c = 0; c < 8; ++c) {
    if (c) j.ch(',');
    j.ch('['); j.qm(at_p[16 + c]); j.ch(','); j.qm(at_p[8 + c]); j.ch(']');
  }
  j.lit("],[");
  for (int c = 0; c < 8; ++c) { if (c) j.ch(','); j.ch('['); j.qm(at_p[24 + c]); j.ch(']'); }
  j.lit("]],\"decommitments\":[");
  for (size_t t = 0; t < 4; ++t) { if (t) j.ch(','); j.lit("{\"hash_witness\":"); plan.json_witness(j, t); j.ch('}'); }
  j.lit("],\"queried_values\":[");
  for (size_t t = 0; t < 4; ++t) { if (t) j.ch(','); plan.json_queried(j, t); }
  j.lit("],\"proof_of_work\":"); j.u(fr.nonce);
  j.lit(",\"fri_proof\":");
  plan.json_fri(j, fr);
  j.ch('}');

  // Self-checks: the lookup balances and the composition matches the constraints at P.
  if (!qiszero(qadd(claimed[0], claimed[1]))) return fail(E_CONSTRAINTS, "LogUp claimed sums do not cancel");
  {
    const QM31 basis[4] = {qone(), qmake(0, 1, 0, 0), qmake(0, 0, 1, 0), qmake(0, 0, 0, 1)};
    QM31 left = qzero(), right = qzero();
    for (int k = 0; k < 4; ++k) {
      left = qadd(left, qmul(at_p[24 + k], basis[k]));
      right = qadd(right, qmul(at_p[28 + k], basis[k]));
    }
    PointQ pp = oods;
    for (uint32_t i = 0; i + 2 < CL; ++i) pp = qpadd(pp, pp);
    const QM31 comp_oods = qadd(left, qmul(pp.x, right));
    auto sv = [&](int first) {  // QM31 of a tree-2 secure column from its 4 coordinate samples
      QM31 r = qzero();
      for (int k = 0; k < 4; ++k) r = qadd(r, qmul(at_p[first + k], basis[k]));
      return r;
    };
    const QM31 sm = sv(8), sm_prev = sv(16), st = sv(12), st_prev = sv(20);
    const QM31 inv_n = qbase(minv((uint32_t)(N % P)));
    const QM31 d_main = qsub(qadd(qadd(at_p[4], qmul(alpha, at_p[5])), qmul(alpha2, at_p[6])), z);
    const QM31 d_table = qsub(qadd(qadd(at_p[0], qmul(alpha, at_p[1])), qmul(alpha2, at_p[2])), z);
    const QM31 c_main = qsub(qmul(qadd(qsub(sm, sm_prev), qmul(claimed[0], inv_n)), d_main), at_p[3]);
    const QM31 c_table = qadd(qmul(qadd(qsub(st, st_prev), qmul(claimed[1], inv_n)), d_table), at_p[7]);
    Coset tc = coset_odds(L);
    const PointTable& pt = host_points();
    PointM ini = pt.at(tc.initial), hs = pt.at(tc.step / 2);
    PointQ q = qpadd(qpadd(oods, PointQ{qbase(ini.x), qneg(qbase(ini.y))}), PointQ{qbase(hs.x), qbase(hs.y)});
    QM31 x = q.x;
    for (uint32_t i = 1; i < tc.log_size; ++i) x = qdouble_x(x);
    const QM31 expect = qmul(qadd(qmul(random_coeff, c_main), c_table), qinv(x));
    if (!qeq(expect, comp_oods)) return fail(E_CONSTRAINTS, "constraints not satisfied at the OODS point");
  }
  out = j.str();
  return OK;
}

}  // namespace sb
