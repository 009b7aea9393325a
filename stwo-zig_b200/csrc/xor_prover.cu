// LogUp XOR-lookup AIR prover on one device stream.
//
// The reference has no such AIR (its LogUp machinery is the relation graph of
// src/backends/metal/shaders/core/relation.metal and cumulativeColumn of
// src/frontends/riscv/air/logup.zig); this AIR is built from the same pieces and the
// reference's lifted PCS, with components of different sizes, every stage on the device:
//
//   sizes     main component M: 2^n rows (n = log_n); table component T: 2^t rows
//             (t = log_table); L = max(n, t). A component's logical row k (coset order) is
//             stored at bitrev(circle index of k) at its own size, as in
//             src/examples/wide_fibonacci/trace.zig:159-162
//   tree 0    preprocessed (T): ta, tb, tc = ta ^ tb, table row k = ta * 2^w + tb for operands
//             of w = t / 2 bits (the layout of src/frontends/riscv/air/preprocessed/bitwise.zig:17-35)
//   tree 1    main: a, b (seeded uniform w-bit values), c = a ^ b (M); m = multiplicity of table
//             row k among M's rows (T)
//   draw      z, alpha; alphas = (1, alpha, alpha^2)
//   tree 2    interaction: S_M (M) and S_T (T), QM31 as 4 columns each: the coset-order cumulative
//             sums with the total/N shift (N = the component's rows) of 1 / (a + alpha b + alpha^2 c - z)
//             and of -m / (ta + alpha tb + alpha^2 tc - z); their totals are the claimed sums
//   mix       both claimed sums; the verifier requires them to add to zero
//   tree 3    composition on CanonicCoset(L+1): rc * C_M / Z_M + C_T / Z_T, split in halves, with
//             C = (S(x) - S(x g^-1) + claimed / N) * d(x) - numerator(x) and Z the component's
//             vanishing polynomial. A component of 2^k rows enters lifted (src/prover/vcs_lifted/
//             leaves.zig:104-115): at position r of a domain of 2^(K+L-k) points it takes its own
//             value at ((r >> (L-k+1)) << 1) + (r & 1), i.e. its polynomial at the point doubled L-k
//             times; one trace-row step at size 2^L doubles to one row step at size 2^k
//   samples   every column at the OODS point P, tree 2 also at P - g_L (the previous row at the
//             maximal size, src/frontends/riscv/air/logup.zig:45-48): a column of 2^k rows is
//             evaluated at those points doubled L-k times
//   quotients on the lifting domain of log size L+B (src/core/pcs/quotients/samples.zig:163-300):
//             random powers over (tree, column, sample), a two-sample column's periodicity sample
//             first, at its current point plus the lifting generator doubled to the column's log
//             size (the identity for k = L), batches by point in order of first appearance
//   trees     trees 1 and 2 are lifted Merkle trees over columns of both sizes (2^(L+B) leaves);
//             tree 0 is committed at its own size and queried at the lifting domain's positions
//             mapped down (preparePreprocessedQueryPositions, src/core/pcs/utils.zig:292-314)
//   tail      FRI, proof of work, queries and decommitment as for wide-Fibonacci.
#include <algorithm>
#include <cstring>

#include "alloc.hpp"
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

// Main component at storage position s of 2^n rows; counts table-row hits.
__global__ void k_xor_main(uint32_t n, uint32_t log_table, uint64_t seed, uint32_t* a_col, uint32_t* b_col,
                           uint32_t* c_col, uint32_t* hist) {
  const uint32_t N = 1u << n, w = log_table / 2, wmask = (1u << w) - 1;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const uint32_t k = coset_row_of(s, n);
    const uint64_t x = xor_mix(seed ^ (0xD6E8FEB86659FD93ull * ((uint64_t)k + 1)));
    const uint32_t a = (uint32_t)x & wmask, b = (uint32_t)(x >> 8) & wmask;
    atomicAdd(hist + (a << w | b), 1u);
    a_col[s] = a;
    b_col[s] = b;
    c_col[s] = a ^ b;
  }
}

// Table component at storage position s of 2^t rows: the table row and its multiplicity.
__global__ void k_xor_table(uint32_t t, const uint32_t* hist, uint32_t* ta_col, uint32_t* tb_col, uint32_t* tc_col,
                            uint32_t* m_col) {
  const uint32_t N = 1u << t, w = t / 2, wmask = (1u << w) - 1;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const uint32_t k = coset_row_of(s, t);
    const uint32_t ta = k >> w, tb = k & wmask;
    ta_col[s] = ta;
    tb_col[s] = tb;
    tc_col[s] = ta ^ tb;
    m_col[s] = hist[k];
  }
}

// dst (2^big words per column) = src (2^small words per column) lifted: position r takes
// ((r >> (big - small + 1)) << 1) + (r & 1) (src/prover/vcs_lifted/leaves.zig:104-115).
__global__ void k_lift_columns(uint32_t n_cols, uint32_t small, uint32_t big, const uint32_t* __restrict__ src,
                               uint64_t ss, uint32_t* dst, uint64_t ds) {
  const uint64_t n = 1ull << big;
  const uint32_t sh = big - small + 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * n_cols;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = i >> big, r = i & (n - 1);
    dst[c * ds + r] = src[c * ss + (((r >> sh) << 1) | (r & 1))];
  }
}

struct XorCompParams {
  QM31 alpha1, alpha2, z, rc, shift_main, shift_table;
  uint32_t den_main[2], den_table[2];
  uint32_t L, CL;
};

__device__ __forceinline__ QM31 ld_q(const uint32_t* c, uint64_t stride, uint32_t r) {
  return qmake(c[r], c[stride + r], c[2 * stride + r], c[3 * stride + r]);
}

// Column slots of the trace trees (each slot a column; tree 0: 0-2, tree 1: 3-6, tree 2: 7-14).
constexpr uint32_t XS_TA = 0, XS_A = 3, XS_M = 6, XS_SM = 7, XS_ST = 11, XS_COLS = 15;

// Composition on CanonicCoset(L+1) from the 15 lifted trace columns (slot order) of 2^CL, stride.
__global__ void __launch_bounds__(256) k_xor_composition(const __grid_constant__ XorCompParams p,
                                                         const uint32_t* __restrict__ cols, uint64_t stride,
                                                         uint32_t* out, uint64_t out_stride) {
  const uint32_t NC = 1u << p.CL;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < NC; r += gridDim.x * blockDim.x) {
    // x g^-1 is two steps back on the doubled coset; lifted, it is one row back at a component's size.
    const uint32_t j = coset_row_of(r, p.CL);
    const uint32_t rp = storage_of((j + NC - 2) & (NC - 1), p.CL);
    const uint32_t ta = cols[XS_TA * stride + r], tb = cols[(XS_TA + 1) * stride + r],
                   tc = cols[(XS_TA + 2) * stride + r];
    const uint32_t a = cols[XS_A * stride + r], b = cols[(XS_A + 1) * stride + r], c = cols[(XS_A + 2) * stride + r],
                   m = cols[XS_M * stride + r];
    const QM31 sm = ld_q(cols + XS_SM * stride, stride, r), sm_prev = ld_q(cols + XS_SM * stride, stride, rp);
    const QM31 st = ld_q(cols + XS_ST * stride, stride, r), st_prev = ld_q(cols + XS_ST * stride, stride, rp);
    const QM31 d_main = qsub(qadd(qadd(qbase(a), qmulm(p.alpha1, b)), qmulm(p.alpha2, c)), p.z);
    const QM31 d_table = qsub(qadd(qadd(qbase(ta), qmulm(p.alpha1, tb)), qmulm(p.alpha2, tc)), p.z);
    const QM31 c_main = qsub(qmul(qadd(qsub(sm, sm_prev), p.shift_main), d_main), qone());
    const QM31 c_table = qadd(qmul(qadd(qsub(st, st_prev), p.shift_table), d_table), qbase(m));
    const uint32_t half = r >> p.L;
    const QM31 q = qadd(qmulm(qmul(p.rc, c_main), p.den_main[half]), qmulm(c_table, p.den_table[half]));
    out[r] = q.c0.a;
    out[out_stride + r] = q.c0.b;
    out[2 * out_stride + r] = q.c1.a;
    out[3 * out_stride + r] = q.c1.b;
  }
}

struct XorShape {
  uint32_t L, B, log_n, log_table, n_inner;
};
struct XorBufs {
  uint32_t *vals, *coeffs, *lde_own, *lde, *eval_own, *eval_c, *comp, *comp_lde, *quot, *hist;
  uint8_t *tree[4], *tree_q, *scratch;
  std::vector<uint32_t*> line;
  std::vector<uint8_t*> line_tree;
  QM31 *oods_partial, *oods_out, *quot_c, *claimed, *logup_scratch;
  const uint32_t** col_ptrs;
  const uint32_t** tree_cols;  // lifted-commit column pointers (8 per tree)
  uint32_t* tree_logs;         // and log sizes
  QuotientBatchDev* batch;
  uint32_t *pow_result, *zero_flag;
  FriChannelDev* chan;
};
// Slots of 2^L words (values, coefficients: a column of 2^k rows uses the first 2^k words) and of
// 2^(L+B) words (own-size LDE, lifted LDE).
XorBufs xor_carve(Arena& a, const XorShape& sh) {
  const uint64_t N = 1ull << sh.L, NL = N << sh.B, NC = N << 1;
  const uint32_t LDE = sh.L + sh.B;
  const uint64_t NT0 = 1ull << (sh.log_table + sh.B);  // tree 0 leaves
  XorBufs b{};
  b.vals = a.take<uint32_t>(XS_COLS * N);
  b.coeffs = a.take<uint32_t>(XS_COLS * N);
  b.lde_own = a.take<uint32_t>(XS_COLS * NL);
  b.lde = a.take<uint32_t>(XS_COLS * NL);
  b.eval_own = sh.B == 1 ? nullptr : a.take<uint32_t>(XS_COLS * NC);
  b.eval_c = sh.B == 1 ? b.lde : a.take<uint32_t>(XS_COLS * NC);
  b.comp = a.take<uint32_t>(4 * NC);
  b.comp_lde = a.take<uint32_t>(8 * NL);
  b.quot = a.take<uint32_t>(4 * NL);
  b.hist = a.take<uint32_t>(1u << sh.log_table);
  b.tree[0] = a.take<uint8_t>((2 * NT0 - 1) * 32);
  for (int t = 1; t < 4; ++t) b.tree[t] = a.take<uint8_t>((2 * NL - 1) * 32);
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
  b.tree_cols = a.take<const uint32_t*>(16);
  b.tree_logs = a.take<uint32_t>(16);
  b.batch = a.take<QuotientBatchDev>(4);
  b.claimed = a.take<QM31>(2);
  b.logup_scratch = a.take<QM31>(logup_scratch_count(sh.L));
  b.pow_result = a.take<uint32_t>(4);
  b.zero_flag = a.take<uint32_t>(4);
  b.chan = a.take<FriChannelDev>(1);
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
  return xor_workspace_bytes(XorShape{L, log_blowup, log_n, log_table, (LDE - 1) - last_log});
}

LogupXorProver::LogupXorProver(Context* ctx) : ctx_(ctx) {
  const StreamPriorities pr = stream_priorities();
  cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, pr.bulk);
  cudaStreamCreateWithPriority(&fast_, cudaStreamNonBlocking, pr.greatest);
  cudaStreamCreateWithPriority(&pow_, cudaStreamNonBlocking, pr.least);
}

LogupXorProver::~LogupXorProver() {
  if (pinned_) cudaFreeHost(pinned_);
  if (fast_) cudaStreamDestroy(fast_);
  if (pow_) cudaStreamDestroy(pow_);
  if (stream_) cudaStreamDestroy(stream_);
}

int32_t LogupXorProver::reserve_staging() {
  if (pinned_) return OK;
  cudaSetDevice(ctx_->device);
  if (host_malloc_pinned(reinterpret_cast<void**>(&pinned_), PINNED_BYTES) != cudaSuccess) {
    pinned_ = nullptr;
    cudaGetLastError();
    return fail(E_OOM, "pinned staging allocation failed");
  }
  return OK;
}

int32_t LogupXorProver::prove(const XorRequest& req, std::string& out) {
  const PcsConfig& cfg = req.config;
  const uint32_t B = cfg.log_blowup_factor;
  if (req.log_n < 1 || req.log_n > 22 || (req.log_table != 8 && req.log_table != 16) || B < 1 || B > 4 ||
      cfg.n_queries == 0 || cfg.n_queries > 4096 || cfg.pow_bits > MAX_POW_BITS)
    return fail(E_INVALID, "unsupported XOR-lookup shape or configuration");
  const uint32_t n = req.log_n, t = req.log_table;
  const uint32_t L = std::max(n, t), LDE = L + B, CL = L + 1;
  if (LDE > ctx_->tables.tower_log + 1 || cfg.log_last_layer_degree_bound + B + 1 > LDE)
    return fail(E_INVALID, "domain too large for the context or last layer too large");
  if (!stream_ || !fast_ || !pow_) return fail(E_CUDA, "stream creation failed");
  cudaSetDevice(ctx_->device);
  // Pinned staging on first use (a failed allocation leaves the prover usable for the next call).
  if (int32_t rc = reserve_staging(); rc != OK) return rc;
  const uint64_t N = 1ull << L, NL = 1ull << LDE, NC = 1ull << CL;
  const uint32_t last_log = cfg.log_last_layer_degree_bound + B;
  const uint32_t n_inner = (LDE - 1) - last_log;
  const DeviceTables& T = ctx_->tables;
  cudaStream_t s = stream_, fs = fast_;
  uint8_t* pin = pinned_;

  // Workspace from the stream-ordered pool, returned on every exit path.
  XorShape shape{L, B, n, t, n_inner};
  const size_t need = xor_workspace_bytes(shape);
  uint8_t* arena_mem = nullptr;
  if (dev_malloc_async(reinterpret_cast<void**>(&arena_mem), need, s) != cudaSuccess) {
    cudaGetLastError();
    return fail(E_OOM, "device workspace allocation failed");
  }
  struct Release {
    uint8_t* p;
    cudaStream_t s, fs, ps;
    ~Release() {
      stream_wait(fs);
      stream_wait(ps);
      cudaFreeAsync(p, s);
    }
  } release{arena_mem, s, fs, pow_};
  Arena arena{arena_mem, 0, need};
  XorBufs b = xor_carve(arena, shape);
  // Log size of each slot's column, and its slot pointers.
  uint32_t klog[XS_COLS];
  for (uint32_t c = 0; c < XS_COLS; ++c) klog[c] = (c < XS_A || c == XS_M || c >= XS_ST) ? t : n;
  auto val = [&](uint32_t c) { return b.vals + c * N; };
  auto coef = [&](uint32_t c) { return b.coeffs + c * N; };
  auto lifted = [&](uint32_t c) { return b.lde + c * NL; };  // 2^(L+B): the lifting domain
  // Own-size LDE (2^(k+B)); a full-size column's is its lifted one.
  auto own = [&](uint32_t c) { return klog[c] == L ? lifted(c) : b.lde_own + c * NL; };

  Channel ch;
  {
    QM31 c = qmake(cfg.pow_bits, B, cfg.n_queries, cfg.log_last_layer_degree_bound);
    ch.mix_felts(&c, 1);
  }
  // Trace: main component (2^n rows), table component and multiplicities (2^t rows).
  SB_CK(cudaMemsetAsync(b.hist, 0, 4ull << t, s));
  k_xor_main<<<grid_of(1ull << n), 256, 0, s>>>(n, t, req.seed, val(XS_A), val(XS_A + 1), val(XS_A + 2), b.hist);
  note_launch();
  k_xor_table<<<grid_of(1ull << t), 256, 0, s>>>(t, b.hist, val(XS_TA), val(XS_TA + 1), val(XS_TA + 2), val(XS_M));
  note_launch();
  SB_CK(cudaGetLastError());
  // Interpolate and extend slots [c0, c0 + cnt) of one size k; lift them to the lifting domain.
  auto lde_group = [&](uint32_t c0, uint32_t cnt) -> int32_t {
    const uint32_t k = klog[c0];
    SB_CK(interpolate_extend(T, k, B, cnt, val(c0), N, coef(c0), N, own(c0), NL, s));
    if (k < L) {
      k_lift_columns<<<grid_of(NL * cnt), 256, 0, s>>>(cnt, k + B, LDE, own(c0), NL, lifted(c0), NL);
      note_launch();
      SB_CK(cudaGetLastError());
    }
    return OK;
  };
  uint8_t roots[4][32];
  auto read_root = [&](int tr, uint64_t leaves) -> int32_t {
    SB_CK(cudaMemcpyAsync(pin, b.tree[tr] + (2 * leaves - 2) * 32, 32, cudaMemcpyDeviceToHost, s));
    SB_CK(stream_wait(s));
    std::memcpy(roots[tr], pin, 32);
    if (deadline_.passed()) return fail(E_TIMEOUT, "proof deadline passed after a commitment");
    ch.mix_root(roots[tr]);
    return OK;
  };
  // A lifted tree over slots [c0, c0 + cnt) (columns of both sizes) on 2^(L+B) leaves; the leaf
  // kernel takes the columns in leaf order, stably sorted by log size.
  auto commit_lifted = [&](int tr, uint32_t c0, uint32_t cnt) -> int32_t {
    const uint32_t** hp = reinterpret_cast<const uint32_t**>(pin + 1024);
    uint32_t* hl = reinterpret_cast<uint32_t*>(pin + 2048);
    std::vector<uint32_t> order(cnt);
    for (uint32_t c = 0; c < cnt; ++c) order[c] = c0 + c;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return klog[x] < klog[y]; });
    for (uint32_t c = 0; c < cnt; ++c) { hp[c] = own(order[c]); hl[c] = klog[order[c]] + B; }
    SB_CK(cudaMemcpyAsync(b.tree_cols + 8 * (tr - 1), hp, cnt * sizeof(void*), cudaMemcpyHostToDevice, s));
    SB_CK(cudaMemcpyAsync(b.tree_logs + 8 * (tr - 1), hl, cnt * 4, cudaMemcpyHostToDevice, s));
    SB_CK(merkle_commit_lifted(LDE, cnt, b.tree_cols + 8 * (tr - 1), b.tree_logs + 8 * (tr - 1), b.tree[tr], s));
    return read_root(tr, NL);
  };
  int32_t rc;
  // Tree 0: the preprocessed table at its own size.
  if ((rc = lde_group(XS_TA, 3)) != OK) return rc;
  SB_CK(merkle_commit(t + B, 3, own(XS_TA), NL, b.tree[0], s));
  if ((rc = read_root(0, 1ull << (t + B))) != OK) return rc;
  // Tree 1: a, b, c (2^n), m (2^t).
  if ((rc = lde_group(XS_A, 3)) != OK) return rc;
  if ((rc = lde_group(XS_M, 1)) != OK) return rc;
  if ((rc = commit_lifted(1, XS_A, 4)) != OK) return rc;
  {
    uint32_t st[2] = {n, t};
    ch.mix_words(st, 2);
  }
  if (req.has_channel_seed) ch.mix_u64(req.channel_seed);

  // Interaction: one LogUp column set per component at its own size (the a20 kernels), tree 2.
  const QM31 z = ch.draw_secure_felt();
  const QM31 alpha = ch.draw_secure_felt();
  const QM31 alpha2 = qsq(alpha);
  QM31 claimed[2];
  {
    LogupParams lp{};
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
    lp.log_rows = n;
    u.words[0] = val(XS_A); u.words[1] = val(XS_A + 1); u.words[2] = val(XS_A + 2);
    u.multiplicity = nullptr;  // every main row looks up once
    u.negate = 0;
    SB_CK(logup_interaction(lp, val(XS_SM), N, b.claimed, b.logup_scratch, b.zero_flag, s));
    lp.log_rows = t;
    u.words[0] = val(XS_TA); u.words[1] = val(XS_TA + 1); u.words[2] = val(XS_TA + 2);
    u.multiplicity = val(XS_M);
    u.negate = 1;
    SB_CK(logup_interaction(lp, val(XS_ST), N, b.claimed + 1, b.logup_scratch, b.zero_flag, s));
    SB_CK(cudaMemcpyAsync(pin, b.claimed, 2 * sizeof(QM31), cudaMemcpyDeviceToHost, s));
    SB_CK(cudaMemcpyAsync(pin + 64, b.zero_flag, 4, cudaMemcpyDeviceToHost, s));
    SB_CK(stream_wait(s));
    std::memcpy(claimed, pin, 2 * sizeof(QM31));
    uint32_t zf;
    std::memcpy(&zf, pin + 64, 4);
    if (zf) return fail(E_DIVISION_BY_ZERO, "LogUp denominator is zero (retry with another channel seed)");
  }
  if ((rc = lde_group(XS_SM, 4)) != OK) return rc;
  if ((rc = lde_group(XS_ST, 4)) != OK) return rc;
  if ((rc = commit_lifted(2, XS_SM, 8)) != OK) return rc;
  ch.mix_felts(claimed, 2);

  // Composition on CanonicCoset(L+1) from the lifted evaluations on that domain.
  const QM31 random_coeff = ch.draw_secure_felt();
  if (B != 1) {
    for (uint32_t c0 : {XS_TA, XS_A, XS_M, XS_SM, XS_ST}) {
      const uint32_t cnt = c0 == XS_TA || c0 == XS_A ? 3 : c0 == XS_M ? 1 : 4;
      const uint32_t k = klog[c0];
      uint32_t* dst = b.eval_c + c0 * NC;
      if (k == L) {
        SB_CK(extend(T, k, 1, cnt, coef(c0), N, dst, NC, s));
      } else {
        SB_CK(extend(T, k, 1, cnt, coef(c0), N, b.eval_own + c0 * NC, NC, s));
        k_lift_columns<<<grid_of(NC * cnt), 256, 0, s>>>(cnt, k + 1, CL, b.eval_own + c0 * NC, NC, dst, NC);
        note_launch();
        SB_CK(cudaGetLastError());
      }
    }
  }
  {
    XorCompParams p{};
    p.alpha1 = alpha;
    p.alpha2 = alpha2;
    p.z = z;
    p.rc = random_coeff;
    p.shift_main = qmulm(claimed[0], minv((uint32_t)((1ull << n) % P)));
    p.shift_table = qmulm(claimed[1], minv((uint32_t)((1ull << t) % P)));
    const PointTable& pt = host_points();
    for (int comp = 0; comp < 2; ++comp) {
      const uint32_t k = comp == 0 ? n : t;
      CircleDomain cd = canonic_domain(k + 1);
      Coset trace_coset = coset_odds(k);
      uint32_t* den = comp == 0 ? p.den_main : p.den_table;
      den[0] = minv(coset_vanishing_m(pt, trace_coset, pt.at(cd.index_at(0))));
      den[1] = minv(coset_vanishing_m(pt, trace_coset, pt.at(cd.index_at(1))));
    }
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
  if ((rc = read_root(3, NL)) != OK) return rc;

  // OODS samples: every column at P, tree 2 also at P - g_L; a column of 2^k rows at those
  // points doubled L - k times.
  const PointQ oods = random_secure_point(ch);
  PointQ prev;
  {
    const PointTable& pt = host_points();
    PointM g = pt.at(coset_odds(L).step);
    prev = qpadd(oods, PointQ{qbase(g.x), qneg(qbase(g.y))});
  }
  auto doubled = [&](PointQ pq, uint32_t k) {
    for (uint32_t i = k; i < L; ++i) pq = qpadd(pq, pq);
    return pq;
  };
  // oods_out: [0, 15) slot c at P, [15, 23) slots 7..14 at P - g_L, [24, 32) composition at P.
  {
    struct Group { uint32_t c0, cnt; bool prev; };
    const Group groups[] = {{XS_TA, 3, false}, {XS_A, 3, false}, {XS_M, 1, false}, {XS_SM, 4, true}, {XS_ST, 4, true}};
    for (const Group& gr : groups) {
      const uint32_t k = klog[gr.c0];
      SB_CK(eval_at_point(T, k, gr.cnt, coef(gr.c0), N, doubled(oods, k), nullptr, b.oods_partial,
                          b.oods_out + gr.c0, fs));
      if (gr.prev)
        SB_CK(eval_at_point(T, k, gr.cnt, coef(gr.c0), N, doubled(prev, k), nullptr, b.oods_partial,
                            b.oods_out + XS_COLS + (gr.c0 - XS_SM), fs));
    }
  }
  SB_CK(eval_at_point(T, L, 4, b.comp, NC, oods, nullptr, b.oods_partial, b.oods_out + 24, fs));
  SB_CK(eval_at_point(T, L, 4, b.comp + N, NC, oods, nullptr, b.oods_partial, b.oods_out + 28, fs));
  SB_CK(cudaMemcpyAsync(pin, b.oods_out, 32 * sizeof(QM31), cudaMemcpyDeviceToHost, fs));
  SB_CK(stream_wait(fs));
  std::vector<QM31> at_p(32);
  std::memcpy(at_p.data(), pin, 32 * sizeof(QM31));
  auto cur_v = [&](uint32_t c) { return at_p[c]; };
  auto prev_v = [&](uint32_t c) { return at_p[XS_COLS + (c - XS_SM)]; };
  // Mix order: tree by tree, column by column, a column's samples in mask order (previous, current).
  {
    std::vector<QM31> flat;
    for (uint32_t c = 0; c < XS_SM; ++c) flat.push_back(cur_v(c));
    for (uint32_t c = XS_SM; c < XS_COLS; ++c) { flat.push_back(prev_v(c)); flat.push_back(cur_v(c)); }
    for (int c = 0; c < 8; ++c) flat.push_back(at_p[24 + c]);
    ch.mix_felts(flat.data(), flat.size());
  }
  const QM31 quot_coeff = ch.draw_secure_felt();

  // Quotient batches on the lifting domain. Random powers run over (tree, column, sample) with a
  // two-sample column's periodicity sample first; batches by point in order of first appearance.
  {
    struct Entry { const uint32_t* col; QM31 v; QM31 rp; };
    std::vector<PointQ> points;
    std::vector<std::vector<Entry>> batches;
    auto batch_of = [&](const PointQ& pq) -> std::vector<Entry>& {
      for (size_t i = 0; i < points.size(); ++i)
        if (qeq(points[i].x, pq.x) && qeq(points[i].y, pq.y)) return batches[i];
      points.push_back(pq);
      batches.emplace_back();
      return batches.back();
    };
    QM31 rp = qone();
    auto next = [&]() { QM31 r = rp; rp = qmul(rp, quot_coeff); return r; };
    for (uint32_t c = 0; c < XS_SM; ++c) batch_of(oods).push_back({lifted(c), cur_v(c), next()});
    for (uint32_t c = XS_SM; c < XS_COLS; ++c) {
      // periodicity point: P plus the lifting generator (order 2^(L+B)) doubled k+B times
      PointQ per = oods;
      if (klog[c] < L) {
        PointM h = host_points().at(1u << (31 - L + klog[c]));
        per = qpadd(oods, PointQ{qbase(h.x), qbase(h.y)});
      }
      batch_of(per).push_back({lifted(c), cur_v(c), next()});
      batch_of(prev).push_back({lifted(c), prev_v(c), next()});
      batch_of(oods).push_back({lifted(c), cur_v(c), next()});
    }
    for (int c = 0; c < 8; ++c) batch_of(oods).push_back({b.comp_lde + (size_t)c * NL, at_p[24 + c], next()});
    QM31* hc = reinterpret_cast<QM31*>(pin);
    const uint32_t** hp = reinterpret_cast<const uint32_t**>(pin + 16 * 1024);
    QuotientBatchDev* hb = reinterpret_cast<QuotientBatchDev*>(pin + 32 * 1024);
    uint32_t at = 0;
    for (size_t bi = 0; bi < batches.size(); ++bi) {
      const PointQ& pnt = points[bi];
      QM31 cy = qsub(qconj(pnt.y), pnt.y);
      QM31 sum_a = qzero(), sum_b = qzero();
      for (const Entry& e : batches[bi]) {
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
      hb[bi].first = at - (uint32_t)batches[bi].size();
      hb[bi].count = (uint32_t)batches[bi].size();
    }
    SB_CK(cudaMemcpyAsync(b.quot_c, hc, at * sizeof(QM31), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.col_ptrs, hp, at * sizeof(void*), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.batch, hb, batches.size() * sizeof(QuotientBatchDev), cudaMemcpyHostToDevice, fs));
    // Columns that all start 16-byte aligned may go through the bulk-staged quotient kernel, its
    // status read back with the FRI channel.
    bool aligned = true;
    for (uint32_t i = 0; i < at; ++i) aligned = aligned && (reinterpret_cast<uintptr_t>(hp[i]) & 15) == 0;
    SB_CK(cudaMemsetAsync(&b.chan->quot_status, 0, sizeof(uint32_t), fs));
    SB_CK(accumulate_quotients(T, LDE, (uint32_t)batches.size(), at, b.batch, b.col_ptrs, b.quot_c, b.quot, NL, fs,
                               aligned ? &b.chan->quot_status : nullptr));
  }

  // Tail: FRI, proof of work, queries, decommitment.
  FriBuffers fbuf{b.quot, b.tree_q, b.line, b.line_tree, b.pow_result, b.chan};
  FriResult fr;
  {
    std::string ferr;
    int32_t frc = fri_pow_queries(T, ctx_->sm_count, ch, cfg, LDE, n_inner, last_log, fbuf, pin, pow_ ? pow_ : s, fs, nullptr,
                                  nullptr, deadline_, fr, ferr);
    if (frc != OK) return fail(frc, ferr);
  }
  DecommitPlan plan;
  {
    // Tree 0 is queried at the lifting domain's positions mapped to its own size.
    std::vector<uint64_t> pre_q;
    const uint32_t sh = LDE - (t + B) + 1;
    for (uint64_t q : fr.queries) pre_q.push_back(((q >> sh) << 1) + (q & 1));
    plan.add_tree(b.tree[0], t + B, {own(XS_TA), own(XS_TA + 1), own(XS_TA + 2)}, pre_q);
    plan.add_tree(b.tree[1], LDE, {lifted(XS_A), lifted(XS_A + 1), lifted(XS_A + 2), lifted(XS_M)}, fr.queries);
    std::vector<const uint32_t*> c2;
    for (uint32_t c = XS_SM; c < XS_COLS; ++c) c2.push_back(lifted(c));
    plan.add_tree(b.tree[2], LDE, c2, fr.queries);
    std::vector<const uint32_t*> c3;
    for (int c = 0; c < 8; ++c) c3.push_back(b.comp_lde + (size_t)c * NL);
    plan.add_tree(b.tree[3], LDE, c3, fr.queries);
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
  for (uint32_t c = XS_TA; c < XS_A; ++c) { if (c) j.ch(','); j.ch('['); j.qm(cur_v(c)); j.ch(']'); }
  j.lit("],[");
  for (uint32_t c = XS_A; c < XS_SM; ++c) { if (c != XS_A) j.ch(','); j.ch('['); j.qm(cur_v(c)); j.ch(']'); }
  j.lit("],[");
  for (uint32_t c = XS_SM; c < XS_COLS; ++c) {
    if (c != XS_SM) j.ch(',');
    j.ch('['); j.qm(prev_v(c)); j.ch(','); j.qm(cur_v(c)); j.ch(']');
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
    auto secure = [&](auto get, uint32_t first) {  // QM31 of a secure column from its 4 coordinates
      QM31 r = qzero();
      for (uint32_t k = 0; k < 4; ++k) r = qadd(r, qmul(get(first + k), basis[k]));
      return r;
    };
    auto at = [&](uint32_t i) { return at_p[i]; };
    const QM31 left = secure(at, 24), right = secure(at, 28);
    PointQ pp = oods;
    for (uint32_t i = 0; i + 2 < CL; ++i) pp = qpadd(pp, pp);
    const QM31 comp_oods = qadd(left, qmul(pp.x, right));
    const QM31 sm = secure(cur_v, XS_SM), sm_prev = secure(prev_v, XS_SM);
    const QM31 st = secure(cur_v, XS_ST), st_prev = secure(prev_v, XS_ST);
    const QM31 d_main =
        qsub(qadd(qadd(cur_v(XS_A), qmul(alpha, cur_v(XS_A + 1))), qmul(alpha2, cur_v(XS_A + 2))), z);
    const QM31 d_table =
        qsub(qadd(qadd(cur_v(XS_TA), qmul(alpha, cur_v(XS_TA + 1))), qmul(alpha2, cur_v(XS_TA + 2))), z);
    const QM31 c_main =
        qsub(qmul(qadd(qsub(sm, sm_prev), qmulm(claimed[0], minv((uint32_t)((1ull << n) % P)))), d_main), qone());
    const QM31 c_table =
        qadd(qmul(qadd(qsub(st, st_prev), qmulm(claimed[1], minv((uint32_t)((1ull << t) % P)))), d_table), cur_v(XS_M));
    const PointTable& pt = host_points();
    auto vanishing = [&](uint32_t k) {  // Z of CanonicCoset(k) at P doubled L - k times
      Coset tc = coset_odds(k);
      PointM ini = pt.at(tc.initial), hs = pt.at(tc.step / 2);
      PointQ q = qpadd(qpadd(doubled(oods, k), PointQ{qbase(ini.x), qneg(qbase(ini.y))}), PointQ{qbase(hs.x), qbase(hs.y)});
      QM31 x = q.x;
      for (uint32_t i = 1; i < tc.log_size; ++i) x = qdouble_x(x);
      return x;
    };
    const QM31 expect = qadd(qmul(qmul(random_coeff, c_main), qinv(vanishing(n))), qmul(c_table, qinv(vanishing(t))));
    if (!qeq(expect, comp_oods)) return fail(E_CONSTRAINTS, "constraints not satisfied at the OODS point");
  }
  out = j.str();
  return OK;
}

}  // namespace sb
