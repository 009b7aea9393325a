// Wide-Fibonacci circle-STARK prover on one B200 stream.
//
// Every column, tree and FRI layer of the proof stays resident in HBM; the
// Fiat-Shamir transcript (Blake2s channel) runs on the host and only roots,
// sampled values, the last FRI layer, the nonce and the decommitment gathers
// cross PCIe. The order of transcript operations follows the reference:
// src/examples/common/prover_transaction.zig:222-340 (config mix, preprocessed
// commit, main commit, statement mix), src/prover/prove.zig:209-389
// (composition, OODS), src/prover/pcs/scheme.zig:633-799 (sampled values, FRI,
// PoW, decommit), src/prover/fri.zig:163-850 (FRI layers and decommitment).
#include <algorithm>
#include <array>
#include <cstring>
#include <stdexcept>

#include "blake2s.cuh"
#include "prover.hpp"

namespace sb {

// ---------------------------------------------------------------------------
// Host Blake2s channel (src/core/channel/blake2s.zig:33-280).
// ---------------------------------------------------------------------------
namespace {

struct Channel {
  uint8_t digest[32] = {0};
  uint32_t n_draws = 0;
  void set(const uint8_t d[32]) { std::memcpy(digest, d, 32); n_draws = 0; }
  void mix_words(const uint32_t* w, size_t n) {
    Blake2sHost h;
    h.update(digest, 32);
    if (n) h.update(w, n * 4);
    uint8_t o[32];
    h.finalize(o);
    set(o);
  }
  void mix_felts(const QM31* f, size_t n) {
    std::vector<uint32_t> w(4 * n);
    for (size_t i = 0; i < n; ++i) qstore4(f[i], &w[4 * i]);
    mix_words(w.data(), w.size());
  }
  void mix_u64(uint64_t v) { uint32_t w[2] = {(uint32_t)v, (uint32_t)(v >> 32)}; mix_words(w, 2); }
  void mix_root(const uint8_t root[32]) {  // src/core/vcs_lifted/blake2_merkle.zig:236-247
    Blake2sHost h;
    h.update(digest, 32);
    h.update(root, 32);
    uint8_t o[32];
    h.finalize(o);
    set(o);
  }
  void draw_u32s(uint32_t out[8]) {
    uint8_t in[37];
    std::memcpy(in, digest, 32);
    std::memcpy(in + 32, &n_draws, 4);
    in[36] = 0;
    n_draws += 1;
    Blake2sHost h;
    h.update(in, 37);
    uint8_t o[32];
    h.finalize(o);
    std::memcpy(out, o, 32);
  }
  QM31 draw_secure_felt() {
    for (;;) {
      uint32_t w[8];
      draw_u32s(w);
      bool ok = true;
      for (uint32_t x : w) if (x >= 2 * P) ok = false;
      if (!ok) continue;
      for (uint32_t& x : w) x = mreduce64(x);
      return qmake(w[0], w[1], w[2], w[3]);
    }
  }
};

// randomSecureFieldPoint (src/core/circle.zig:159-167).
PointQ random_secure_point(Channel& ch) {
  QM31 t = ch.draw_secure_felt();
  QM31 t2 = qsq(t);
  QM31 inv = qinv(qadd(t2, qone()));
  return {qmul(qsub(qone(), t2), inv), qmul(qadd(t, t), inv)};
}

// cosetVanishing (src/core/constraints.zig:17-27) on base and secure points.
uint32_t coset_vanishing_m(const PointTable& pt, const Coset& c, PointM p) {
  PointM q = padd(padd(p, pconj(pt.at(c.initial))), pt.at(c.step / 2));
  uint32_t x = q.x;
  for (uint32_t i = 1; i < c.log_size; ++i) x = double_x(x);
  return x;
}

const PointTable& host_points() {
  static std::vector<PointM> t = build_point_table();
  static PointTable pt{t.data()};
  return pt;
}

struct Json {
  std::string s;
  void u(uint64_t v) { s += std::to_string(v); }
  void hash(const uint8_t* h) { s += '['; for (int i = 0; i < 32; ++i) { if (i) s += ','; u(h[i]); } s += ']'; }
  void qm(QM31 q) { uint32_t w[4]; qstore4(q, w); s += '['; for (int i = 0; i < 4; ++i) { if (i) s += ','; u(w[i]); } s += ']'; }
};

// Decommitment plan of a lifted tree at sorted unique leaf positions: the nodes
// whose hashes are witnesses, in proof order (src/prover/vcs_lifted/decommit.zig:154-230).
std::vector<uint64_t> witness_nodes(uint32_t max_log, const std::vector<uint64_t>& positions) {
  std::vector<uint64_t> out, prev = positions, cur;
  for (int layer = (int)max_log - 1; layer >= 0; --layer) {
    cur.clear();
    size_t q = 0;
    while (q < prev.size()) {
      uint64_t first = prev[q];
      bool sib = q + 1 < prev.size() && (first ^ 1) == prev[q + 1];
      if (!sib) out.push_back(merkle_layer_offset(max_log, layer + 1) + (first ^ 1));
      cur.push_back(first >> 1);
      q += sib ? 2 : 1;
    }
    prev.swap(cur);
  }
  return out;
}

struct Arena {
  uint8_t* base;
  size_t off = 0, cap;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    if (off > cap) throw std::runtime_error("arena overflow");
    return p;
  }
};

struct Layout {
  uint32_t n, W, B, L, CL, n_inner, last_log;
  size_t N, NL, NC;
  size_t bytes;
};

Layout layout_for(uint32_t n, uint32_t W, uint32_t B, uint32_t log_last) {
  Layout l{};
  l.n = n; l.W = W; l.B = B; l.L = n + B; l.CL = n + 1;
  l.N = 1ull << n; l.NL = 1ull << l.L; l.NC = 1ull << l.CL;
  l.last_log = log_last + B;
  l.n_inner = (l.L - 1) - l.last_log;
  return l;
}

struct Buffers {
  uint32_t *trace, *coeffs, *lde, *eval_c, *comp, *comp_lde, *quot;
  uint8_t *tree1, *tree2, *tree_q;
  std::vector<uint32_t*> line;   // FRI line layers 0..n_inner (last one is the last layer)
  std::vector<uint8_t*> line_tree;
  QM31 *comp_coeffs, *oods_partial, *oods_out, *quot_c;
  const uint32_t** col_ptrs;
  QuotientBatchDev* batch;
  uint32_t* pow_result;
  uint8_t* scratch;  // gathers
  size_t scratch_bytes;
};

constexpr size_t GATHER_SCRATCH = 8 << 20;

Buffers carve(Arena& a, const Layout& l) {
  Buffers b{};
  b.trace = a.take<uint32_t>(l.W * l.N);
  b.coeffs = a.take<uint32_t>(l.W * l.N);
  b.lde = a.take<uint32_t>(l.W * l.NL);
  b.eval_c = l.B == 1 ? b.lde : a.take<uint32_t>(l.W * l.NC);
  b.comp = a.take<uint32_t>(4 * l.NC);
  b.comp_lde = a.take<uint32_t>(8 * l.NL);
  b.quot = a.take<uint32_t>(4 * l.NL);
  b.tree1 = a.take<uint8_t>((2 * l.NL - 1) * 32);
  b.tree2 = a.take<uint8_t>((2 * l.NL - 1) * 32);
  b.tree_q = a.take<uint8_t>((2 * l.NL - 1) * 32);
  for (uint32_t k = 0; k <= l.n_inner; ++k) {
    size_t sz = 1ull << (l.L - 1 - k);
    b.line.push_back(a.take<uint32_t>(4 * sz));
    b.line_tree.push_back(k < l.n_inner ? a.take<uint8_t>((2 * sz - 1) * 32) : nullptr);
  }
  b.comp_coeffs = a.take<QM31>(l.W);
  size_t parts = eval_at_point_partial_count(l.n, l.W + 8);
  b.oods_partial = a.take<QM31>(parts);
  b.oods_out = a.take<QM31>(l.W + 8);
  b.quot_c = a.take<QM31>(l.W + 8);
  b.col_ptrs = a.take<const uint32_t*>(l.W + 8);
  b.batch = a.take<QuotientBatchDev>(1);
  b.pow_result = a.take<uint32_t>(4);
  b.scratch = a.take<uint8_t>(GATHER_SCRATCH);
  b.scratch_bytes = GATHER_SCRATCH;
  return b;
}

size_t layout_bytes(const Layout& l) {
  Arena a{nullptr, 0, SIZE_MAX};
  carve(a, l);
  return a.off + 256;
}

#define SB_CK(expr)                                                                                    \
  do {                                                                                                 \
    cudaError_t _e = (expr);                                                                           \
    if (_e != cudaSuccess) return fail(E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

}  // namespace

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
Context::~Context() {
  for (WideFibProver* p : pool) delete p;
  if (tables.points) cudaFree(tables.points);
  if (tables.tw) cudaFree(tables.tw);
  if (tables.itw) cudaFree(tables.itw);
  if (small) cudaFree(small);
  if (stream) cudaStreamDestroy(stream);
}

int32_t Context::init(int dev, uint32_t tower_log) {
  device = dev;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= dev) return E_NO_DEVICE;
  if (cudaSetDevice(dev) != cudaSuccess) return E_CUDA;
  cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return E_CUDA;
  // Keep freed stream-ordered allocations cached in this process's default pool
  // instead of returning them to the driver at every synchronization.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  if (cudaMalloc(&small, 256) != cudaSuccess) return E_OOM;
  std::vector<PointM> pts = build_point_table();
  if (cudaMalloc(&tables.points, pts.size() * sizeof(PointM)) != cudaSuccess) return E_OOM;
  if (cudaMemcpy(tables.points, pts.data(), pts.size() * sizeof(PointM), cudaMemcpyHostToDevice) != cudaSuccess)
    return E_CUDA;
  size_t tw_words = (size_t)1 << tower_log;
  if (cudaMalloc(&tables.tw, tw_words * 4) != cudaSuccess) return E_OOM;
  if (cudaMalloc(&tables.itw, tw_words * 4) != cudaSuccess) return E_OOM;
  if (build_twiddle_tower(tables, tower_log, stream) != cudaSuccess) return E_CUDA;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return E_CUDA;
  return OK;
}

WideFibProver* Context::acquire() {
  std::lock_guard<std::mutex> g(mu);
  if (!pool.empty()) {
    WideFibProver* p = pool.back();
    pool.pop_back();
    return p;
  }
  cudaStream_t s;
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  return new WideFibProver(this, s);
}

void Context::release(WideFibProver* p) {
  std::lock_guard<std::mutex> g(mu);
  pool.push_back(p);
}

// ---------------------------------------------------------------------------
// Prover
// ---------------------------------------------------------------------------
WideFibProver::WideFibProver(Context* ctx, cudaStream_t stream) : ctx_(ctx), stream_(stream) {
  for (auto& e : ev_) cudaEventCreate(&e);
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
      cudaStreamCreateWithPriority(&fast_, cudaStreamNonBlocking, greatest) != cudaSuccess) {
    cudaGetLastError();
    fast_ = nullptr;
  }
}

WideFibProver::~WideFibProver() {
  release();
  for (auto& e : ev_) cudaEventDestroy(e);
  if (fast_) cudaStreamDestroy(fast_);
  if (stream_) cudaStreamDestroy(stream_);
}

void WideFibProver::release() {
  if (arena_) cudaFree(arena_);
  if (pinned_) cudaFreeHost(pinned_);
  arena_ = nullptr; pinned_ = nullptr; arena_size_ = 0; pinned_size_ = 0;
  ws_log_n_ = ws_W_ = ws_B_ = 0;
}

size_t WideFibProver::workspace_bytes(uint32_t log_n, uint32_t W, uint32_t B) {
  return layout_bytes(layout_for(log_n, W, B, 0)) + (1 << 20);
}

void WideFibProver::set_transient(bool on) {
  if (on && !transient_ && arena_) {
    cudaFree(arena_);
    arena_ = nullptr;
    arena_size_ = 0;
    ws_log_n_ = ws_W_ = ws_B_ = 0;
  }
  transient_ = on;
}

int32_t WideFibProver::ensure_workspace(uint32_t log_n, uint32_t W, uint32_t B) {
  if (!pinned_) {
    pinned_size_ = GATHER_SCRATCH + (1 << 20);
    if (cudaMallocHost(&pinned_, pinned_size_) != cudaSuccess) { pinned_ = nullptr; return fail(E_OOM, "pinned staging allocation failed"); }
  }
  size_t need = workspace_bytes(log_n, W, B);
  if (transient_) {
    if (cudaMallocAsync(&arena_, need, stream_) != cudaSuccess) {
      arena_ = nullptr;
      cudaGetLastError();
      return fail(E_OOM, "device workspace allocation failed");
    }
    arena_size_ = need;
    ws_log_n_ = log_n; ws_W_ = W; ws_B_ = B;
    return OK;
  }
  if (arena_ && ws_log_n_ == log_n && ws_W_ == W && ws_B_ == B) return OK;
  if (arena_ && arena_size_ >= need) {
    ws_log_n_ = log_n; ws_W_ = W; ws_B_ = B;
    return OK;
  }
  if (arena_) { cudaFree(arena_); arena_ = nullptr; }
  if (cudaMalloc(&arena_, need) != cudaSuccess) { arena_ = nullptr; cudaGetLastError(); return fail(E_OOM, "device workspace allocation failed"); }
  arena_size_ = need;
  ws_log_n_ = log_n; ws_W_ = W; ws_B_ = B;
  return OK;
}

int32_t WideFibProver::prove(const ProveRequest& req, std::string& out, StageTimes* times) {
  const uint32_t n = req.log_n_rows, W = req.sequence_len;
  const PcsConfig& cfg = req.config;
  const uint32_t B = cfg.log_blowup_factor;
  if (n < 1 || n > 22 || W < 2 || W > 1000 || B < 1 || B > 4 || n + B > ctx_->tables.tower_log + 1 ||
      n + 1 > ctx_->tables.tower_log + 1 || cfg.n_queries == 0 || cfg.n_queries > 4096 || cfg.pow_bits > 64)
    return fail(E_INVALID, "unsupported proof shape or configuration");
  if (n + B < cfg.log_last_layer_degree_bound + B + 1) return fail(E_INVALID, "last layer larger than the domain");
  cudaSetDevice(ctx_->device);
  int32_t rc = ensure_workspace(n, W, B);
  if (rc != OK) return rc;
  // On every exit path: the high-priority stream is drained (an early error return may leave
  // its work in flight), then in transient mode the workspace goes back to the stream-ordered pool.
  struct TransientRelease {
    WideFibProver* p;
    ~TransientRelease() {
      if (p->fast_) cudaStreamSynchronize(p->fast_);
      if (p->transient_ && p->arena_) {
        cudaFreeAsync(p->arena_, p->stream_);
        p->arena_ = nullptr;
        p->arena_size_ = 0;
        p->ws_log_n_ = p->ws_W_ = p->ws_B_ = 0;
      }
    }
  } transient_release{this};
  Layout l = layout_for(n, W, B, cfg.log_last_layer_degree_bound);
  Arena arena{arena_, 0, arena_size_};
  Buffers b;
  try { b = carve(arena, l); } catch (...) { return fail(E_OOM, "workspace too small"); }
  const DeviceTables& T = ctx_->tables;
  cudaStream_t s = stream_;
  uint8_t* pin = pinned_;
  auto sync = [&]() -> cudaError_t { return cudaStreamSynchronize(s); };
  cudaStream_t fs = fast_ ? fast_ : s;
  auto fsync = [&]() -> cudaError_t { return cudaStreamSynchronize(fs); };

  Channel ch;
  SB_CK(cudaEventRecord(ev_[0], s));
  // Trace in HBM.
  const uint32_t* trace = b.trace;
  if (req.trace_device) {
    trace = req.trace_device;
  } else if (req.trace_host) {
    SB_CK(cudaMemcpyAsync(b.trace, req.trace_host, (size_t)W * l.N * 4, cudaMemcpyHostToDevice, s));
  }
  SB_CK(cudaEventRecord(ev_[1], s));
  if (!req.trace_device && !req.trace_host) SB_CK(wide_fib_trace(n, W, req.trace_kind, req.trace_seed, b.trace, l.N, s));
  SB_CK(cudaEventRecord(ev_[2], s));

  // PcsConfig.mixInto (src/core/pcs/mod.zig:32-52).
  {
    QM31 c = qmake(cfg.pow_bits, B, cfg.n_queries, cfg.log_last_layer_degree_bound);
    ch.mix_felts(&c, 1);
  }
  // Tree 0: preprocessed, no columns: root = Blake2s("leaf" block).
  uint8_t root0[32];
  {
    Blake2sHost h;
    uint8_t blk[64] = {0};
    std::memcpy(blk, "leaf", 4);
    h.update(blk, 64);
    h.finalize(root0);
  }
  ch.mix_root(root0);

  // Tree 1: interpolate, extend, commit.
  SB_CK(interpolate_extend(T, n, B, W, trace, l.N, b.coeffs, l.N, b.lde, l.NL, s));
  SB_CK(merkle_commit(l.L, W, b.lde, l.NL, b.tree1, s));
  uint8_t root1[32], root2[32];
  SB_CK(cudaMemcpyAsync(pin, b.tree1 + (2 * l.NL - 2) * 32, 32, cudaMemcpyDeviceToHost, s));
  SB_CK(cudaEventRecord(ev_[3], s));
  SB_CK(sync());
  std::memcpy(root1, pin, 32);
  ch.mix_root(root1);
  {
    uint32_t st[2] = {n, W};
    ch.mix_words(st, 2);
  }
  if (req.has_channel_seed) ch.mix_u64(req.channel_seed);

  // Composition on CanonicCoset(n+1).
  QM31 random_coeff = ch.draw_secure_felt();
  const uint32_t n_cons = W - 2;
  {
    std::vector<QM31> pw(n_cons);
    QM31 cur = qone();
    for (uint32_t i = 0; i < n_cons; ++i) { pw[i] = cur; cur = qmul(cur, random_coeff); }
    QM31* hc = reinterpret_cast<QM31*>(pin);
    for (uint32_t k = 0; k < n_cons; ++k) hc[k] = pw[n_cons - 1 - k];
    SB_CK(cudaMemcpyAsync(b.comp_coeffs, hc, n_cons * sizeof(QM31), cudaMemcpyHostToDevice, s));
  }
  if (B != 1) SB_CK(extend(T, n, 1, W, b.coeffs, l.N, b.eval_c, l.NC, s));
  {
    const PointTable& pt = host_points();
    CircleDomain cd = canonic_domain(l.CL);
    Coset trace_coset = coset_odds(n);
    uint32_t d0 = minv(coset_vanishing_m(pt, trace_coset, pt.at(cd.index_at(0))));
    uint32_t d1 = minv(coset_vanishing_m(pt, trace_coset, pt.at(cd.index_at(1))));
    SB_CK(wide_fib_composition(n, W, b.eval_c, B == 1 ? l.NL : l.NC, b.comp_coeffs, d0, d1, b.comp, l.NC, s));
  }
  SB_CK(cudaEventRecord(ev_[4], s));
  // Interpolate the 4 coordinates, split at mid: left = low half, right = high half.
  SB_CK(fft_columns(T, true, l.CL, 4, b.comp, l.NC, s));
  SB_CK(extend(T, n, B, 4, b.comp, l.NC, b.comp_lde, l.NL, s));
  SB_CK(extend(T, n, B, 4, b.comp + l.N, l.NC, b.comp_lde + 4 * l.NL, l.NL, s));
  SB_CK(merkle_commit(l.L, 8, b.comp_lde, l.NL, b.tree2, s));
  SB_CK(cudaMemcpyAsync(pin, b.tree2 + (2 * l.NL - 2) * 32, 32, cudaMemcpyDeviceToHost, s));
  SB_CK(cudaEventRecord(ev_[5], s));
  SB_CK(sync());
  std::memcpy(root2, pin, 32);
  ch.mix_root(root2);

  // OODS point and sampled values of every coefficient column.
  PointQ oods = random_secure_point(ch);
  SB_CK(eval_at_point(T, n, W, b.coeffs, l.N, oods, nullptr, b.oods_partial, b.oods_out, fs));
  SB_CK(eval_at_point(T, n, 4, b.comp, l.NC, oods, nullptr, b.oods_partial, b.oods_out + W, fs));
  SB_CK(eval_at_point(T, n, 4, b.comp + l.N, l.NC, oods, nullptr, b.oods_partial, b.oods_out + W + 4, fs));
  std::vector<QM31> sampled(W + 8);
  SB_CK(cudaMemcpyAsync(pin, b.oods_out, (W + 8) * sizeof(QM31), cudaMemcpyDeviceToHost, fs));
  SB_CK(cudaEventRecord(ev_[6], fs));
  SB_CK(fsync());
  std::memcpy(sampled.data(), pin, (W + 8) * sizeof(QM31));
  ch.mix_felts(sampled.data(), sampled.size());
  QM31 quot_coeff = ch.draw_secure_felt();

  // Line coefficients of the single sample batch (src/core/constraints.zig:87-97).
  {
    const uint32_t nq = W + 8;
    QM31* hc = reinterpret_cast<QM31*>(pin);
    QM31 rp = qone(), sum_a = qzero(), sum_b = qzero();
    QM31 cy = qsub(qconj(oods.y), oods.y);
    for (uint32_t i = 0; i < nq; ++i) {
      QM31 v = sampled[i];
      QM31 a = qsub(qconj(v), v);
      QM31 bb = qsub(qmul(v, cy), qmul(a, oods.y));
      hc[i] = qmul(rp, cy);
      sum_a = qadd(sum_a, qmul(rp, a));
      sum_b = qadd(sum_b, qmul(rp, bb));
      rp = qmul(rp, quot_coeff);
    }
    const uint32_t** hp = reinterpret_cast<const uint32_t**>(pin + 64 * 1024);
    for (uint32_t i = 0; i < W; ++i) hp[i] = b.lde + (size_t)i * l.NL;
    for (uint32_t i = 0; i < 8; ++i) hp[W + i] = b.comp_lde + (size_t)i * l.NL;
    QuotientBatchDev* hb = reinterpret_cast<QuotientBatchDev*>(pin + 128 * 1024);
    hb->point = oods; hb->sum_a = sum_a; hb->sum_b = sum_b; hb->first = 0; hb->count = nq;
    SB_CK(cudaMemcpyAsync(b.quot_c, hc, nq * sizeof(QM31), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.col_ptrs, hp, nq * sizeof(void*), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.batch, hb, sizeof(QuotientBatchDev), cudaMemcpyHostToDevice, fs));
  }
  SB_CK(accumulate_quotients(T, l.L, 1, b.batch, b.col_ptrs, b.quot_c, b.quot, l.NL, fs));
  SB_CK(cudaEventRecord(ev_[7], fs));

  // FRI: first layer, then inner layers each committed before its fold.
  std::vector<std::array<uint8_t, 32>> fri_roots;
  {
    SB_CK(merkle_commit(l.L, 4, b.quot, l.NL, b.tree_q, fs));
    SB_CK(cudaMemcpyAsync(pin, b.tree_q + (2 * l.NL - 2) * 32, 32, cudaMemcpyDeviceToHost, fs));
    SB_CK(fsync());
    std::array<uint8_t, 32> r;
    std::memcpy(r.data(), pin, 32);
    fri_roots.push_back(r);
    ch.mix_root(r.data());
    QM31 alpha = ch.draw_secure_felt();
    // Each fold writes the next line layer and, unless it is the last layer,
    // commits it in the same launch sequence.
    SB_CK(fri_fold_commit(T, true, l.L, b.quot, l.NL, alpha, b.line[0], 1ull << (l.L - 1),
                          l.n_inner > 0 ? b.line_tree[0] : nullptr, fs));
    for (uint32_t k = 0; k < l.n_inner; ++k) {
      uint32_t lg = l.L - 1 - k;
      size_t sz = 1ull << lg;
      SB_CK(cudaMemcpyAsync(pin, b.line_tree[k] + (2 * sz - 2) * 32, 32, cudaMemcpyDeviceToHost, fs));
      SB_CK(fsync());
      std::memcpy(r.data(), pin, 32);
      fri_roots.push_back(r);
      ch.mix_root(r.data());
      QM31 a = ch.draw_secure_felt();
      SB_CK(fri_fold_commit(T, false, lg, b.line[k], sz, a, b.line[k + 1], sz / 2,
                            k + 1 < l.n_inner ? b.line_tree[k + 1] : nullptr, fs));
    }
  }
  // Last layer: line IFFT of 2^last_log values (src/backend/line_evaluation.zig:97-145).
  std::vector<QM31> last_coeffs;
  {
    size_t m = 1ull << l.last_log;
    SB_CK(cudaMemcpyAsync(pin, b.line[l.n_inner], 4 * m * 4, cudaMemcpyDeviceToHost, fs));
    SB_CK(fsync());
    const uint32_t* w = reinterpret_cast<const uint32_t*>(pin);
    std::vector<QM31> v(m);
    for (size_t i = 0; i < m; ++i) v[i] = qmake(w[i], w[m + i], w[2 * m + i], w[3 * m + i]);
    auto brev = [&](std::vector<QM31>& x) {
      uint32_t lg = l.last_log;
      for (size_t i = 0; i < x.size(); ++i) { size_t j = bitrev((uint32_t)i, lg); if (j > i) std::swap(x[i], x[j]); }
    };
    brev(v);
    const PointTable& pt = host_points();
    Coset d = coset_half_odds(l.last_log);
    while (d.log_size > 0) {
      size_t chunk = 1ull << d.log_size, half = chunk / 2;
      for (size_t st = 0; st < m; st += chunk)
        for (size_t i = 0; i < half; ++i) {
          uint32_t ix = minv(pt.at(d.index_at(i)).x);
          QM31 a = v[st + i], c = v[st + half + i];
          v[st + i] = qadd(a, c);
          v[st + half + i] = qmulm(qsub(a, c), ix);
        }
      d = d.dbl();
    }
    uint32_t li = minv((uint32_t)(m % P));
    for (QM31& x : v) x = qmulm(x, li);
    brev(v);
    size_t bound = 1ull << cfg.log_last_layer_degree_bound;
    for (size_t i = bound; i < m; ++i)
      if (!qiszero(v[i])) return fail(E_CONSTRAINTS, "last FRI layer exceeds its degree bound");
    last_coeffs.assign(v.begin(), v.begin() + bound);
    if (last_coeffs.size() > 1) {
      uint32_t lg = 0; while ((1ull << lg) < last_coeffs.size()) ++lg;
      for (size_t i = 0; i < last_coeffs.size(); ++i) { size_t j = bitrev((uint32_t)i, lg); if (j > i) std::swap(last_coeffs[i], last_coeffs[j]); }
    }
    ch.mix_felts(last_coeffs.data(), last_coeffs.size());
  }
  SB_CK(cudaEventRecord(ev_[8], fs));

  // Proof of work on the device.
  uint64_t nonce = 0;
  if (cfg.pow_bits > 0) {
    uint8_t prefix[32];
    {
      Blake2sHost h;
      uint32_t tag = 0x12345678u;
      uint8_t z[12] = {0};
      h.update(&tag, 4); h.update(z, 12); h.update(ch.digest, 32); h.update(&cfg.pow_bits, 4);
      h.finalize(prefix);
    }
    uint32_t pw[8];
    std::memcpy(pw, prefix, 32);
    // Rounds of ~17M nonces, four per check; the search bound is 2^(bits+16) nonces.
    const uint64_t max_nonce = cfg.pow_bits >= 48 ? ~0ull : (1ull << (cfg.pow_bits + 16));
    const uint64_t per_round = pow_round_nonces(ctx_->sm_count);
    SB_CK(cudaMemsetAsync(b.pow_result, 0xff, 8, s));
    nonce = ~0ull;
    for (uint64_t base = 0; base < max_nonce && nonce == ~0ull;) {
      for (int r = 0; r < 4 && base < max_nonce; ++r, base += per_round)
        SB_CK(pow_round(pw, cfg.pow_bits, base, b.pow_result, ctx_->sm_count, s));
      SB_CK(cudaMemcpyAsync(pin, b.pow_result, 8, cudaMemcpyDeviceToHost, s));
      SB_CK(sync());
      std::memcpy(&nonce, pin, 8);
    }
    if (nonce == ~0ull) return fail(E_TIMEOUT, "proof-of-work search bound reached");
  }
  ch.mix_u64(nonce);
  SB_CK(cudaEventRecord(ev_[9], s));

  // Queries (src/core/queries.zig:8-60).
  std::vector<uint64_t> queries;
  {
    uint32_t mask = (uint32_t)((1ull << l.L) - 1);
    while (queries.size() < cfg.n_queries) {
      uint32_t w[8];
      ch.draw_u32s(w);
      for (uint32_t x : w) { queries.push_back(x & mask); if (queries.size() == cfg.n_queries) break; }
    }
    std::sort(queries.begin(), queries.end());
    queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  }

  // Decommitment plan: gather words and hashes in one pass.
  std::vector<GatherItem> words;
  std::vector<HashGatherItem> hashes;
  struct LayerPlan { size_t wit_word0, n_wit, hash0, n_hash; };
  // trace trees
  size_t q1_words = words.size();
  for (uint32_t c = 0; c < W; ++c)
    for (uint64_t q : queries) words.push_back({b.lde + (size_t)c * l.NL, q});
  size_t q2_words = words.size();
  for (uint32_t c = 0; c < 8; ++c)
    for (uint64_t q : queries) words.push_back({b.comp_lde + (size_t)c * l.NL, q});
  std::vector<uint64_t> wn1 = witness_nodes(l.L, queries);
  size_t h1 = hashes.size();
  for (uint64_t nd : wn1) hashes.push_back({b.tree1, nd});
  size_t h2 = hashes.size();
  for (uint64_t nd : wn1) hashes.push_back({b.tree2, nd});
  // FRI layers
  std::vector<LayerPlan> fplan;
  std::vector<std::vector<uint64_t>> fpos;  // decommitment positions per layer
  {
    std::vector<uint64_t> lq = queries;
    for (uint32_t k = 0; k <= l.n_inner; ++k) {
      // k = 0: first layer (quotient column, log L); k >= 1: inner layer k-1.
      const uint32_t* colbase = k == 0 ? b.quot : b.line[k - 1];
      uint64_t csz = k == 0 ? l.NL : (1ull << (l.L - k));
      uint32_t lg = k == 0 ? l.L : l.L - k;
      const uint8_t* tree = k == 0 ? b.tree_q : b.line_tree[k - 1];
      LayerPlan lp{words.size(), 0, hashes.size(), 0};
      std::vector<uint64_t> positions;
      size_t q = 0;
      while (q < lq.size()) {
        uint64_t key = lq[q] >> 1;
        size_t end = q + 1;
        while (end < lq.size() && (lq[end] >> 1) == key) ++end;
        size_t at = q;
        for (uint64_t pos = key << 1; pos < (key << 1) + 2; ++pos) {
          positions.push_back(pos);
          if (at < end && lq[at] == pos) { ++at; continue; }
          for (int c = 0; c < 4; ++c) words.push_back({colbase + c * csz, pos});
          lp.n_wit += 1;
        }
        q = end;
      }
      std::vector<uint64_t> wn = witness_nodes(lg, positions);
      for (uint64_t nd : wn) hashes.push_back({tree, nd});
      lp.n_hash = wn.size();
      fplan.push_back(lp);
      // fold queries
      std::vector<uint64_t> nq;
      for (uint64_t p : lq) { uint64_t f = p >> 1; if (nq.empty() || nq.back() != f) nq.push_back(f); }
      lq.swap(nq);
    }
  }
  size_t words_bytes = words.size() * sizeof(GatherItem), hash_items_bytes = hashes.size() * sizeof(HashGatherItem);
  size_t out_words_bytes = words.size() * 4, out_hash_bytes = hashes.size() * 32;
  size_t total = 4 * 256 + words_bytes + hash_items_bytes + out_words_bytes + out_hash_bytes;
  if (total > b.scratch_bytes || total > pinned_size_) return fail(E_INVALID, "decommitment exceeds staging capacity");
  size_t o_items = 0, o_hitems = (words_bytes + 255) & ~255ull, o_outw = (o_hitems + hash_items_bytes + 255) & ~255ull,
         o_outh = (o_outw + out_words_bytes + 255) & ~255ull;
  std::memcpy(pin + o_items, words.data(), words_bytes);
  std::memcpy(pin + o_hitems, hashes.data(), hash_items_bytes);
  SB_CK(cudaMemcpyAsync(b.scratch, pin, o_outw, cudaMemcpyHostToDevice, fs));
  SB_CK(gather_words(reinterpret_cast<GatherItem*>(b.scratch + o_items), (uint32_t)words.size(),
                     reinterpret_cast<uint32_t*>(b.scratch + o_outw), fs));
  SB_CK(gather_hashes(reinterpret_cast<HashGatherItem*>(b.scratch + o_hitems), (uint32_t)hashes.size(),
                      b.scratch + o_outh, fs));
  SB_CK(cudaMemcpyAsync(pin + o_outw, b.scratch + o_outw, o_outh - o_outw + out_hash_bytes, cudaMemcpyDeviceToHost, fs));
  SB_CK(cudaEventRecord(ev_[10], fs));
  SB_CK(fsync());
  const uint32_t* gw = reinterpret_cast<const uint32_t*>(pin + o_outw);
  const uint8_t* gh = pin + o_outh;

  // Wire encoding (src/interop/proof_wire.zig:19-77).
  Json j;
  j.s.reserve(1 << 16);
  j.s += "{\"config\":{\"pow_bits\":"; j.u(cfg.pow_bits);
  j.s += ",\"fri_config\":{\"log_blowup_factor\":"; j.u(B);
  j.s += ",\"log_last_layer_degree_bound\":"; j.u(cfg.log_last_layer_degree_bound);
  j.s += ",\"n_queries\":"; j.u(cfg.n_queries);
  j.s += ",\"fold_step\":1},\"lifting_log_size\":null},\"commitments\":[";
  j.hash(root0); j.s += ','; j.hash(root1); j.s += ','; j.hash(root2);
  j.s += "],\"sampled_values\":[[],[";
  for (uint32_t c = 0; c < W; ++c) { if (c) j.s += ','; j.s += '['; j.qm(sampled[c]); j.s += ']'; }
  j.s += "],[";
  for (uint32_t c = 0; c < 8; ++c) { if (c) j.s += ','; j.s += '['; j.qm(sampled[W + c]); j.s += ']'; }
  auto hash_list = [&](size_t first, size_t count) {
    j.s += '[';
    for (size_t i = 0; i < count; ++i) { if (i) j.s += ','; j.hash(gh + (first + i) * 32); }
    j.s += ']';
  };
  j.s += "]],\"decommitments\":[{\"hash_witness\":[]},{\"hash_witness\":";
  hash_list(h1, wn1.size());
  j.s += "},{\"hash_witness\":";
  hash_list(h2, wn1.size());
  j.s += "}],\"queried_values\":[[],[";
  const size_t nqv = queries.size();
  auto qv = [&](size_t first, uint32_t cols) {
    for (uint32_t c = 0; c < cols; ++c) {
      if (c) j.s += ',';
      j.s += '[';
      for (size_t q = 0; q < nqv; ++q) { if (q) j.s += ','; j.u(gw[first + c * nqv + q]); }
      j.s += ']';
    }
  };
  qv(q1_words, W);
  j.s += "],[";
  qv(q2_words, 8);
  j.s += "]],\"proof_of_work\":"; j.u(nonce);
  auto layer = [&](size_t k) {
    const LayerPlan& lp = fplan[k];
    j.s += "{\"fri_witness\":[";
    for (size_t i = 0; i < lp.n_wit; ++i) {
      if (i) j.s += ',';
      const uint32_t* w = gw + lp.wit_word0 + 4 * i;
      j.qm(qmake(w[0], w[1], w[2], w[3]));
    }
    j.s += "],\"decommitment\":{\"hash_witness\":";
    hash_list(lp.hash0, lp.n_hash);
    j.s += "},\"commitment\":"; j.hash(fri_roots[k].data()); j.s += '}';
  };
  j.s += ",\"fri_proof\":{\"first_layer\":"; layer(0);
  j.s += ",\"inner_layers\":[";
  for (uint32_t k = 1; k <= l.n_inner; ++k) { if (k > 1) j.s += ','; layer(k); }
  j.s += "],\"last_layer_poly\":[";
  for (size_t i = 0; i < last_coeffs.size(); ++i) { if (i) j.s += ','; j.qm(last_coeffs[i]); }
  j.s += "]}}";

  // Prover self-check of the composition OODS value (src/prover/prove.zig:366-386).
  {
    const QM31 basis[4] = {qone(), qmake(0, 1, 0, 0), qmake(0, 0, 1, 0), qmake(0, 0, 0, 1)};
    QM31 left = qzero(), right = qzero();
    for (int k = 0; k < 4; ++k) {
      left = qadd(left, qmul(sampled[W + k], basis[k]));
      right = qadd(right, qmul(sampled[W + 4 + k], basis[k]));
    }
    PointQ p = oods;
    for (uint32_t i = 0; i + 2 < l.CL; ++i) p = qpadd(p, p);
    QM31 comp_oods = qadd(left, qmul(p.x, right));
    // vanishing of CanonicCoset(n) at the OODS point
    Coset tc = coset_odds(n);
    const PointTable& pt = host_points();
    PointM ini = pt.at(tc.initial), hs = pt.at(tc.step / 2);
    PointQ q = qpadd(qpadd(oods, PointQ{qbase(ini.x), qneg(qbase(ini.y))}), PointQ{qbase(hs.x), qbase(hs.y)});
    QM31 x = q.x;
    for (uint32_t i = 1; i < tc.log_size; ++i) x = qdouble_x(x);
    QM31 dinv = qinv(x);
    QM31 acc = qzero(), a = sampled[0], bb = sampled[1];
    for (uint32_t k = 2; k < W; ++k) {
      QM31 c = sampled[k];
      acc = qadd(qmul(acc, random_coeff), qmul(qsub(c, qadd(qsq(a), qsq(bb))), dinv));
      a = bb; bb = c;
    }
    if (!qeq(acc, comp_oods)) return fail(E_CONSTRAINTS, "constraints not satisfied at the OODS point");
  }

  if (times) {
    auto el = [&](int a, int c) { float ms = 0; cudaEventElapsedTime(&ms, ev_[a], ev_[c]); return ms; };
    times->upload = el(0, 1);
    times->trace = el(1, 2);
    times->main_commit = el(2, 3);
    times->composition = el(3, 4);
    times->composition_commit = el(4, 5);
    times->oods = el(5, 6);
    times->quotients = el(6, 7);
    times->fri = el(7, 8);
    times->pow = el(8, 9);
    times->decommit = el(9, 10);
    times->total = el(0, 10);
  }
  out.swap(j.s);
  return OK;
}

const char* status_string(int32_t code) {
  switch (code) {
    case OK: return "ok";
    case E_INVALID: return "invalid argument";
    case E_OOM: return "out of device memory";
    case E_CUDA: return "CUDA error";
    case E_TIMEOUT: return "device search bound reached";
    case E_CONSTRAINTS: return "constraints not satisfied";
    case E_BUFFER_TOO_SMALL: return "output buffer too small";
    case E_FALLBACK: return "operation not taken by the device";
    case E_NO_DEVICE: return "no CUDA device";
    case E_DIVISION_BY_ZERO: return "division by zero";
    case E_REJECTED: return "admission rejected";
    default: return "unknown status";
  }
}

}  // namespace sb
