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
#include <chrono>
#include <cstring>
#include <stdexcept>

#include "alloc.hpp"
#include "blake2s.cuh"
#include "prover.hpp"
#include "prover_common.hpp"

namespace sb {

namespace {

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
  FriChannelDev* chan;
  uint8_t* scratch;  // gathers
  size_t scratch_bytes;
};

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
  b.chan = a.take<FriChannelDev>(1);
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
  for (LogupXorProver* p : xor_pool) delete p;
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
  tables.sm_count = (uint32_t)std::max(sm_count, 1);
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
  if (cudaMalloc(&tables.tw, tw_words * 8) != cudaSuccess) return E_OOM;
  if (cudaMalloc(&tables.itw, tw_words * 8) != cudaSuccess) return E_OOM;
  tables.tw2 = tables.tw + tw_words;
  tables.itw2 = tables.itw + tw_words;
  if (build_twiddle_tower(tables, tower_log, stream) != cudaSuccess) return E_CUDA;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return E_CUDA;
  return OK;
}

StreamPriorities stream_priorities() {
  StreamPriorities r;
  if (cudaDeviceGetStreamPriorityRange(&r.least, &r.greatest) != cudaSuccess) {
    cudaGetLastError();
    r.least = r.greatest = 0;
  }
  r.bulk = r.greatest < r.least ? r.least - 1 : r.least;
  return r;
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
  if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, stream_priorities().bulk) != cudaSuccess) return nullptr;
  return new WideFibProver(this, s);
}

void Context::release(WideFibProver* p) {
  std::lock_guard<std::mutex> g(mu);
  pool.push_back(p);
}

LogupXorProver* Context::acquire_xor() {
  {
    std::lock_guard<std::mutex> g(mu);
    if (!xor_pool.empty()) {
      LogupXorProver* p = xor_pool.back();
      xor_pool.pop_back();
      return p;
    }
  }
  cudaSetDevice(device);
  return new LogupXorProver(this);
}

void Context::release_xor(LogupXorProver* p) {
  std::lock_guard<std::mutex> g(mu);
  xor_pool.push_back(p);
}

// ---------------------------------------------------------------------------
// Prover
// ---------------------------------------------------------------------------
WideFibProver::WideFibProver(Context* ctx, cudaStream_t stream) : ctx_(ctx), stream_(stream) {
  for (auto& e : ev_) cudaEventCreate(&e);
  const StreamPriorities pr = stream_priorities();
  if (cudaStreamCreateWithPriority(&fast_, cudaStreamNonBlocking, pr.greatest) != cudaSuccess) {
    cudaGetLastError();
    fast_ = nullptr;
  }
  if (cudaStreamCreateWithPriority(&pow_, cudaStreamNonBlocking, pr.least) != cudaSuccess) {
    cudaGetLastError();
    pow_ = nullptr;
  }
}

WideFibProver::~WideFibProver() {
  release();
  for (auto& e : ev_) cudaEventDestroy(e);
  if (fast_) cudaStreamDestroy(fast_);
  if (pow_) cudaStreamDestroy(pow_);
  if (stream_) cudaStreamDestroy(stream_);
}

void WideFibProver::drop_workspace() {
  if (transient_ || !arena_) return;
  cudaSetDevice(ctx_->device);
  cudaFree(arena_);
  arena_ = nullptr;
  arena_size_ = 0;
  ws_log_n_ = ws_W_ = ws_B_ = 0;
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

int32_t WideFibProver::reserve(uint32_t log_n, uint32_t W, uint32_t B, size_t* held) {
  if (!transient_) {
    cudaSetDevice(ctx_->device);
    int32_t rc = ensure_workspace(log_n, W, B);
    if (rc != OK) return rc;
  }
  if (held) *held = transient_ ? 0 : arena_size_;
  return OK;
}

int32_t WideFibProver::ensure_workspace(uint32_t log_n, uint32_t W, uint32_t B) {
  if (!pinned_) {
    pinned_size_ = GATHER_SCRATCH + (1 << 20);
    if (host_malloc_pinned(reinterpret_cast<void**>(&pinned_), pinned_size_) != cudaSuccess) { pinned_ = nullptr; return fail(E_OOM, "pinned staging allocation failed"); }
  }
  size_t need = workspace_bytes(log_n, W, B);
  if (transient_) {
    if (dev_malloc_async(reinterpret_cast<void**>(&arena_), need, stream_) != cudaSuccess) {
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
  if (dev_malloc(reinterpret_cast<void**>(&arena_), need) != cudaSuccess) { arena_ = nullptr; cudaGetLastError(); return fail(E_OOM, "device workspace allocation failed"); }
  arena_size_ = need;
  ws_log_n_ = log_n; ws_W_ = W; ws_B_ = B;
  return OK;
}

int32_t WideFibProver::prove(const ProveRequest& req, std::string& out, StageTimes* times) {
  const uint32_t n = req.log_n_rows, W = req.sequence_len;
  const PcsConfig& cfg = req.config;
  const uint32_t B = cfg.log_blowup_factor;
  if (n < 1 || n > 22 || W < 2 || W > 1000 || B < 1 || B > 4 || n + B > ctx_->tables.tower_log + 1 ||
      n + 1 > ctx_->tables.tower_log + 1 || cfg.n_queries == 0 || cfg.n_queries > 4096 || cfg.pow_bits > MAX_POW_BITS)
    return fail(E_INVALID, "unsupported proof shape or configuration");
  if (n + B < cfg.log_last_layer_degree_bound + B + 1) return fail(E_INVALID, "last layer larger than the domain");
  if (req.trace_kind < 0 || req.trace_kind > TRACE_FIRST_COLUMNS)
    return fail(E_INVALID, "unknown trace kind");
  if (req.trace_kind == TRACE_FIRST_COLUMNS && !req.trace_host && !req.trace_device)
    return fail(E_INVALID, "the first two trace columns are missing");
  cudaSetDevice(ctx_->device);
  int32_t rc = ensure_workspace(n, W, B);
  if (rc != OK) return rc;
  // On every exit path: the high-priority and grind streams are drained (an early error return may
  // leave their work in flight), then in transient mode the workspace goes back to the
  // stream-ordered pool.
  struct TransientRelease {
    WideFibProver* p;
    ~TransientRelease() {
      if (p->fast_) stream_wait(p->fast_);
      if (p->pow_) stream_wait(p->pow_);
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
  auto sync = [&]() -> cudaError_t { return stream_wait(s); };
  cudaStream_t fs = fast_ ? fast_ : s;
  auto fsync = [&]() -> cudaError_t { return stream_wait(fs); };

  Channel ch;
  SB_CK(cudaEventRecord(ev_[0], s));
  // Trace in HBM.
  // A full trace is used where it lies (device) or uploaded (host); with TRACE_FIRST_COLUMNS only
  // col0/col1 are given and the device derives the other columns.
  const uint32_t* trace = b.trace;
  const bool first_two = req.trace_kind == TRACE_FIRST_COLUMNS;
  if (req.trace_device) {
    if (first_two) SB_CK(cudaMemcpyAsync(b.trace, req.trace_device, 2 * l.N * 4, cudaMemcpyDeviceToDevice, s));
    else trace = req.trace_device;
  } else if (req.trace_host) {
    // Host uploads go one at a time (FIFO on the context's lock, each held until its copy has
    // landed): concurrent copies of several proofs would share the host link and all finish
    // late, while one after the other each proof starts computing as soon as its own trace is in.
    std::lock_guard<std::mutex> g(ctx_->h2d_mu);
    const size_t cols = first_two ? 2 : W;
    SB_CK(cudaMemcpyAsync(b.trace, req.trace_host, cols * l.N * 4, cudaMemcpyHostToDevice, s));
    SB_CK(cudaEventRecord(ev_[1], s));
    SB_CK(event_wait(ev_[1]));
  }
  if (!req.trace_host) SB_CK(cudaEventRecord(ev_[1], s));
  if (first_two || (!req.trace_device && !req.trace_host))
    SB_CK(wide_fib_trace(n, W, req.trace_kind, req.trace_seed, b.trace, l.N, s));
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
  Clock::time_point gap = Clock::now();
  float host_gaps = 0;
  auto gap_end = [&]() { host_gaps += std::chrono::duration<float, std::milli>(Clock::now() - gap).count(); };
  std::memcpy(root1, pin, 32);
  if (deadline_.passed()) return fail(E_TIMEOUT, "proof deadline passed after the main commitment");
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
    gap_end();
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
  gap = Clock::now();
  std::memcpy(root2, pin, 32);
  if (deadline_.passed()) return fail(E_TIMEOUT, "proof deadline passed after the composition commitment");
  ch.mix_root(root2);

  // OODS point and sampled values of every coefficient column.
  PointQ oods = random_secure_point(ch);
  gap_end();
  SB_CK(eval_at_point(T, n, W, b.coeffs, l.N, oods, nullptr, b.oods_partial, b.oods_out, fs));
  SB_CK(eval_at_point(T, n, 4, b.comp, l.NC, oods, nullptr, b.oods_partial, b.oods_out + W, fs));
  SB_CK(eval_at_point(T, n, 4, b.comp + l.N, l.NC, oods, nullptr, b.oods_partial, b.oods_out + W + 4, fs));
  std::vector<QM31> sampled(W + 8);
  SB_CK(cudaMemcpyAsync(pin, b.oods_out, (W + 8) * sizeof(QM31), cudaMemcpyDeviceToHost, fs));
  SB_CK(cudaEventRecord(ev_[6], fs));
  SB_CK(fsync());
  gap = Clock::now();
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
    gap_end();
    SB_CK(cudaMemcpyAsync(b.quot_c, hc, nq * sizeof(QM31), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.col_ptrs, hp, nq * sizeof(void*), cudaMemcpyHostToDevice, fs));
    SB_CK(cudaMemcpyAsync(b.batch, hb, sizeof(QuotientBatchDev), cudaMemcpyHostToDevice, fs));
  }
  // The workspace columns start 16-byte aligned: the bulk-staged quotient kernel may run, its status
  // read back with the FRI channel.
  SB_CK(cudaMemsetAsync(&b.chan->quot_status, 0, sizeof(uint32_t), fs));
  SB_CK(accumulate_quotients(T, l.L, 1, W + 8, b.batch, b.col_ptrs, b.quot_c, b.quot, l.NL, fs, &b.chan->quot_status));
  SB_CK(cudaEventRecord(ev_[7], fs));

  // FRI, last layer, proof of work and queries.
  FriBuffers fbuf{b.quot, b.tree_q, b.line, b.line_tree, b.pow_result, b.chan};
  FriResult fr;
  {
    std::string ferr;
    int32_t frc = fri_pow_queries(T, ctx_->sm_count, ch, cfg, l.L, l.n_inner, l.last_log, fbuf, pin, pow_ ? pow_ : s, fs, ev_[8],
                                  ev_[9], deadline_, fr, ferr);
    if (frc != OK) return fail(frc, ferr);
  }
  const std::vector<uint64_t>& queries = fr.queries;

  // Decommitment: queried values and witnesses of the trace trees and the FRI layers.
  DecommitPlan plan;
  {
    std::vector<const uint32_t*> c1, c2;
    for (uint32_t c = 0; c < W; ++c) c1.push_back(b.lde + (size_t)c * l.NL);
    for (uint32_t c = 0; c < 8; ++c) c2.push_back(b.comp_lde + (size_t)c * l.NL);
    plan.add_tree(nullptr, 0, {}, queries);  // preprocessed: empty
    plan.add_tree(b.tree1, l.L, c1, queries);
    plan.add_tree(b.tree2, l.L, c2, queries);
    plan.add_fri(fbuf, l.L, l.n_inner, queries);
    host_gaps += fr.host_gap_ms + std::chrono::duration<float, std::milli>(Clock::now() - fr.gap_start).count();
    std::string gerr;
    int32_t grc = plan.gather(b.scratch, b.scratch_bytes, pin, pinned_size_, fs, ev_[10], gerr);
    if (grc != OK) return fail(grc, gerr);
  }

  const auto t_encode = std::chrono::steady_clock::now();
  // Wire encoding (src/interop/proof_wire.zig:19-77).
  Json j;
  j.reserve(3 << 20);
  j.lit("{\"config\":{\"pow_bits\":"); j.u(cfg.pow_bits);
  j.lit(",\"fri_config\":{\"log_blowup_factor\":"); j.u(B);
  j.lit(",\"log_last_layer_degree_bound\":"); j.u(cfg.log_last_layer_degree_bound);
  j.lit(",\"n_queries\":"); j.u(cfg.n_queries);
  j.lit(",\"fold_step\":1},\"lifting_log_size\":null},\"commitments\":[");
  j.hash(root0); j.ch(','); j.hash(root1); j.ch(','); j.hash(root2);
  j.lit("],\"sampled_values\":[[],[");
  for (uint32_t c = 0; c < W; ++c) { if (c) j.ch(','); j.ch('['); j.qm(sampled[c]); j.ch(']'); }
  j.lit("],[");
  for (uint32_t c = 0; c < 8; ++c) { if (c) j.ch(','); j.ch('['); j.qm(sampled[W + c]); j.ch(']'); }
  j.lit("]],\"decommitments\":[");
  for (size_t t = 0; t < 3; ++t) { if (t) j.ch(','); j.lit("{\"hash_witness\":"); plan.json_witness(j, t); j.ch('}'); }
  j.lit("],\"queried_values\":[");
  for (size_t t = 0; t < 3; ++t) { if (t) j.ch(','); plan.json_queried(j, t); }
  j.lit("],\"proof_of_work\":"); j.u(fr.nonce);
  j.lit(",\"fri_proof\":");
  plan.json_fri(j, fr);
  j.ch('}');

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
    times->host_encode =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_encode).count();
    times->host_gaps = host_gaps;
  }
  out = j.str();
  return OK;
}

const char* status_string(int32_t code) {
  switch (code) {
    case OK: return "ok";
    case E_INVALID: return "invalid argument";
    case E_OOM: return "out of device memory";
    case E_CUDA: return "CUDA error";
    case E_TIMEOUT: return "deadline or search bound reached";
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
