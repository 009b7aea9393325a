// Proof tail shared by the provers (declarations in prover_common.hpp).
#include "prover_common.hpp"

#include <algorithm>

namespace sb {

#define SB_CKE(expr)                                                           \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      err = std::string(#expr) + ": " + cudaGetErrorString(_e);                \
      return E_CUDA;                                                           \
    }                                                                          \
  } while (0)

int32_t fri_pow_queries(const DeviceTables& T, int sm_count, Channel& ch, const PcsConfig& cfg, uint32_t L,
                        uint32_t n_inner, uint32_t last_log, const FriBuffers& fb, uint8_t* pin, cudaStream_t s,
                        cudaStream_t fs, cudaEvent_t ev_fri, cudaEvent_t ev_pow, const Deadline& deadline,
                        FriResult& out, std::string& err) {
  const uint64_t NL = 1ull << L;
  // FRI: first layer, then inner layers each committed before its fold. The channel steps
  // between them (mix the layer's root, draw its alpha) run on the device, so the layers
  // follow one another on `fs` without a host round trip.
  std::vector<std::array<uint8_t, 32>>& fri_roots = out.roots;
  if (n_inner + 1 > FRI_MAX_LAYERS) { err = "too many FRI layers"; return E_INVALID; }
  const size_t m_last = 1ull << last_log;
  constexpr size_t LAST_OFF = (sizeof(FriChannelDev) + 255) & ~size_t(255);
  {
    uint32_t* up = reinterpret_cast<uint32_t*>(pin);
    std::memcpy(up, ch.digest, 32);
    up[8] = ch.n_draws;
    up[9] = 0;  // status
    SB_CKE(cudaMemcpyAsync(fb.chan, up, 40, cudaMemcpyHostToDevice, fs));
    SB_CKE(merkle_commit(L, 4, fb.quot, NL, fb.tree_q, fs));
    SB_CKE(fri_channel_step(fb.chan, fb.tree_q + (2 * NL - 2) * 32, 0, fs));
    // Each fold writes the next line layer and, unless it is the last layer,
    // commits it in the same launch sequence.
    SB_CKE(fri_fold_commit(T, true, L, fb.quot, NL, &fb.chan->alpha[0], fb.line[0], 1ull << (L - 1),
                          n_inner > 0 ? fb.line_tree[0] : nullptr, fs));
    // Large layers one launch sequence each; the small ones (at most 2^12 values) in one CTA.
    const uint32_t k_tail = fri_tail_first(L, n_inner);
    for (uint32_t k = 0; k < k_tail; ++k) {
      uint32_t lg = L - 1 - k;
      size_t sz = 1ull << lg;
      SB_CKE(fri_channel_step(fb.chan, fb.line_tree[k] + (2 * sz - 2) * 32, k + 1, fs));
      SB_CKE(fri_fold_commit(T, false, lg, fb.line[k], sz, &fb.chan->alpha[k + 1], fb.line[k + 1], sz / 2,
                            k + 1 < n_inner ? fb.line_tree[k + 1] : nullptr, fs));
    }
    SB_CKE(fri_tail(T, fb.chan, L, k_tail, n_inner, fb.line.data(), fb.line_tree.data(), fs));
    // One copy back: the device channel (roots, alphas) and the last layer's values.
    SB_CKE(cudaMemcpyAsync(pin, fb.chan, sizeof(FriChannelDev), cudaMemcpyDeviceToHost, fs));
    SB_CKE(cudaMemcpyAsync(pin + LAST_OFF, fb.line[n_inner], 4 * m_last * 4, cudaMemcpyDeviceToHost, fs));
    SB_CKE(stream_wait(fs));
    out.gap_start = Clock::now();
    FriChannelDev dc;
    std::memcpy(&dc, pin, sizeof(dc));
    if (dc.quot_status != 0) {
      err = (dc.quot_status & QUOT_STATUS_TIMEOUT) ? "a staged column load of the quotient kernel ran out of time"
                                                    : "the quotient batches do not fit the staged kernel's item table";
      return E_CUDA;
    }
    for (uint32_t k = 0; k <= n_inner; ++k) {
      std::array<uint8_t, 32> r;
      std::memcpy(r.data(), dc.roots[k], 32);
      fri_roots.push_back(r);
      ch.mix_root(r.data());
      QM31 a = ch.draw_secure_felt();
      if (dc.status != 0 || !qeq(a, dc.alpha[k])) {
        err = "device FRI channel diverged from the host transcript";
        return E_CUDA;
      }
    }
  }
  // Last layer: line IFFT of 2^last_log values (src/backend/line_evaluation.zig:97-145).
  std::vector<QM31>& last_coeffs = out.last_coeffs;
  {
    const size_t m = m_last;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(pin + LAST_OFF);
    std::vector<QM31> v(m);
    for (size_t i = 0; i < m; ++i) v[i] = qmake(w[i], w[m + i], w[2 * m + i], w[3 * m + i]);
    auto brev = [&](std::vector<QM31>& x) {
      uint32_t lg = last_log;
      for (size_t i = 0; i < x.size(); ++i) { size_t j = bitrev((uint32_t)i, lg); if (j > i) std::swap(x[i], x[j]); }
    };
    brev(v);
    const PointTable& pt = host_points();
    Coset d = coset_half_odds(last_log);
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
      if (!qiszero(v[i])) { err = "last FRI layer exceeds its degree bound"; return E_CONSTRAINTS; }
    last_coeffs.assign(v.begin(), v.begin() + bound);
    if (last_coeffs.size() > 1) {
      uint32_t lg = 0; while ((1ull << lg) < last_coeffs.size()) ++lg;
      for (size_t i = 0; i < last_coeffs.size(); ++i) { size_t j = bitrev((uint32_t)i, lg); if (j > i) std::swap(last_coeffs[i], last_coeffs[j]); }
    }
    ch.mix_felts(last_coeffs.data(), last_coeffs.size());
  }
  if (ev_fri) SB_CKE(cudaEventRecord(ev_fri, fs));

  // Proof of work on the device.
  uint64_t& nonce = out.nonce;
  nonce = 0;
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
    const uint64_t per_round = pow_round_nonces(sm_count);
    SB_CKE(cudaMemsetAsync(fb.pow_result, 0xff, 8, s));
    nonce = ~0ull;
    for (uint64_t base = 0; base < max_nonce && nonce == ~0ull;) {
      out.host_gap_ms += std::chrono::duration<float, std::milli>(Clock::now() - out.gap_start).count();
      for (int r = 0; r < 4 && base < max_nonce; ++r, base += per_round)
        SB_CKE(pow_round(pw, cfg.pow_bits, base, fb.pow_result, sm_count, s));
      SB_CKE(cudaMemcpyAsync(pin, fb.pow_result, 8, cudaMemcpyDeviceToHost, s));
      SB_CKE(stream_wait(s));
      out.gap_start = Clock::now();
      std::memcpy(&nonce, pin, 8);
      if (nonce == ~0ull && deadline.passed()) {
        err = "proof deadline passed during the proof-of-work search";
        return E_TIMEOUT;
      }
    }
    if (nonce == ~0ull) { err = "proof-of-work search bound reached"; return E_TIMEOUT; }
  }
  ch.mix_u64(nonce);
  if (ev_pow) SB_CKE(cudaEventRecord(ev_pow, s));

  // Queries (src/core/queries.zig:8-60).
  std::vector<uint64_t>& queries = out.queries;
  {
    uint32_t mask = (uint32_t)((1ull << L) - 1);
    while (queries.size() < cfg.n_queries) {
      uint32_t w[8];
      ch.draw_u32s(w);
      for (uint32_t x : w) { queries.push_back(x & mask); if (queries.size() == cfg.n_queries) break; }
    }
    std::sort(queries.begin(), queries.end());
    queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  }

  return OK;
}

void DecommitPlan::add_tree(const uint8_t* layers, uint32_t max_log, const std::vector<const uint32_t*>& cols,
                            const std::vector<uint64_t>& queries) {
  TreePlan tp;
  n_queries_ = queries.size();
  tp.word0 = words_.size();
  tp.n_cols = cols.size();
  words_.reserve(words_.size() + cols.size() * queries.size());
  if (!cols.empty()) hashes_.reserve(hashes_.size() + queries.size() * max_log);
  for (const uint32_t* c : cols)
    for (uint64_t q : queries) words_.push_back({c, q});
  tp.hash0 = hashes_.size();
  if (!cols.empty()) {
    std::vector<uint64_t> uniq(queries);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    for (uint64_t nd : witness_nodes(max_log, uniq)) hashes_.push_back({layers, nd});
  }
  tp.n_hash = hashes_.size() - tp.hash0;
  trees_.push_back(tp);
}

void DecommitPlan::add_fri(const FriBuffers& fb, uint32_t L, uint32_t n_inner, const std::vector<uint64_t>& queries) {
  std::vector<uint64_t> lq = queries;
  // At most two positions per query and layer: four coordinate words each, and their witnesses.
  words_.reserve(words_.size() + (size_t)(n_inner + 1) * 8 * queries.size());
  hashes_.reserve(hashes_.size() + (size_t)(n_inner + 1) * 2 * queries.size() * L);
  std::vector<uint64_t> positions;
  positions.reserve(2 * queries.size());
  for (uint32_t k = 0; k <= n_inner; ++k) {
    // k = 0: first layer (quotient column, log L); k >= 1: inner layer k-1.
    const uint32_t* colbase = k == 0 ? fb.quot : fb.line[k - 1];
    uint64_t csz = k == 0 ? (1ull << L) : (1ull << (L - k));
    uint32_t lg = k == 0 ? L : L - k;
    const uint8_t* tree = k == 0 ? fb.tree_q : fb.line_tree[k - 1];
    LayerPlan lp{words_.size(), 0, hashes_.size(), 0};
    positions.clear();
    size_t q = 0;
    while (q < lq.size()) {
      uint64_t key = lq[q] >> 1;
      size_t end = q + 1;
      while (end < lq.size() && (lq[end] >> 1) == key) ++end;
      size_t at = q;
      for (uint64_t pos = key << 1; pos < (key << 1) + 2; ++pos) {
        positions.push_back(pos);
        if (at < end && lq[at] == pos) { ++at; continue; }
        for (int c = 0; c < 4; ++c) words_.push_back({colbase + c * csz, pos});
        lp.n_wit += 1;
      }
      q = end;
    }
    std::vector<uint64_t> wn = witness_nodes(lg, positions);
    for (uint64_t nd : wn) hashes_.push_back({tree, nd});
    lp.n_hash = wn.size();
    fri_.push_back(lp);
    // fold queries
    std::vector<uint64_t> nq;
    for (uint64_t p : lq) { uint64_t f = p >> 1; if (nq.empty() || nq.back() != f) nq.push_back(f); }
    lq.swap(nq);
  }
}

int32_t DecommitPlan::gather(uint8_t* scratch, size_t scratch_bytes, uint8_t* pin, size_t pin_bytes, cudaStream_t fs,
                             cudaEvent_t ev_done, std::string& err) {
  size_t words_bytes = words_.size() * sizeof(GatherItem), hash_items_bytes = hashes_.size() * sizeof(HashGatherItem);
  size_t out_words_bytes = words_.size() * 4, out_hash_bytes = hashes_.size() * 32;
  size_t total = 4 * 256 + words_bytes + hash_items_bytes + out_words_bytes + out_hash_bytes;
  if (total > scratch_bytes || total > pin_bytes) {
    err = "decommitment exceeds staging capacity";
    return E_INVALID;
  }
  size_t o_items = 0, o_hitems = (words_bytes + 255) & ~255ull, o_outw = (o_hitems + hash_items_bytes + 255) & ~255ull,
         o_outh = (o_outw + out_words_bytes + 255) & ~255ull;
  std::memcpy(pin + o_items, words_.data(), words_bytes);
  std::memcpy(pin + o_hitems, hashes_.data(), hash_items_bytes);
  SB_CKE(cudaMemcpyAsync(scratch, pin, o_outw, cudaMemcpyHostToDevice, fs));
  SB_CKE(gather_words(reinterpret_cast<GatherItem*>(scratch + o_items), (uint32_t)words_.size(),
                      reinterpret_cast<uint32_t*>(scratch + o_outw), fs));
  SB_CKE(gather_hashes(reinterpret_cast<HashGatherItem*>(scratch + o_hitems), (uint32_t)hashes_.size(),
                       scratch + o_outh, fs));
  SB_CKE(cudaMemcpyAsync(pin + o_outw, scratch + o_outw, o_outh - o_outw + out_hash_bytes, cudaMemcpyDeviceToHost,
                         fs));
  if (ev_done) SB_CKE(cudaEventRecord(ev_done, fs));
  SB_CKE(stream_wait(fs));
  gw_ = reinterpret_cast<const uint32_t*>(pin + o_outw);
  gh_ = pin + o_outh;
  return OK;
}

void DecommitPlan::hash_list(Json& j, size_t first, size_t count) const {
  j.ch('[');
  for (size_t i = 0; i < count; ++i) { if (i) j.ch(','); j.hash(gh_ + (first + i) * 32); }
  j.ch(']');
}

void DecommitPlan::json_witness(Json& j, size_t tree) const {
  hash_list(j, trees_[tree].hash0, trees_[tree].n_hash);
}

void DecommitPlan::json_queried(Json& j, size_t tree) const {
  const TreePlan& tp = trees_[tree];
  j.ch('[');
  for (size_t c = 0; c < tp.n_cols; ++c) {
    if (c) j.ch(',');
    j.ch('[');
    for (size_t q = 0; q < n_queries_; ++q) { if (q) j.ch(','); j.u(gw_[tp.word0 + c * n_queries_ + q]); }
    j.ch(']');
  }
  j.ch(']');
}

void DecommitPlan::json_fri(Json& j, const FriResult& fr) const {
  auto layer = [&](size_t k) {
    const LayerPlan& lp = fri_[k];
    j.lit("{\"fri_witness\":[");
    for (size_t i = 0; i < lp.n_wit; ++i) {
      if (i) j.ch(',');
      const uint32_t* w = gw_ + lp.wit_word0 + 4 * i;
      j.qm(qmake(w[0], w[1], w[2], w[3]));
    }
    j.lit("],\"decommitment\":{\"hash_witness\":");
    hash_list(j, lp.hash0, lp.n_hash);
    j.lit("},\"commitment\":");
    j.hash(fr.roots[k].data());
    j.ch('}');
  };
  j.lit("{\"first_layer\":");
  layer(0);
  j.lit(",\"inner_layers\":[");
  for (size_t k = 1; k < fri_.size(); ++k) { if (k > 1) j.ch(','); layer(k); }
  j.lit("],\"last_layer_poly\":[");
  for (size_t i = 0; i < fr.last_coeffs.size(); ++i) { if (i) j.ch(','); j.qm(fr.last_coeffs[i]); }
  j.lit("]}");
}

}  // namespace sb
