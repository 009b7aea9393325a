// Host-side verifier of the proofs this library emits (wide-Fibonacci and the LogUp
// XOR-lookup AIR), run on host threads so that a serving loop can check every proof
// without stalling the device. It follows the reference verifier:
//   src/examples/wide_fibonacci.zig:360-433 (verify), src/core/verifier.zig (OODS check),
//   src/core/pcs/verifier.zig:79-178, src/core/pcs/quotients/fri_answers.zig (quotient
//   answers), src/core/fri.zig (FRI layers and last layer), src/core/vcs_lifted/verifier.zig
//   (lifted Merkle decommitment), src/core/channel/blake2s.zig (channel and PoW),
// reading the JSON wire layout of src/interop/proof_wire.zig:19-77. No device code.
#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "prover_common.hpp"
#include "verifier.hpp"

namespace sb {

namespace {

// ---- minimal JSON reader for the proof wire (unsigned integers, arrays, objects, null) ------
struct JV {
  enum Kind { NUM, ARR, OBJ, NUL } kind = NUL;
  uint64_t num = 0;
  std::vector<JV> arr;
  std::vector<std::pair<std::string, JV>> obj;
  const JV& at(size_t i) const {
    if (kind != ARR || i >= arr.size()) throw std::runtime_error("proof shape");
    return arr[i];
  }
  const JV& operator[](const char* key) const {
    if (kind == OBJ)
      for (const auto& kv : obj)
        if (kv.first == key) return kv.second;
    throw std::runtime_error(std::string("missing field ") + key);
  }
  size_t size() const {
    if (kind != ARR) throw std::runtime_error("proof shape");
    return arr.size();
  }
  uint64_t u() const {
    if (kind != NUM) throw std::runtime_error("proof shape");
    return num;
  }
};

struct Parser {
  const char* p;
  const char* end;
  int depth = 0;
  void ws() { while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p; }
  JV value() {
    if (++depth > 64) throw std::runtime_error("proof nesting");
    ws();
    if (p >= end) throw std::runtime_error("truncated proof");
    JV v;
    if (*p == '[') {
      v.kind = JV::ARR;
      ++p;
      ws();
      if (p < end && *p == ']') { ++p; --depth; return v; }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (p < end && *p == ',') { ++p; continue; }
        if (p < end && *p == ']') { ++p; break; }
        throw std::runtime_error("bad array");
      }
    } else if (*p == '{') {
      v.kind = JV::OBJ;
      ++p;
      ws();
      if (p < end && *p == '}') { ++p; --depth; return v; }
      for (;;) {
        ws();
        if (p >= end || *p != '"') throw std::runtime_error("bad object key");
        const char* k0 = ++p;
        while (p < end && *p != '"') ++p;
        if (p >= end) throw std::runtime_error("bad object key");
        std::string key(k0, p - k0);
        ++p;
        ws();
        if (p >= end || *p != ':') throw std::runtime_error("bad object");
        ++p;
        v.obj.emplace_back(key, value());
        ws();
        if (p < end && *p == ',') { ++p; continue; }
        if (p < end && *p == '}') { ++p; break; }
        throw std::runtime_error("bad object");
      }
    } else if (*p >= '0' && *p <= '9') {
      v.kind = JV::NUM;
      uint64_t x = 0;
      while (p < end && *p >= '0' && *p <= '9') {
        uint64_t d = (uint64_t)(*p - '0');
        if (x > (~0ull - d) / 10) throw std::runtime_error("number overflow");
        x = x * 10 + d;
        ++p;
      }
      v.num = x;
    } else if (end - p >= 4 && std::string(p, 4) == "null") {
      p += 4;
    } else {
      throw std::runtime_error("unexpected token");
    }
    --depth;
    return v;
  }
};

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

uint32_t canon(uint64_t v) {
  if (v >= P) throw Fail("non-canonical field element");
  return (uint32_t)v;
}
QM31 qm(const JV& v) {
  if (v.size() != 4) throw Fail("QM31 shape");
  return qmake(canon(v.at(0).u()), canon(v.at(1).u()), canon(v.at(2).u()), canon(v.at(3).u()));
}
std::array<uint8_t, 32> hash_of(const JV& v) {
  if (v.size() != 32) throw Fail("hash shape");
  std::array<uint8_t, 32> h;
  for (int i = 0; i < 32; ++i) {
    uint64_t b = v.at(i).u();
    if (b > 255) throw Fail("hash byte");
    h[i] = (uint8_t)b;
  }
  return h;
}

using Hash = std::array<uint8_t, 32>;

Hash b2s(const void* a, size_t la, const void* b = nullptr, size_t lb = 0) {
  Blake2sHost h;
  h.update(a, la);
  if (lb) h.update(b, lb);
  Hash o;
  h.finalize(o.data());
  return o;
}

// Prefixed lifted-Merkle leaf and node hashes (src/core/vcs_lifted/blake2_merkle.zig).
Hash leaf_hash(const std::vector<uint32_t>& row) {
  uint8_t prefix[64] = {0};
  std::memcpy(prefix, "leaf", 4);
  return b2s(prefix, 64, row.data(), row.size() * 4);
}
Hash node_hash(const Hash& l, const Hash& r) {
  uint8_t buf[128] = {0};
  std::memcpy(buf, "node", 4);
  std::memcpy(buf + 64, l.data(), 32);
  std::memcpy(buf + 96, r.data(), 32);
  return b2s(buf, 128);
}

// Equal-size columns at `positions` (any order, duplicates allowed): cols[c][j] is column c at
// positions[j] (src/core/vcs_lifted/verifier.zig:94-250).
// A leaf hashes its row of values in column order stably sorted by log size (`col_logs`; equal
// sizes when empty), a smaller column's value being the one at the lifted index.
void merkle_verify(const Hash& root, uint32_t max_log, const std::vector<uint64_t>& positions,
                   const std::vector<std::vector<uint32_t>>& cols, const std::vector<Hash>& witness,
                   const std::vector<uint32_t>& col_logs = {}) {
  if (cols.empty()) {
    if (!witness.empty()) throw Fail("witness for an empty tree");
    return;
  }
  std::vector<size_t> corder(cols.size());
  for (size_t c = 0; c < cols.size(); ++c) corder[c] = c;
  if (!col_logs.empty())
    std::stable_sort(corder.begin(), corder.end(), [&](size_t x, size_t y) { return col_logs[x] < col_logs[y]; });
  std::map<uint64_t, Hash> leaves;
  for (size_t j = 0; j < positions.size(); ++j) {
    std::vector<uint32_t> row(cols.size());
    for (size_t c = 0; c < cols.size(); ++c) row[c] = cols[corder[c]][j];
    Hash h = leaf_hash(row);
    auto it = leaves.find(positions[j]);
    if (it != leaves.end() && it->second != h) throw Fail("duplicate query mismatch");
    leaves[positions[j]] = h;
  }
  std::vector<std::pair<uint64_t, Hash>> prev(leaves.begin(), leaves.end()), cur;
  size_t wi = 0;
  for (uint32_t layer = 0; layer < max_log; ++layer) {
    cur.clear();
    size_t p = 0;
    while (p < prev.size()) {
      uint64_t idx = prev[p].first;
      Hash left, right;
      size_t step;
      if (p + 1 < prev.size() && prev[p + 1].first == (idx ^ 1)) {
        left = prev[p].second;
        right = prev[p + 1].second;
        step = 2;
      } else {
        if (wi >= witness.size()) throw Fail("witness too short");
        const Hash& w = witness[wi++];
        left = (idx & 1) == 0 ? prev[p].second : w;
        right = (idx & 1) == 0 ? w : prev[p].second;
        step = 1;
      }
      cur.emplace_back(idx >> 1, node_hash(left, right));
      p += step;
    }
    prev.swap(cur);
  }
  if (wi != witness.size()) throw Fail("witness too long");
  if (prev.size() != 1 || prev[0].second != root) throw Fail("root mismatch");
}

bool pow_ok(const uint8_t digest[32], uint32_t bits, uint64_t nonce) {
  uint8_t pre_in[52] = {0};
  uint32_t tag = 0x12345678u;
  std::memcpy(pre_in, &tag, 4);
  std::memcpy(pre_in + 16, digest, 32);
  std::memcpy(pre_in + 48, &bits, 4);
  Hash prefix = b2s(pre_in, 52);
  uint8_t in[40];
  std::memcpy(in, prefix.data(), 32);
  std::memcpy(in + 32, &nonce, 8);
  Hash h = b2s(in, 40);
  uint32_t tz = 0;
  for (int i = 0; i < 16 && tz == 8u * i; ++i) {
    uint8_t b = h[i];
    if (b == 0) tz += 8;
    else { tz += __builtin_ctz(b); break; }
  }
  return tz >= bits;
}

PointM index_point(uint32_t idx) { return host_points().at(idx); }

QM31 coset_vanishing_q(uint32_t log, uint32_t initial, uint32_t step, PointQ p) {
  PointM ini = index_point(initial), hs = index_point(step / 2);
  PointQ q = qpadd(qpadd(p, PointQ{qbase(ini.x), qneg(qbase(ini.y))}), PointQ{qbase(hs.x), qbase(hs.y)});
  QM31 x = q.x;
  for (uint32_t i = 1; i < log; ++i) x = qdouble_x(x);
  return x;
}

uint32_t bitrev_h(uint64_t i, uint32_t log) {
  uint64_t r = 0;
  for (uint32_t k = 0; k < log; ++k) { r = (r << 1) | (i & 1); i >>= 1; }
  return (uint32_t)r;
}

struct Cfg {
  uint32_t pow_bits, B, log_last, n_queries;
};

Cfg read_config(const JV& pr) {
  const JV& cfg = pr["config"];
  const JV& fc = cfg["fri_config"];
  Cfg c{(uint32_t)cfg["pow_bits"].u(), (uint32_t)fc["log_blowup_factor"].u(),
        (uint32_t)fc["log_last_layer_degree_bound"].u(), (uint32_t)fc["n_queries"].u()};
  if (fc["fold_step"].u() != 1 || cfg["lifting_log_size"].kind != JV::NUL) throw Fail("unsupported config");
  if (c.B < 1 || c.B > 8 || c.n_queries == 0 || c.n_queries > 4096 || c.pow_bits > 64 || c.log_last > 20)
    throw Fail("config out of range");
  return c;
}

QM31 secure_of(const QM31* v) {
  return qadd(qadd(v[0], qmul(v[1], qmake(0, 1, 0, 0))), qadd(qmul(v[2], qmake(0, 0, 1, 0)), qmul(v[3], qmake(0, 0, 0, 1))));
}

struct BatchEntry {
  size_t col;
  QM31 value, rp;
};
struct Batch {
  PointQ point;
  std::vector<BatchEntry> entries;
};

// FRI commitments and alphas, last layer, PoW, queries, tree decommitments and quotient answers,
// FRI decommitment (the verifier's PCS tail).
// tree_logs (optional): the committed log sizes of each tree's columns. A tree's depth is its largest
// column; the preprocessed tree (tree 0), when smaller than the lifting domain, is queried at the
// positions mapped down (preparePreprocessedQueryPositions, src/core/pcs/utils.zig:292-314).
void pcs_tail(const JV& pr, Channel& ch, const std::vector<Hash>& roots, const std::vector<uint32_t>& tree_cols,
              const std::vector<Batch>& batches, uint32_t L, const Cfg& cfg,
              const std::vector<std::vector<uint32_t>>& tree_logs = {}) {
  const JV& fri = pr["fri_proof"];
  ch.mix_root(hash_of(fri["first_layer"]["commitment"]).data());
  std::vector<QM31> alphas{ch.draw_secure_felt()};
  if (cfg.log_last + cfg.B + 1 > L) throw Fail("last layer larger than the domain");
  const uint32_t n_inner = (L - 1) - (cfg.log_last + cfg.B);
  const JV& inner = fri["inner_layers"];
  if (inner.size() != n_inner) throw Fail("number of FRI layers");
  for (size_t k = 0; k < n_inner; ++k) {
    ch.mix_root(hash_of(inner.at(k)["commitment"]).data());
    alphas.push_back(ch.draw_secure_felt());
  }
  std::vector<QM31> last;
  for (const JV& v : fri["last_layer_poly"].arr) last.push_back(qm(v));
  if (last.size() > (1ull << cfg.log_last)) throw Fail("last layer degree");
  ch.mix_felts(last.data(), last.size());
  const uint64_t nonce = pr["proof_of_work"].u();
  if (!pow_ok(ch.digest, cfg.pow_bits, nonce)) throw Fail("proof of work");
  ch.mix_u64(nonce);
  std::vector<uint64_t> queries;
  {
    const uint32_t mask = (uint32_t)((1ull << L) - 1);
    while (queries.size() < cfg.n_queries) {
      uint32_t w[8];
      ch.draw_u32s(w);
      for (uint32_t x : w) { queries.push_back(x & mask); if (queries.size() == cfg.n_queries) break; }
    }
    std::sort(queries.begin(), queries.end());
    queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  }
  const JV& qv = pr["queried_values"];
  const JV& dec = pr["decommitments"];
  if (qv.size() != tree_cols.size() || dec.size() != tree_cols.size()) throw Fail("number of trees");
  std::vector<std::vector<uint32_t>> cols;  // flattened over the trees with columns
  for (size_t t = 0; t < tree_cols.size(); ++t) {
    const JV& tq = qv.at(t);
    if (tq.size() != tree_cols[t]) throw Fail("queried values shape");
    std::vector<std::vector<uint32_t>> tc;
    for (const JV& c : tq.arr) {
      if (c.size() != queries.size()) throw Fail("queried values shape");
      std::vector<uint32_t> col;
      for (const JV& x : c.arr) col.push_back(canon(x.u()));
      tc.push_back(std::move(col));
    }
    std::vector<Hash> wit;
    for (const JV& h : dec.at(t)["hash_witness"].arr) wit.push_back(hash_of(h));
    if (tree_cols[t] == 0) {
      if (!wit.empty()) throw Fail("preprocessed tree shape");
      continue;
    }
    const std::vector<uint32_t> logs = tree_logs.empty() ? std::vector<uint32_t>{} : tree_logs[t];
    const uint32_t depth = logs.empty() ? L : *std::max_element(logs.begin(), logs.end());
    std::vector<uint64_t> positions = queries;
    if (depth != L) {
      if (t != 0 || depth > L) throw Fail("tree size");
      const uint32_t sh = L - depth + 1;
      for (uint64_t& p : positions) p = ((p >> sh) << 1) + (p & 1);
    }
    merkle_verify(roots[t], depth, positions, tc, wit, logs);
    for (auto& c : tc) cols.push_back(std::move(c));
  }
  // quotient answers at the queries
  struct Const { PointQ point; std::vector<std::pair<size_t, QM31>> lc; QM31 sum_a, sum_b; };
  std::vector<Const> consts;
  for (const Batch& b : batches) {
    Const c{b.point, {}, qzero(), qzero()};
    QM31 cy = qsub(qconj(b.point.y), b.point.y);
    for (const BatchEntry& e : b.entries) {
      if (e.col >= cols.size()) throw Fail("sample column");
      QM31 aa = qsub(qconj(e.value), e.value);
      QM31 bb = qsub(qmul(e.value, cy), qmul(aa, b.point.y));
      c.lc.emplace_back(e.col, qmul(e.rp, cy));
      c.sum_a = qadd(c.sum_a, qmul(e.rp, aa));
      c.sum_b = qadd(c.sum_b, qmul(e.rp, bb));
    }
    consts.push_back(std::move(c));
  }
  CircleDomain dom = canonic_domain(L);
  std::vector<QM31> answers;
  for (size_t j = 0; j < queries.size(); ++j) {
    PointM dp = index_point(dom.index_at(bitrev_h(queries[j], L)));
    QM31 acc = qzero();
    for (const Const& c : consts) {
      QM31 num = qzero();
      for (const auto& e : c.lc) num = qadd(num, qmulm(e.second, cols[e.first][j]));
      num = qsub(num, qadd(qmulm(c.sum_a, dp.y), c.sum_b));
      CM31 prx = c.point.x.c0, pry = c.point.y.c0, pix = c.point.x.c1, piy = c.point.y.c1;
      CM31 den = csub(cmul(csub(prx, CM31{dp.x, 0}), piy), cmul(csub(pry, CM31{dp.y, 0}), pix));
      if (den.a == 0 && den.b == 0) throw Fail("degenerate quotient denominator");
      acc = qadd(acc, qmulc(num, cinv(den)));
    }
    answers.push_back(acc);
  }
  // FRI layers: (positions, evaluations) folded layer by layer
  auto ibfly_fold = [](QM31 f0, QM31 f1, uint32_t inv_t, QM31 alpha) {
    return qadd(qadd(f0, f1), qmul(alpha, qmulm(qsub(f0, f1), inv_t)));
  };
  auto layer_check = [&](const JV& layer, std::vector<uint64_t>& qpos, std::vector<QM31>& qev, uint32_t log_size,
                         auto fold) {
    std::vector<QM31> witness;
    for (const JV& w : layer["fri_witness"].arr) witness.push_back(qm(w));
    size_t wi = 0;
    std::vector<uint64_t> dpos;
    std::vector<QM31> dvals, folded;
    size_t i = 0;
    while (i < qpos.size()) {
      uint64_t key = qpos[i] >> 1;
      size_t end = i;
      while (end < qpos.size() && (qpos[end] >> 1) == key) ++end;
      QM31 sub[2];
      size_t at = i;
      for (int k = 0; k < 2; ++k) {
        uint64_t pos = (key << 1) + k;
        dpos.push_back(pos);
        if (at < end && qpos[at] == pos) {
          sub[k] = qev[at++];
        } else {
          if (wi >= witness.size()) throw Fail("fri witness too short");
          sub[k] = witness[wi++];
        }
        dvals.push_back(sub[k]);
      }
      folded.push_back(fold(key, sub[0], sub[1]));
      i = end;
    }
    if (wi != witness.size()) throw Fail("fri witness too long");
    std::vector<std::vector<uint32_t>> colvals(4);
    for (const QM31& v : dvals) {
      uint32_t w[4];
      qstore4(v, w);
      for (int k = 0; k < 4; ++k) colvals[k].push_back(w[k]);
    }
    std::vector<Hash> hw;
    for (const JV& h : layer["decommitment"]["hash_witness"].arr) hw.push_back(hash_of(h));
    merkle_verify(hash_of(layer["commitment"]), log_size, dpos, colvals, hw);
    std::vector<uint64_t> nq;
    for (uint64_t p : qpos) { uint64_t f = p >> 1; if (nq.empty() || nq.back() != f) nq.push_back(f); }
    qpos.swap(nq);
    qev.swap(folded);
  };
  std::vector<uint64_t> qpos = queries;
  std::vector<QM31> qev = answers;
  {
    Coset half = coset_half_odds(L - 1);
    layer_check(fri["first_layer"], qpos, qev, L, [&](uint64_t key, QM31 f0, QM31 f1) {
      uint32_t y = index_point(half.index_at(bitrev_h(key, L - 1))).y;
      return ibfly_fold(f0, f1, minv(y), alphas[0]);
    });
  }
  for (uint32_t k = 0; k < n_inner; ++k) {
    const uint32_t lg = L - 1 - k;
    Coset c = coset_half_odds(lg);
    layer_check(inner.at(k), qpos, qev, lg, [&](uint64_t key, QM31 f0, QM31 f1) {
      uint32_t x = index_point(c.index_at(bitrev_h(key, lg - 1))).x;
      return ibfly_fold(f0, f1, minv(x), alphas[k + 1]);
    });
  }
  // last layer: the remaining evaluations equal the last polynomial (LinePoly.evalAtPoint)
  const uint32_t last_log = cfg.log_last + cfg.B;
  Coset dom_l = coset_half_odds(last_log);
  uint32_t lg = 0;
  while ((1ull << lg) < last.size()) ++lg;
  for (size_t i = 0; i < qpos.size(); ++i) {
    QM31 x = qbase(index_point(dom_l.index_at(bitrev_h(qpos[i], last_log))).x);
    std::vector<QM31> factors;
    QM31 cur = x;
    for (uint32_t k = 0; k < lg; ++k) { factors.push_back(cur); cur = qdouble_x(cur); }
    std::vector<QM31> v = last;
    for (uint32_t k = lg; k-- > 0;) {  // fold halves with the factor of this level
      size_t h = v.size() / 2;
      for (size_t t = 0; t < h; ++t) v[t] = qadd(v[t], qmul(v[h + t], factors[lg - 1 - k]));
      v.resize(h);
    }
    QM31 val = v.empty() ? qzero() : v[0];
    if (!qeq(val, qev[i])) throw Fail("last layer evaluation");
  }
}

PointQ oods_point(Channel& ch) { return random_secure_point(ch); }

}  // namespace

int32_t verify_wide_fib_json(const std::string& proof, uint32_t log_n, uint32_t W, bool has_seed, uint64_t seed,
                             std::string& err) {
  try {
    Parser ps{proof.data(), proof.data() + proof.size()};
    JV pr = ps.value();
    if (log_n < 1 || log_n > 28 || W < 2) throw Fail("bad statement");
    const Cfg cfg = read_config(pr);
    std::vector<Hash> roots;
    for (const JV& c : pr["commitments"].arr) roots.push_back(hash_of(c));
    if (roots.size() != 3) throw Fail("expected 3 commitments");
    Channel ch;
    {
      QM31 c = qmake(cfg.pow_bits, cfg.B, cfg.n_queries, cfg.log_last);
      ch.mix_felts(&c, 1);
    }
    ch.mix_root(roots[0].data());
    ch.mix_root(roots[1].data());
    { uint32_t st[2] = {log_n, W}; ch.mix_words(st, 2); }
    if (has_seed) ch.mix_u64(seed);
    const QM31 random_coeff = ch.draw_secure_felt();
    ch.mix_root(roots[2].data());
    const PointQ oods = oods_point(ch);
    const JV& sv = pr["sampled_values"];
    if (sv.size() != 3 || sv.at(0).size() != 0 || sv.at(1).size() != W || sv.at(2).size() != 8)
      throw Fail("sampled values shape");
    std::vector<QM31> vals;
    for (size_t t = 1; t < 3; ++t)
      for (const JV& c : sv.at(t).arr) {
        if (c.size() != 1) throw Fail("sampled values shape");
        vals.push_back(qm(c.at(0)));
      }
    // composition OODS check
    QM31 left = secure_of(&vals[W]), right = secure_of(&vals[W + 4]);
    PointQ pt = oods;
    for (uint32_t i = 0; i + 1 < log_n; ++i) pt = qpadd(pt, pt);
    const QM31 comp = qadd(left, qmul(pt.x, right));
    const QM31 dinv = qinv(coset_vanishing_q(log_n, 1u << (31 - (log_n + 1)), 1u << (31 - log_n), oods));
    QM31 acc = qzero(), a = vals[0], b = vals[1];
    for (uint32_t k = 2; k < W; ++k) {
      QM31 c = vals[k];
      acc = qadd(qmul(acc, random_coeff), qmul(qsub(c, qadd(qsq(a), qsq(b))), dinv));
      a = b;
      b = c;
    }
    if (!qeq(acc, comp)) throw Fail("OODS mismatch");
    ch.mix_felts(vals.data(), vals.size());
    const QM31 quot_coeff = ch.draw_secure_felt();
    Batch batch{oods, {}};
    QM31 rp = qone();
    for (size_t c = 0; c < vals.size(); ++c) {
      batch.entries.push_back({c, vals[c], rp});
      rp = qmul(rp, quot_coeff);
    }
    pcs_tail(pr, ch, roots, {0, W, 8}, {batch}, log_n + cfg.B, cfg);
    return OK;
  } catch (const std::exception& e) {
    err = e.what();
    return E_CONSTRAINTS;
  }
}

int32_t verify_logup_xor_json(const std::string& proof, uint32_t log_n, uint32_t log_table, bool has_seed,
                              uint64_t seed, std::string& err) {
  try {
    Parser ps{proof.data(), proof.data() + proof.size()};
    JV pr = ps.value();
    if (log_n < 1 || log_n > 28 || (log_table != 8 && log_table != 16)) throw Fail("bad statement");
    const Cfg cfg = read_config(pr);
    const JV& stm = pr["statement"];
    if (stm["log_n"].u() != log_n || stm["log_table"].u() != log_table) throw Fail("statement mismatch");
    const uint32_t n = log_n, t = log_table, L = std::max(n, t), B = cfg.B;
    std::vector<Hash> roots;
    for (const JV& c : pr["commitments"].arr) roots.push_back(hash_of(c));
    if (roots.size() != 4) throw Fail("expected 4 commitments");
    Channel ch;
    {
      QM31 c = qmake(cfg.pow_bits, cfg.B, cfg.n_queries, cfg.log_last);
      ch.mix_felts(&c, 1);
    }
    ch.mix_root(roots[0].data());
    ch.mix_root(roots[1].data());
    { uint32_t st[2] = {log_n, log_table}; ch.mix_words(st, 2); }
    if (has_seed) ch.mix_u64(seed);
    const QM31 z = ch.draw_secure_felt();
    const QM31 alpha = ch.draw_secure_felt();
    const QM31 alpha2 = qsq(alpha);
    ch.mix_root(roots[2].data());
    const JV& cs = pr["claimed_sums"];
    if (cs.size() != 2) throw Fail("claimed sums");
    QM31 claimed[2] = {qm(cs.at(0)), qm(cs.at(1))};
    ch.mix_felts(claimed, 2);
    if (!qiszero(qadd(claimed[0], claimed[1]))) throw Fail("LogUp claimed sums do not cancel");
    const QM31 random_coeff = ch.draw_secure_felt();
    ch.mix_root(roots[3].data());
    const PointQ oods = oods_point(ch);
    PointM g = index_point(1u << (31 - L));
    const PointQ prev = qpadd(oods, PointQ{qbase(g.x), qneg(qbase(g.y))});  // previous row at the maximal size
    auto doubled = [&](PointQ p, uint32_t k) {  // the point seen by a column of 2^k rows
      for (uint32_t i = k; i < L; ++i) p = qpadd(p, p);
      return p;
    };
    const JV& sv = pr["sampled_values"];
    const size_t shape[4] = {3, 4, 8, 8};
    if (sv.size() != 4) throw Fail("sampled values shape");
    std::vector<QM31> pre, mainv, ic, ip, comp;
    for (size_t tr = 0; tr < 4; ++tr) {
      if (sv.at(tr).size() != shape[tr]) throw Fail("sampled values shape");
      for (const JV& c : sv.at(tr).arr) {
        if (c.size() != (tr == 2 ? 2u : 1u)) throw Fail("sampled values shape");
        if (tr == 0) pre.push_back(qm(c.at(0)));
        if (tr == 1) mainv.push_back(qm(c.at(0)));
        if (tr == 2) { ip.push_back(qm(c.at(0))); ic.push_back(qm(c.at(1))); }
        if (tr == 3) comp.push_back(qm(c.at(0)));
      }
    }
    const QM31 left = secure_of(&comp[0]), right = secure_of(&comp[4]);
    PointQ pt = oods;
    for (uint32_t i = 0; i + 1 < L; ++i) pt = qpadd(pt, pt);
    const QM31 comp_eval = qadd(left, qmul(pt.x, right));
    const QM31 sm = secure_of(&ic[0]), smp = secure_of(&ip[0]), st = secure_of(&ic[4]), stp = secure_of(&ip[4]);
    const QM31 d_main = qsub(qadd(qadd(mainv[0], qmul(alpha, mainv[1])), qmul(alpha2, mainv[2])), z);
    const QM31 d_table = qsub(qadd(qadd(pre[0], qmul(alpha, pre[1])), qmul(alpha2, pre[2])), z);
    const QM31 c_main =
        qsub(qmul(qadd(qsub(sm, smp), qmulm(claimed[0], minv((uint32_t)((1ull << n) % P)))), d_main), qone());
    const QM31 c_table =
        qadd(qmul(qadd(qsub(st, stp), qmulm(claimed[1], minv((uint32_t)((1ull << t) % P)))), d_table), mainv[3]);
    const QM31 z_main = coset_vanishing_q(n, 1u << (31 - (n + 1)), 1u << (31 - n), doubled(oods, n));
    const QM31 z_table = coset_vanishing_q(t, 1u << (31 - (t + 1)), 1u << (31 - t), doubled(oods, t));
    if (!qeq(qadd(qmul(qmul(random_coeff, c_main), qinv(z_main)), qmul(c_table, qinv(z_table))), comp_eval))
      throw Fail("OODS mismatch");
    std::vector<QM31> flat(pre);
    flat.insert(flat.end(), mainv.begin(), mainv.end());
    for (int c = 0; c < 8; ++c) { flat.push_back(ip[c]); flat.push_back(ic[c]); }
    flat.insert(flat.end(), comp.begin(), comp.end());
    ch.mix_felts(flat.data(), flat.size());
    const QM31 quot_coeff = ch.draw_secure_felt();
    // random powers over (tree, column, sample), a two-sample column's periodicity sample first;
    // batches by point in order of first appearance (src/core/pcs/quotients/samples.zig:163-300)
    QM31 rp = qone();
    auto nxt = [&]() { QM31 r = rp; rp = qmul(rp, quot_coeff); return r; };
    std::vector<Batch> batches;
    auto add = [&](const PointQ& p, size_t col, QM31 v) {
      for (Batch& bt : batches)
        if (qeq(bt.point.x, p.x) && qeq(bt.point.y, p.y)) { bt.entries.push_back({col, v, nxt()}); return; }
      batches.push_back(Batch{p, {}});
      batches.back().entries.push_back({col, v, nxt()});
    };
    for (int c = 0; c < 3; ++c) add(oods, (size_t)c, pre[c]);
    for (int c = 0; c < 4; ++c) add(oods, (size_t)(3 + c), mainv[c]);
    for (int c = 0; c < 8; ++c) {
      const uint32_t k = c < 4 ? n : t;
      PointQ per = oods;
      if (k < L) {
        PointM h = index_point(1u << (31 - L + k));
        per = qpadd(oods, PointQ{qbase(h.x), qbase(h.y)});
      }
      add(per, (size_t)(7 + c), ic[c]);
      add(prev, (size_t)(7 + c), ip[c]);
      add(oods, (size_t)(7 + c), ic[c]);
    }
    for (int c = 0; c < 8; ++c) add(oods, (size_t)(15 + c), comp[c]);
    const std::vector<std::vector<uint32_t>> logs = {
        {t + B, t + B, t + B}, {n + B, n + B, n + B, t + B}, {n + B, n + B, n + B, n + B, t + B, t + B, t + B, t + B},
        std::vector<uint32_t>(8, L + B)};
    pcs_tail(pr, ch, roots, {3, 4, 8, 8}, batches, L + B, cfg, logs);
    return OK;
  } catch (const std::exception& e) {
    err = e.what();
    return E_CONSTRAINTS;
  }
}

}  // namespace sb
