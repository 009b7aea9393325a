// Host-side pieces shared by the provers: the Blake2s channel, proof JSON
// writer, Merkle witness plans, workspace arena, and the proof tail (FRI, last
// layer, proof of work, queries, decommitment gathers) over a quotient column.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "blake2s.cuh"
#include "host_wait.hpp"
#include "prover.hpp"

namespace sb {

// ---------------------------------------------------------------------------
// Host Blake2s channel (src/core/channel/blake2s.zig:33-280).
// ---------------------------------------------------------------------------
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
inline PointQ random_secure_point(Channel& ch) {
  QM31 t = ch.draw_secure_felt();
  QM31 t2 = qsq(t);
  QM31 inv = qinv(qadd(t2, qone()));
  return {qmul(qsub(qone(), t2), inv), qmul(qadd(t, t), inv)};
}

// cosetVanishing (src/core/constraints.zig:17-27) on base and secure points.
inline uint32_t coset_vanishing_m(const PointTable& pt, const Coset& c, PointM p) {
  PointM q = padd(padd(p, pconj(pt.at(c.initial))), pt.at(c.step / 2));
  uint32_t x = q.x;
  for (uint32_t i = 1; i < c.log_size; ++i) x = double_x(x);
  return x;
}

inline const PointTable& host_points() {
  static std::vector<PointM> t = build_point_table();
  static PointTable pt{t.data()};
  return pt;
}

// Proof JSON writer. A proof holds hundreds of thousands of decimal numbers (hash bytes
// above all), so the text goes straight into a growable byte buffer: digits two at a time
// from a table, hashes from per-byte strings, one bounds check per item.
class Json {
 public:
  Json() = default;
  Json(const Json&) = delete;
  Json& operator=(const Json&) = delete;
  ~Json() { std::free(buf_); }
  void reserve(size_t k) { grow(k); }
  void ch(char c) {
    grow(1);
    buf_[n_++] = c;
  }
  template <size_t K>
  void lit(const char (&text)[K]) {  // a string literal, without its terminator
    grow(K - 1);
    std::memcpy(buf_ + n_, text, K - 1);
    n_ += K - 1;
  }
  void u(uint64_t v) {
    grow(20);
    n_ += digits(v, buf_ + n_);
  }
  void hash(const uint8_t* h) {
    const Bytes& t = bytes();
    grow(1 + 32 * 4);
    char* p = buf_ + n_;
    *p++ = '[';
    for (int i = 0; i < 32; ++i) {
      std::memcpy(p, t.txt[h[i]], 4);  // fixed-size copy; only len bytes are kept
      p += t.len[h[i]];
    }
    p[-1] = ']';  // the last ',' closes the list
    n_ = p - buf_;
  }
  void qm(QM31 q) {
    uint32_t w[4];
    qstore4(q, w);
    grow(4 * 11 + 2);
    char* p = buf_ + n_;
    *p++ = '[';
    for (int i = 0; i < 4; ++i) {
      if (i) *p++ = ',';
      p += digits(w[i], p);
    }
    *p++ = ']';
    n_ = p - buf_;
  }
  std::string str() const { return std::string(buf_ ? buf_ : "", n_); }

 private:
  struct Bytes {  // decimal text of every byte value followed by ',', and its length
    char txt[256][4];
    uint8_t len[256];
    Bytes() {
      for (int b = 0; b < 256; ++b) {
        char t[8];
        int n = std::snprintf(t, sizeof(t), "%d,", b);
        std::memcpy(txt[b], t, 4);
        len[b] = (uint8_t)n;
      }
    }
  };
  static const Bytes& bytes() {
    static const Bytes b;
    return b;
  }
  // Writes v in decimal at p; returns the number of characters.
  static size_t digits(uint64_t v, char* p) {
    static const char* kPairs =
        "00010203040506070809101112131415161718192021222324252627282930313233343536373839"
        "40414243444546474849505152535455565758596061626364656667686970717273747576777879"
        "8081828384858687888990919293949596979899";
    char tmp[24];
    char* e = tmp + sizeof(tmp);
    char* q = e;
    while (v >= 100) {
      const unsigned r = (unsigned)(v % 100);
      v /= 100;
      q -= 2;
      q[0] = kPairs[2 * r];
      q[1] = kPairs[2 * r + 1];
    }
    if (v >= 10) {
      q -= 2;
      q[0] = kPairs[2 * v];
      q[1] = kPairs[2 * v + 1];
    } else {
      *--q = (char)('0' + v);
    }
    const size_t k = e - q;
    std::memcpy(p, q, k);
    return k;
  }
  void grow(size_t k) {
    if (n_ + k <= cap_) return;
    size_t cap = std::max(cap_ * 2, n_ + k + 4096);
    char* nb = static_cast<char*>(std::realloc(buf_, cap));
    if (!nb) throw std::bad_alloc();
    buf_ = nb;
    cap_ = cap;
  }
  char* buf_ = nullptr;
  size_t n_ = 0, cap_ = 0;
};

// Decommitment plan of a lifted tree at sorted unique leaf positions: the nodes
// whose hashes are witnesses, in proof order (src/prover/vcs_lifted/decommit.zig:154-230).
inline std::vector<uint64_t> witness_nodes(uint32_t max_log, const std::vector<uint64_t>& positions) {
  std::vector<uint64_t> out, prev = positions, cur;
  out.reserve(positions.size() * max_log);
  cur.reserve(positions.size());
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


constexpr size_t GATHER_SCRATCH = 8 << 20;

// ---------------------------------------------------------------------------
// Proof tail over a committed quotient column (src/prover/fri.zig:163-619,
// src/prover/pcs/scheme.zig:633-799): FRI first layer and inner layers (each
// root mixed before its fold's alpha is drawn), the last layer's coefficients,
// the proof of work and the queries.
// ---------------------------------------------------------------------------
struct FriBuffers {
  uint32_t* quot;                   // 4 coordinate columns of 2^L
  uint8_t* tree_q;                  // first-layer tree
  std::vector<uint32_t*> line;      // line layers 0..n_inner (the last one is the last layer)
  std::vector<uint8_t*> line_tree;  // trees of line layers 0..n_inner-1
  uint32_t* pow_result;             // 2 words of device scratch
  FriChannelDev* chan;              // device channel of the FRI commit phase
};
struct FriResult {
  std::vector<std::array<uint8_t, 32>> roots;  // first layer, then inner layers
  std::vector<QM31> last_coeffs;
  uint64_t nonce = 0;
  std::vector<uint64_t> queries;  // sorted, unique
  // Host time between the stream synchronizations of the tail and the next device work (the
  // FRI channel replay and last layer, the proof-of-work checks, the query draw), milliseconds.
  float host_gap_ms = 0;
  Clock::time_point gap_start;    // when the last synchronization of the tail returned
};
// Runs on `fs` (FRI, latency-bound) and `s` (proof of work); `pin` is pinned host staging
// (at least 64 KB). The FRI layers draw their alphas on the device (FriChannelDev); the
// host replays the same channel steps from the returned roots and checks every alpha.
// ev_fri and ev_pow (nullable) are recorded after the last layer and after the grind. A deadline
// that passes during the grind ends it after the current rounds with E_TIMEOUT.
int32_t fri_pow_queries(const DeviceTables& T, int sm_count, Channel& ch, const PcsConfig& cfg, uint32_t L,
                        uint32_t n_inner, uint32_t last_log, const FriBuffers& fb, uint8_t* pin, cudaStream_t s,
                        cudaStream_t fs, cudaEvent_t ev_fri, cudaEvent_t ev_pow, const Deadline& deadline,
                        FriResult& out, std::string& err);

// ---------------------------------------------------------------------------
// Decommitment (src/prover/vcs_lifted/decommit.zig:56-352, src/prover/fri.zig:624-850):
// the queried values and witness hashes of every tree, and the FRI layers' witnesses,
// gathered on the device in one pass and copied back once.
// ---------------------------------------------------------------------------
class DecommitPlan {
 public:
  // A trace tree of `cols` columns (each 2^max_log words): their values at `queries` (one
  // position per query, in query order; repeats allowed, as when a smaller preprocessed tree
  // takes the lifting domain's positions mapped down) and the witness of the sorted unique
  // positions. A tree without columns contributes nothing.
  void add_tree(const uint8_t* layers, uint32_t max_log, const std::vector<const uint32_t*>& cols,
                const std::vector<uint64_t>& queries);
  void add_fri(const FriBuffers& fb, uint32_t L, uint32_t n_inner, const std::vector<uint64_t>& queries);
  // Gathers through `scratch` (device) and `pin` (pinned host); synchronizes `fs`.
  int32_t gather(uint8_t* scratch, size_t scratch_bytes, uint8_t* pin, size_t pin_bytes, cudaStream_t fs,
                 cudaEvent_t ev_done, std::string& err);
  void json_witness(Json& j, size_t tree) const;   // [hash, ...]
  void json_queried(Json& j, size_t tree) const;   // [[col 0 values], [col 1 values], ...]
  void json_fri(Json& j, const FriResult& fr) const;

 private:
  struct TreePlan { size_t word0 = 0, n_cols = 0, hash0 = 0, n_hash = 0; };
  struct LayerPlan { size_t wit_word0, n_wit, hash0, n_hash; };
  std::vector<GatherItem> words_;
  std::vector<HashGatherItem> hashes_;
  std::vector<TreePlan> trees_;
  std::vector<LayerPlan> fri_;
  size_t n_queries_ = 0;
  const uint32_t* gw_ = nullptr;
  const uint8_t* gh_ = nullptr;
  void hash_list(Json& j, size_t first, size_t count) const;
};

}  // namespace sb
