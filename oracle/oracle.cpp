// CPU oracle: a plain C++ restatement of the reference prover's algorithm for
// the wide-Fibonacci circle-STARK proof (fields, circle FFT, lifted Blake2s
// Merkle, Blake2s channel, composition, OODS, DEEP quotients, FRI, PoW,
// decommitment, JSON proof wire).
//
// TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline legs may load it, as the checker or as the timed CPU baseline. The
// product library never calls it.
//
// Every section cites the reference file it restates (paths relative to the
// stwo-zig project root). Arithmetic is exact, so any evaluation order that
// computes the same field expression gives the same bits; the order of
// transcript operations, the index maps and the byte layouts follow the
// reference exactly.

#include "oracle_api.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Fields: M31, CM31 = M31[i]/(i^2+1), QM31 = CM31[u]/(u^2-(2+i)).
// src/core/fields/m31.zig:49-75, cm31.zig:97-160, qm31.zig:13,153-223.
// ---------------------------------------------------------------------------
constexpr uint32_t P = 0x7fffffffu;

inline uint32_t madd(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P ? s - P : s; }
inline uint32_t msub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }
inline uint32_t mneg(uint32_t a) { return a == 0 ? 0 : P - a; }
inline uint32_t mmul(uint32_t a, uint32_t b) {
  uint64_t x = (uint64_t)a * b;
  uint64_t r = (x & P) + (x >> 31);
  r = (r & P) + (r >> 31);
  return r >= P ? (uint32_t)(r - P) : (uint32_t)r;
}
inline uint32_t mreduce64(uint64_t x) {  // M31.fromU64
  uint64_t r = (x & P) + (x >> 31);
  r = (r & P) + (r >> 31);
  r = (r & P) + (r >> 31);
  return r >= P ? (uint32_t)(r - P) : (uint32_t)r;
}
uint32_t mpow(uint32_t a, uint64_t e) {
  uint32_t acc = 1;
  while (e) { if (e & 1) acc = mmul(acc, a); a = mmul(a, a); e >>= 1; }
  return acc;
}
inline uint32_t minv(uint32_t a) { return mpow(a, P - 2); }

struct CM31 { uint32_t a, b; };
inline CM31 cadd(CM31 x, CM31 y) { return {madd(x.a, y.a), madd(x.b, y.b)}; }
inline CM31 csub(CM31 x, CM31 y) { return {msub(x.a, y.a), msub(x.b, y.b)}; }
inline CM31 cneg(CM31 x) { return {mneg(x.a), mneg(x.b)}; }
inline CM31 cmul(CM31 x, CM31 y) {
  return {msub(mmul(x.a, y.a), mmul(x.b, y.b)), madd(mmul(x.a, y.b), mmul(x.b, y.a))};
}
inline CM31 cmulm(CM31 x, uint32_t m) { return {mmul(x.a, m), mmul(x.b, m)}; }
inline bool ceq(CM31 x, CM31 y) { return x.a == y.a && x.b == y.b; }
inline bool czero(CM31 x) { return x.a == 0 && x.b == 0; }
CM31 cinv(CM31 x) {
  uint32_t d = minv(madd(mmul(x.a, x.a), mmul(x.b, x.b)));
  return {mmul(x.a, d), mmul(mneg(x.b), d)};
}

struct QM31 { CM31 c0, c1; };
inline QM31 qfrom(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return {{a, b}, {c, d}}; }
inline QM31 qbase(uint32_t a) { return {{a, 0}, {0, 0}}; }
inline QM31 qzero() { return qbase(0); }
inline QM31 qone() { return qbase(1); }
inline QM31 qadd(QM31 x, QM31 y) { return {cadd(x.c0, y.c0), cadd(x.c1, y.c1)}; }
inline QM31 qsub(QM31 x, QM31 y) { return {csub(x.c0, y.c0), csub(x.c1, y.c1)}; }
inline QM31 qneg(QM31 x) { return {cneg(x.c0), cneg(x.c1)}; }
inline CM31 mul_by_r(CM31 x) {  // x * (2 + i)
  return {msub(madd(x.a, x.a), x.b), madd(x.a, madd(x.b, x.b))};
}
inline QM31 qmul(QM31 x, QM31 y) {
  CM31 ac = cmul(x.c0, y.c0), bd = cmul(x.c1, y.c1);
  CM31 cross = csub(csub(cmul(cadd(x.c0, x.c1), cadd(y.c0, y.c1)), ac), bd);
  return {cadd(ac, mul_by_r(bd)), cross};
}
inline QM31 qmulm(QM31 x, uint32_t m) { return {cmulm(x.c0, m), cmulm(x.c1, m)}; }
inline QM31 qmulc(QM31 x, CM31 c) { return {cmul(x.c0, c), cmul(x.c1, c)}; }
inline QM31 qsq(QM31 x) { return qmul(x, x); }
inline bool qeq(QM31 x, QM31 y) { return ceq(x.c0, y.c0) && ceq(x.c1, y.c1); }
inline bool qiszero(QM31 x) { return czero(x.c0) && czero(x.c1); }
inline QM31 qconj(QM31 x) { return {x.c0, cneg(x.c1)}; }
QM31 qinv(QM31 x) {
  // (a + bu)^-1 = (a - bu) / (a^2 - (2+i) b^2)   (qm31.zig:206-222)
  CM31 b2 = cmul(x.c1, x.c1);
  CM31 rb2 = mul_by_r(b2);
  CM31 denom = csub(cmul(x.c0, x.c0), rb2);
  CM31 di = cinv(denom);
  return {cmul(x.c0, di), cmul(cneg(x.c1), di)};
}
inline void qstore(QM31 v, uint32_t out[4]) { out[0] = v.c0.a; out[1] = v.c0.b; out[2] = v.c1.a; out[3] = v.c1.b; }
inline QM31 qload(const uint32_t in[4]) { return qfrom(in[0], in[1], in[2], in[3]); }

// ---------------------------------------------------------------------------
// Circle group over M31 and QM31. src/core/circle.zig:8-131,137-168,172-375.
// ---------------------------------------------------------------------------
struct PointM { uint32_t x, y; };
struct PointQ { QM31 x, y; };
inline PointM padd(PointM a, PointM b) {
  return {msub(mmul(a.x, b.x), mmul(a.y, b.y)), madd(mmul(a.x, b.y), mmul(a.y, b.x))};
}
inline PointM pconj(PointM a) { return {a.x, mneg(a.y)}; }
inline PointM pdbl(PointM a) { return padd(a, a); }
inline PointQ qpadd(PointQ a, PointQ b) {
  return {qsub(qmul(a.x, b.x), qmul(a.y, b.y)), qadd(qmul(a.x, b.y), qmul(a.y, b.x))};
}
inline PointQ qpneg(PointQ a) { return {a.x, qneg(a.y)}; }
inline PointQ qpdbl(PointQ a) { return qpadd(a, a); }
inline PointQ qpfromm(PointM a) { return {qbase(a.x), qbase(a.y)}; }
inline uint32_t double_x(uint32_t x) { uint32_t s = mmul(x, x); return msub(madd(s, s), 1); }
inline QM31 qdouble_x(QM31 x) { QM31 s = qsq(x); return qsub(qadd(s, s), qone()); }

constexpr uint32_t LOG_ORDER = 31;
constexpr uint32_t ORDER_MASK = (1u << 31) - 1;
const PointM GEN = {2, 1268011823};

struct GenDoubles {
  PointM d[LOG_ORDER];
  GenDoubles() { PointM c = GEN; for (uint32_t i = 0; i < LOG_ORDER; ++i) { d[i] = c; c = pdbl(c); } }
};
const GenDoubles& gen_doubles() { static GenDoubles g; return g; }

PointM index_to_point(uint32_t idx) {
  PointM acc = {1, 0};
  uint32_t bits = idx & ORDER_MASK;
  const GenDoubles& g = gen_doubles();
  while (bits) { int b = __builtin_ctz(bits); acc = padd(acc, g.d[b]); bits &= bits - 1; }
  return acc;
}
inline uint32_t subgroup_gen(uint32_t log_size) { return 1u << (LOG_ORDER - log_size); }

struct Coset {
  uint32_t initial_index, step_size, log_size;
  size_t size() const { return (size_t)1 << log_size; }
  uint32_t index_at(size_t i) const { return (initial_index + (uint32_t)((uint64_t)step_size * i)) & ORDER_MASK; }
  PointM at(size_t i) const { return index_to_point(index_at(i)); }
  Coset dbl() const { return {(initial_index * 2) & ORDER_MASK, (step_size * 2) & ORDER_MASK, log_size - 1}; }
  PointM initial() const { return index_to_point(initial_index); }
  PointM half_step() const { return index_to_point(step_size / 2); }
  // Points in natural order (coset.iter()).
  std::vector<PointM> points(size_t n) const {
    std::vector<PointM> out(n);
    PointM cur = initial(), step = index_to_point(step_size);
    for (size_t i = 0; i < n; ++i) { out[i] = cur; cur = padd(cur, step); }
    return out;
  }
};
inline Coset coset_new(uint32_t initial_index, uint32_t log_size) { return {initial_index, subgroup_gen(log_size), log_size}; }
inline Coset coset_odds(uint32_t log_size) { return coset_new(subgroup_gen(log_size + 1), log_size); }
inline Coset coset_half_odds(uint32_t log_size) { return coset_new(subgroup_gen(log_size + 2), log_size); }

// CanonicCoset(n).circleDomain() = CircleDomain(halfOdds(n-1))  (poly/circle/canonic.zig:12-27)
struct CircleDomain {
  Coset half;
  uint32_t log_size() const { return half.log_size + 1; }
  size_t size() const { return (size_t)1 << log_size(); }
  uint32_t index_at(size_t i) const {
    size_t hs = half.size();
    if (i < hs) return half.index_at(i);
    return (0u - half.index_at(i - hs)) & ORDER_MASK;
  }
  PointM at(size_t i) const { return index_to_point(index_at(i)); }
};
inline CircleDomain canonic_domain(uint32_t log_size) { return {coset_half_odds(log_size - 1)}; }

inline size_t bit_reverse_index(size_t i, uint32_t log_size) {
  if (log_size == 0) return i;
  uint64_t v = i, r = 0;
  for (uint32_t k = 0; k < log_size; ++k) { r = (r << 1) | (v & 1); v >>= 1; }
  return (size_t)r;
}
template <class T>
void bit_reverse(std::vector<T>& v) {
  size_t n = v.size();
  uint32_t log_n = 0; while (((size_t)1 << log_n) < n) ++log_n;
  for (size_t i = 0; i < n; ++i) { size_t j = bit_reverse_index(i, log_n); if (j > i) std::swap(v[i], v[j]); }
}

// ---------------------------------------------------------------------------
// Twiddles: per line layer j the x-coordinates of the first half of the j-times
// doubled half coset, bit-reversed within the layer.
// src/prover/poly/twiddles.zig:37-91.
// ---------------------------------------------------------------------------
struct Twiddles {
  uint32_t line_log;  // log size of the half coset
  std::vector<std::vector<uint32_t>> layer, ilayer;  // layer[j] has 2^(line_log-1-j) entries
};
Twiddles make_twiddles(const Coset& half) {
  Twiddles t;
  t.line_log = half.log_size;
  Coset c = half;
  for (uint32_t j = 0; j < half.log_size; ++j) {
    size_t len = c.size() / 2;
    std::vector<PointM> pts = c.points(len);
    std::vector<uint32_t> xs(len), ixs(len);
    for (size_t i = 0; i < len; ++i) xs[i] = pts[i].x;
    bit_reverse(xs);
    for (size_t i = 0; i < len; ++i) ixs[i] = minv(xs[i]);
    t.layer.push_back(std::move(xs));
    t.ilayer.push_back(std::move(ixs));
    c = c.dbl();
  }
  return t;
}

inline void butterfly(uint32_t& v0, uint32_t& v1, uint32_t t) {
  uint32_t m = mmul(v1, t);
  v1 = msub(v0, m);
  v0 = madd(v0, m);
}
inline void ibutterfly(uint32_t& v0, uint32_t& v1, uint32_t it) {
  uint32_t a = v0;
  v0 = madd(a, v1);
  v1 = mmul(msub(a, v1), it);
}
inline void qibutterfly(QM31& v0, QM31& v1, uint32_t it) {
  QM31 a = v0;
  v0 = qadd(a, v1);
  v1 = qmulm(qsub(a, v1), it);
}

// Circle FFT over one buffer in bit-reversed circle-domain order.
// src/prover/poly/circle/transforms.zig:132-248 (evaluate), 249-362 (interpolate);
// first-layer twiddle pattern [y, -y, -x, x] at :233-247 / :309-321.
void circle_evaluate(uint32_t* v, const CircleDomain& dom, const Twiddles& tw) {
  uint32_t L = dom.half.log_size;
  if (L == 0) { PointM i0 = dom.half.initial(); butterfly(v[0], v[1], i0.y); return; }
  if (L == 1) {
    PointM i0 = dom.half.initial();
    butterfly(v[0], v[2], i0.x); butterfly(v[1], v[3], i0.x);
    butterfly(v[0], v[1], i0.y); butterfly(v[2], v[3], mneg(i0.y));
    return;
  }
  for (int j = (int)L - 1; j >= 0; --j) {
    const std::vector<uint32_t>& t = tw.layer[j];
    size_t half_block = (size_t)1 << (j + 1);
    for (size_t h = 0; h < t.size(); ++h) {
      size_t base = h << (j + 2);
      for (size_t l = 0; l < half_block; ++l) butterfly(v[base + l], v[base + l + half_block], t[h]);
    }
  }
  const std::vector<uint32_t>& t0 = tw.layer[0];
  for (size_t m = 0; 2 * m + 1 < t0.size(); ++m) {
    uint32_t x = t0[2 * m], y = t0[2 * m + 1];
    size_t h = 4 * m;
    butterfly(v[2 * h], v[2 * h + 1], y);
    butterfly(v[2 * h + 2], v[2 * h + 3], mneg(y));
    butterfly(v[2 * h + 4], v[2 * h + 5], mneg(x));
    butterfly(v[2 * h + 6], v[2 * h + 7], x);
  }
}

void circle_interpolate(uint32_t* v, const CircleDomain& dom, const Twiddles& tw) {
  uint32_t L = dom.half.log_size;
  size_t n = dom.size();
  if (L == 0) {
    PointM i0 = dom.half.initial();
    uint32_t yn_inv = minv(mmul(i0.y, 2));
    uint32_t y_inv = mmul(yn_inv, 2), n_inv = mmul(yn_inv, i0.y);
    ibutterfly(v[0], v[1], y_inv);
    v[0] = mmul(v[0], n_inv); v[1] = mmul(v[1], n_inv);
    return;
  }
  if (L == 1) {
    PointM i0 = dom.half.initial();
    uint32_t xyn_inv = minv(mmul(mmul(i0.x, i0.y), 4));
    uint32_t x_inv = mmul(mmul(xyn_inv, i0.y), 4), y_inv = mmul(mmul(xyn_inv, i0.x), 4);
    uint32_t n_inv = mmul(mmul(xyn_inv, i0.x), i0.y);
    ibutterfly(v[0], v[1], y_inv); ibutterfly(v[2], v[3], mneg(y_inv));
    ibutterfly(v[0], v[2], x_inv); ibutterfly(v[1], v[3], x_inv);
    for (int k = 0; k < 4; ++k) v[k] = mmul(v[k], n_inv);
    return;
  }
  const std::vector<uint32_t>& t0 = tw.ilayer[0];
  for (size_t m = 0; 2 * m + 1 < t0.size(); ++m) {
    uint32_t x = t0[2 * m], y = t0[2 * m + 1];
    size_t h = 4 * m;
    ibutterfly(v[2 * h], v[2 * h + 1], y);
    ibutterfly(v[2 * h + 2], v[2 * h + 3], mneg(y));
    ibutterfly(v[2 * h + 4], v[2 * h + 5], mneg(x));
    ibutterfly(v[2 * h + 6], v[2 * h + 7], x);
  }
  for (uint32_t j = 0; j < L; ++j) {
    const std::vector<uint32_t>& t = tw.ilayer[j];
    size_t half_block = (size_t)1 << (j + 1);
    for (size_t h = 0; h < t.size(); ++h) {
      size_t base = h << (j + 2);
      for (size_t l = 0; l < half_block; ++l) ibutterfly(v[base + l], v[base + l + half_block], t[h]);
    }
  }
  uint32_t n_inv = minv((uint32_t)(n % P));
  for (size_t i = 0; i < n; ++i) v[i] = mmul(v[i], n_inv);
}

// Coefficients (2^log_size) -> evaluations on CanonicCoset(log_size+blowup) (zero-extended).
// src/prover/pcs/columns/circle_transforms.zig (extend), transforms.zig:132-147.
void circle_extend(const uint32_t* coeffs, uint32_t log_size, uint32_t log_blowup, uint32_t* out,
                   const Twiddles& tw_ext) {
  size_t n = (size_t)1 << log_size, m = n << log_blowup;
  std::memcpy(out, coeffs, n * 4);
  std::memset(out + n, 0, (m - n) * 4);
  circle_evaluate(out, canonic_domain(log_size + log_blowup), tw_ext);
}

// ---------------------------------------------------------------------------
// Blake2s-256 (RFC 7693), unkeyed, 32-byte digest. Used by the channel
// (src/core/channel/blake2s.zig) and the lifted Merkle hasher
// (src/core/vcs_lifted/blake2_merkle.zig).
// ---------------------------------------------------------------------------
const uint32_t B2S_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                            0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
const uint8_t B2S_SIGMA[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
    {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4},
    {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13},
    {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11},
    {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5},
    {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

void b2s_compress(uint32_t h[8], const uint32_t m[16], uint64_t t, bool last) {
  uint32_t v[16];
  for (int i = 0; i < 8; ++i) { v[i] = h[i]; v[i + 8] = B2S_IV[i]; }
  v[12] ^= (uint32_t)t; v[13] ^= (uint32_t)(t >> 32);
  if (last) v[14] = ~v[14];
  auto G = [&](int a, int b, int c, int d, uint32_t x, uint32_t y) {
    v[a] = v[a] + v[b] + x; v[d] = rotr(v[d] ^ v[a], 16);
    v[c] = v[c] + v[d];     v[b] = rotr(v[b] ^ v[c], 12);
    v[a] = v[a] + v[b] + y; v[d] = rotr(v[d] ^ v[a], 8);
    v[c] = v[c] + v[d];     v[b] = rotr(v[b] ^ v[c], 7);
  };
  for (int r = 0; r < 10; ++r) {
    const uint8_t* s = B2S_SIGMA[r];
    G(0, 4, 8, 12, m[s[0]], m[s[1]]);   G(1, 5, 9, 13, m[s[2]], m[s[3]]);
    G(2, 6, 10, 14, m[s[4]], m[s[5]]);  G(3, 7, 11, 15, m[s[6]], m[s[7]]);
    G(0, 5, 10, 15, m[s[8]], m[s[9]]);  G(1, 6, 11, 12, m[s[10]], m[s[11]]);
    G(2, 7, 8, 13, m[s[12]], m[s[13]]); G(3, 4, 9, 14, m[s[14]], m[s[15]]);
  }
  for (int i = 0; i < 8; ++i) h[i] ^= v[i] ^ v[i + 8];
}

struct Blake2s {
  uint32_t h[8];
  uint8_t buf[64];
  size_t buflen = 0;
  uint64_t t = 0;
  Blake2s() { std::memcpy(h, B2S_IV, 32); h[0] ^= 0x01010020u; }
  void block(bool last) {
    uint32_t m[16];
    for (int i = 0; i < 16; ++i)
      m[i] = (uint32_t)buf[4 * i] | ((uint32_t)buf[4 * i + 1] << 8) | ((uint32_t)buf[4 * i + 2] << 16) |
             ((uint32_t)buf[4 * i + 3] << 24);
    b2s_compress(h, m, t, last);
  }
  void update(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    while (len > 0) {
      if (buflen == 64) { t += 64; block(false); buflen = 0; }
      size_t take = std::min(len, 64 - buflen);
      std::memcpy(buf + buflen, p, take);
      buflen += take; p += take; len -= take;
    }
  }
  void finalize(uint8_t out[32]) {
    t += buflen;
    std::memset(buf + buflen, 0, 64 - buflen);
    block(true);
    for (int i = 0; i < 8; ++i) { out[4 * i] = h[i]; out[4 * i + 1] = h[i] >> 8; out[4 * i + 2] = h[i] >> 16; out[4 * i + 3] = h[i] >> 24; }
  }
};

using Hash = std::array<uint8_t, 32>;
Hash b2s(const void* data, size_t len) { Blake2s s; s.update(data, len); Hash o; s.finalize(o.data()); return o; }

// "leaf"/"node" 64-byte domain prefixes (blake2_merkle.zig:9-10, 258-262).
struct Prefixes {
  uint8_t leaf[64], node[64];
  Prefixes() { std::memset(leaf, 0, 64); std::memset(node, 0, 64); std::memcpy(leaf, "leaf", 4); std::memcpy(node, "node", 4); }
};
const Prefixes& prefixes() { static Prefixes p; return p; }

Hash hash_node(const Hash& l, const Hash& r) {
  Blake2s s; s.update(prefixes().node, 64); s.update(l.data(), 32); s.update(r.data(), 32);
  Hash o; s.finalize(o.data()); return o;
}

// ---------------------------------------------------------------------------
// Blake2s channel. src/core/channel/blake2s.zig:33-280.
// ---------------------------------------------------------------------------
struct Channel {
  Hash digest{};
  uint32_t n_draws = 0;
  void update(const Hash& d) { digest = d; n_draws = 0; }
  void mix_felts(const std::vector<QM31>& f) {
    Blake2s s; s.update(digest.data(), 32);
    for (const QM31& q : f) { uint32_t w[4]; qstore(q, w); s.update(w, 16); }
    Hash o; s.finalize(o.data()); update(o);
  }
  void mix_u32s(const std::vector<uint32_t>& d) {
    Blake2s s; s.update(digest.data(), 32);
    if (!d.empty()) s.update(d.data(), d.size() * 4);
    Hash o; s.finalize(o.data()); update(o);
  }
  void mix_u64(uint64_t v) { mix_u32s({(uint32_t)v, (uint32_t)(v >> 32)}); }
  void mix_root(const Hash& root) {  // blake2_merkle.zig:236-247
    Blake2s s; s.update(digest.data(), 32); s.update(root.data(), 32);
    Hash o; s.finalize(o.data()); update(o);
  }
  std::array<uint32_t, 8> draw_u32s() {
    uint8_t in[37];
    std::memcpy(in, digest.data(), 32);
    uint32_t c = n_draws;
    std::memcpy(in + 32, &c, 4);
    in[36] = 0;
    n_draws += 1;
    Hash h = b2s(in, 37);
    std::array<uint32_t, 8> out;
    std::memcpy(out.data(), h.data(), 32);
    return out;
  }
  std::array<uint32_t, 8> draw_base_felts() {
    for (;;) {
      std::array<uint32_t, 8> w = draw_u32s();
      bool ok = true;
      for (uint32_t x : w) if (x >= 2 * P) { ok = false; break; }
      if (!ok) continue;
      for (uint32_t& x : w) x = mreduce64(x);
      return w;
    }
  }
  QM31 draw_secure_felt() { auto f = draw_base_felts(); return qfrom(f[0], f[1], f[2], f[3]); }
};

// PoW: H(H(LE32 0x12345678 || 0^12 || digest || LE32 bits) || LE64 nonce), trailing zeros of the
// first 16 bytes, lowest valid nonce. src/core/channel/blake2s.zig:135-240, 289-300.
Hash pow_prefix(const Hash& digest, uint32_t n_bits) {
  Blake2s s;
  uint32_t pre = 0x12345678u; s.update(&pre, 4);
  uint8_t z[12] = {0}; s.update(z, 12);
  s.update(digest.data(), 32);
  s.update(&n_bits, 4);
  Hash o; s.finalize(o.data()); return o;
}
uint32_t trailing_zero_bits16(const uint8_t* b) {
  uint32_t c = 0;
  for (int i = 0; i < 16; ++i) { if (b[i] == 0) { c += 8; continue; } c += __builtin_ctz(b[i]); break; }
  return c;
}
bool pow_check(const Hash& prefix, uint64_t nonce, uint32_t n_bits) {
  Blake2s s; s.update(prefix.data(), 32); s.update(&nonce, 8);
  Hash o; s.finalize(o.data());
  return trailing_zero_bits16(o.data()) >= n_bits;
}
uint64_t pow_grind(const Hash& digest, uint32_t n_bits, int n_threads) {
  if (n_bits == 0) return 0;
  Hash prefix = pow_prefix(digest, n_bits);
  std::atomic<uint64_t> found(~0ull);
#ifdef _OPENMP
  if (n_threads < 1) n_threads = omp_get_max_threads();
#else
  n_threads = 1;
#endif
#pragma omp parallel num_threads(n_threads)
  {
    int tid = 0, nt = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num(); nt = omp_get_num_threads();
#endif
    for (uint64_t nonce = tid; nonce < found.load(std::memory_order_relaxed); nonce += nt) {
      if (pow_check(prefix, nonce, n_bits)) {
        uint64_t cur = found.load();
        while (nonce < cur && !found.compare_exchange_weak(cur, nonce)) {}
        break;
      }
    }
  }
  return found.load();
}

// ---------------------------------------------------------------------------
// Lifted Blake2s Merkle tree. Leaves hash "leaf"-prefix || LE32 of every column's
// value at the lifted index, columns stably sorted by log size ascending.
// src/prover/vcs_lifted/leaves.zig:24-115, layers.zig:99-194, decommit.zig:56-240,
// src/core/vcs_lifted/verifier.zig.
// ---------------------------------------------------------------------------
struct ColRef { const uint32_t* data; uint32_t log_size; };

struct MerkleTree {
  uint32_t max_log = 0;
  std::vector<std::vector<Hash>> layers;  // layers[k] has 2^k nodes; layers[max_log] = leaves
  std::vector<ColRef> sorted;             // columns in leaf order
  Hash root() const { return layers[0][0]; }
};

inline size_t lifted_index(size_t pos, uint32_t max_log, uint32_t log_size) {
  uint32_t shift = max_log - log_size;
  return ((pos >> (shift + 1)) << 1) + (pos & 1);
}

MerkleTree merkle_commit(const std::vector<ColRef>& cols) {
  MerkleTree t;
  for (const ColRef& c : cols) t.max_log = std::max(t.max_log, c.log_size);
  t.sorted = cols;
  std::stable_sort(t.sorted.begin(), t.sorted.end(), [](const ColRef& a, const ColRef& b) { return a.log_size < b.log_size; });
  t.layers.resize(t.max_log + 1);
  size_t n = (size_t)1 << t.max_log;
  std::vector<Hash>& leaves = t.layers[t.max_log];
  leaves.resize(n);
#pragma omp parallel for schedule(static)
  for (long long pos = 0; pos < (long long)n; ++pos) {
    Blake2s s;
    s.update(prefixes().leaf, 64);
    for (const ColRef& c : t.sorted) {
      uint32_t v = c.data[lifted_index(pos, t.max_log, c.log_size)];
      s.update(&v, 4);
    }
    s.finalize(leaves[pos].data());
  }
  for (int k = (int)t.max_log - 1; k >= 0; --k) {
    std::vector<Hash>& cur = t.layers[k];
    const std::vector<Hash>& prev = t.layers[k + 1];
    cur.resize((size_t)1 << k);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)cur.size(); ++i) cur[i] = hash_node(prev[2 * i], prev[2 * i + 1]);
  }
  return t;
}

struct Decommitment {
  std::vector<std::vector<uint32_t>> queried;  // [column in original order][query]
  std::vector<Hash> witness;
};

Decommitment merkle_decommit(const MerkleTree& t, const std::vector<ColRef>& cols_original_order,
                             const std::vector<size_t>& positions) {
  Decommitment d;
  for (const ColRef& c : cols_original_order) {
    std::vector<uint32_t> q(positions.size());
    for (size_t j = 0; j < positions.size(); ++j) q[j] = c.data[lifted_index(positions[j], t.max_log, c.log_size)];
    d.queried.push_back(std::move(q));
  }
  // The witness covers the sorted unique positions, the order in which the reference verifier
  // walks them (src/core/vcs_lifted/verifier.zig:109-138). The reference prover walks the positions
  // as given, dropping only adjacent repeats (src/prover/vcs_lifted/decommit.zig:166-176): the same
  // witness for sorted positions (every trace tree and FRI layer), but not for the preprocessed
  // positions of a tree smaller than the lifting domain, which preparePreprocessedQueryPositions can
  // leave out of order (src/core/pcs/utils.zig:292-314) and which only a proof the verifier accepts
  // may carry.
  std::vector<size_t> prev(positions);
  std::sort(prev.begin(), prev.end());
  prev.erase(std::unique(prev.begin(), prev.end()), prev.end());
  for (int layer = (int)t.max_log - 1; layer >= 0; --layer) {
    const std::vector<Hash>& child = t.layers[layer + 1];
    std::vector<size_t> cur;
    size_t q = 0;
    while (q < prev.size()) {
      size_t first = prev[q];
      bool has_sib = q + 1 < prev.size() && (first ^ 1) == prev[q + 1];
      if (!has_sib) d.witness.push_back(child[first ^ 1]);
      cur.push_back(first >> 1);
      q += has_sib ? 2 : 1;
    }
    prev.swap(cur);
  }
  return d;
}

// ---------------------------------------------------------------------------
// Circle polynomial evaluation at a QM31 point: coefficients in bit-reversed
// basis order, folding factors [pi^{L-2}(x), ..., x, y]
// (src/prover/poly/circle/poly.zig:62-230, src/core/poly/utils.zig fold).
// ---------------------------------------------------------------------------
QM31 eval_at_point(const uint32_t* coeffs, uint32_t log_size, PointQ p) {
  if (log_size == 0) return qbase(coeffs[0]);
  std::vector<QM31> mappings;  // mappings[0] multiplies the top index bit
  mappings.push_back(p.y);
  QM31 x = p.x;
  for (uint32_t i = 1; i < log_size; ++i) { mappings.push_back(x); x = qdouble_x(x); }
  std::reverse(mappings.begin(), mappings.end());
  // fold(values, factors): lhs + rhs * factor[0] recursively; done bottom-up.
  size_t n = (size_t)1 << log_size;
  std::vector<QM31> cur(n / 2);
  const QM31& f_last = mappings[log_size - 1];
  for (size_t i = 0; i < n / 2; ++i) cur[i] = qadd(qbase(coeffs[2 * i]), qmulm(f_last, coeffs[2 * i + 1]));
  for (int k = (int)log_size - 2; k >= 0; --k) {
    size_t m = cur.size() / 2;
    for (size_t i = 0; i < m; ++i) cur[i] = qadd(cur[2 * i], qmul(cur[2 * i + 1], mappings[k]));
    cur.resize(m);
  }
  return cur[0];
}

// randomSecureFieldPoint (src/core/circle.zig:159-167).
PointQ random_secure_point(Channel& ch) {
  QM31 t = ch.draw_secure_felt();
  QM31 t2 = qsq(t);
  QM31 inv = qinv(qadd(t2, qone()));
  return {qmul(qsub(qone(), t2), inv), qmul(qadd(t, t), inv)};
}

// cosetVanishing (src/core/constraints.zig:17-27), base and secure forms.
uint32_t coset_vanishing_m(const Coset& c, PointM p) {
  PointM q = padd(padd(p, pconj(c.initial())), c.half_step());
  uint32_t x = q.x;
  for (uint32_t i = 1; i < c.log_size; ++i) x = double_x(x);
  return x;
}
QM31 coset_vanishing_q(const Coset& c, PointQ p) {
  PointQ q = qpadd(qpadd(p, qpneg(qpfromm(c.initial()))), qpfromm(c.half_step()));
  QM31 x = q.x;
  for (uint32_t i = 1; i < c.log_size; ++i) x = qdouble_x(x);
  return x;
}

// ---------------------------------------------------------------------------
// Wide-Fibonacci trace. Storage position s holds logical row
// circleDomainIndexToCosetIndex(bitReverse(s)) (src/examples/wide_fibonacci/trace.zig:159-162).
// ---------------------------------------------------------------------------
inline size_t logical_row(uint32_t log_n, size_t s) {
  size_t ci = bit_reverse_index(s, log_n);
  size_t n = (size_t)1 << log_n;
  return ci < n / 2 ? ci * 2 : (n - 1 - ci) * 2 + 1;
}
inline uint64_t splitmix64(uint64_t& state) {
  state += 0x9E3779B97F4A7C15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Seeded uniform value in [0, p-1) for (seed, column, logical row): SplitMix64 stream keyed by
// seed ^ (0xD1B54A32D192ED03 * (2*row + column + 1)), top 31 bits, rejection of values >= p-1.
inline uint32_t seeded_value(uint64_t seed, uint32_t column, uint64_t row) {
  uint64_t state = seed ^ (0xD1B54A32D192ED03ull * (2 * row + column + 1));
  for (;;) {
    uint32_t v = (uint32_t)(splitmix64(state) >> 33);
    if (v < P - 1) return v;
  }
}
void gen_trace(uint32_t log_n, uint32_t W, int kind, uint64_t seed, uint32_t* out) {
  size_t n = (size_t)1 << log_n;
#pragma omp parallel for schedule(static)
  for (long long s = 0; s < (long long)n; ++s) {
    size_t row = logical_row(log_n, s);
    uint32_t a, b;
    if (kind == 0) { a = 1; b = (uint32_t)(row % P); }
    else { a = seeded_value(seed, 0, row); b = seeded_value(seed, 1, row); }
    out[s] = a; out[n + s] = b;
    for (uint32_t k = 2; k < W; ++k) {
      uint32_t c = madd(mmul(a, a), mmul(b, b));
      out[(size_t)k * n + s] = c;
      a = b; b = c;
    }
  }
}

// ---------------------------------------------------------------------------
// JSON proof wire (src/interop/proof_wire.zig:19-77): compact std.json, fields
// in ProofWire order, hashes as arrays of 32 numbers, QM31 as [4]u32.
// ---------------------------------------------------------------------------
struct Json {
  std::string s;
  void u(uint64_t v) { s += std::to_string(v); }
  void hash(const Hash& h) { s += '['; for (int i = 0; i < 32; ++i) { if (i) s += ','; u(h[i]); } s += ']'; }
  void qm(QM31 q) { uint32_t w[4]; qstore(q, w); s += '['; for (int i = 0; i < 4; ++i) { if (i) s += ','; u(w[i]); } s += ']'; }
  void hashes(const std::vector<Hash>& hs) { s += '['; for (size_t i = 0; i < hs.size(); ++i) { if (i) s += ','; hash(hs[i]); } s += ']'; }
  void qms(const std::vector<QM31>& qs) { s += '['; for (size_t i = 0; i < qs.size(); ++i) { if (i) s += ','; qm(qs[i]); } s += ']'; }
};

struct FriLayerProof { std::vector<QM31> witness; std::vector<Hash> hash_witness; Hash commitment; };

// FRI decommitment of one layer: full subsets of size 2^fold_step around each query, witness =
// subset values that are not queries (src/prover/fri.zig:624-700).
FriLayerProof fri_decommit_layer(const MerkleTree& tree, const std::vector<uint32_t> coords[4],
                                 const std::vector<size_t>& queries) {
  FriLayerProof out;
  std::vector<size_t> positions;
  size_t q = 0;
  while (q < queries.size()) {
    size_t key = queries[q] >> 1;
    size_t end = q + 1;
    while (end < queries.size() && (queries[end] >> 1) == key) ++end;
    size_t at = q;
    for (size_t pos = key << 1; pos < (key << 1) + 2; ++pos) {
      positions.push_back(pos);
      if (at < end && queries[at] == pos) { ++at; continue; }
      out.witness.push_back(qfrom(coords[0][pos], coords[1][pos], coords[2][pos], coords[3][pos]));
    }
    q = end;
  }
  std::vector<ColRef> cols;
  uint32_t lg = tree.max_log;
  for (int c = 0; c < 4; ++c) cols.push_back({coords[c].data(), lg});
  out.hash_witness = merkle_decommit(tree, cols, positions).witness;
  out.commitment = tree.root();
  return out;
}

std::vector<size_t> fold_queries(const std::vector<size_t>& q) {
  std::vector<size_t> out;
  for (size_t p : q) { size_t f = p >> 1; if (out.empty() || out.back() != f) out.push_back(f); }
  return out;
}

// DEEP quotient batches (src/core/pcs/quotients/samples.zig:163-300): samples grouped by point in
// order of first appearance, each sample a committed column (its LDE at its own log size, read at
// the lifted index of the lifting domain) with its sampled value and random-coefficient power.
struct QuotientSample { const uint32_t* col; uint32_t log_size; QM31 value; QM31 rp; };
struct QuotientBatch { PointQ point; std::vector<QuotientSample> samples; };

QuotientBatch& batch_for(std::vector<QuotientBatch>& batches, const PointQ& p) {
  for (QuotientBatch& b : batches)
    if (qeq(b.point.x, p.x) && qeq(b.point.y, p.y)) return b;
  batches.push_back({p, {}});
  return batches.back();
}

// Row values of the DEEP quotient on CanonicCoset(lifting), bit-reversed
// (src/core/pcs/quotients/row_evaluation.zig:24-140,402-521; line coefficients
// src/core/constraints.zig:87-97): per batch at point P, with a = conj(v) - v, c = conj(Py) - Py,
// b = v c - a Py, the row (x, y) adds (sum_i rp_i c v_i(x, y) - sum_i rp_i (a y + b)) divided by
// (Re Px - x) Im Py - (Re Py - y) Im Px.
void quotient_columns(const std::vector<QuotientBatch>& batches, uint32_t lifting, std::vector<uint32_t> out[4]) {
  const size_t NL = (size_t)1 << lifting;
  struct Lc { const uint32_t* col; uint32_t log_size; QM31 c; };
  struct Prepared { CM31 prx, pry, pix, piy; QM31 sum_a, sum_b; std::vector<Lc> lc; };
  std::vector<Prepared> prep;
  for (const QuotientBatch& b : batches) {
    Prepared p;
    p.prx = b.point.x.c0; p.pry = b.point.y.c0; p.pix = b.point.x.c1; p.piy = b.point.y.c1;
    p.sum_a = qzero(); p.sum_b = qzero();
    QM31 cy = qsub(qconj(b.point.y), b.point.y);
    for (const QuotientSample& q : b.samples) {
      QM31 a = qsub(qconj(q.value), q.value);
      QM31 bb = qsub(qmul(q.value, cy), qmul(a, b.point.y));
      p.sum_a = qadd(p.sum_a, qmul(q.rp, a));
      p.sum_b = qadd(p.sum_b, qmul(q.rp, bb));
      p.lc.push_back({q.col, q.log_size, qmul(q.rp, cy)});
    }
    prep.push_back(std::move(p));
  }
  for (int k = 0; k < 4; ++k) out[k].assign(NL, 0);
  CircleDomain qdom = canonic_domain(lifting);
#pragma omp parallel for schedule(static)
  for (long long row = 0; row < (long long)NL; ++row) {
    PointM dp = qdom.at(bit_reverse_index(row, lifting));
    QM31 acc = qzero();
    for (const Prepared& p : prep) {
      QM31 num = qzero();
      for (const Lc& l : p.lc) num = qadd(num, qmulm(l.c, l.col[lifted_index(row, lifting, l.log_size)]));
      num = qsub(num, qadd(qmulm(p.sum_a, dp.y), p.sum_b));
      CM31 den = csub(cmul(csub(p.prx, CM31{dp.x, 0}), p.piy), cmul(csub(p.pry, CM31{dp.y, 0}), p.pix));
      acc = qadd(acc, qmulc(num, cinv(den)));
    }
    uint32_t w[4]; qstore(acc, w);
    for (int k = 0; k < 4; ++k) out[k][row] = w[k];
  }
}

// FRI commitment over the quotient column, the last layer, the proof of work and the queries
// (src/prover/fri.zig:163-620, verifier order src/core/fri.zig:54-145; src/prover/pcs/scheme.zig:
// 731-745; src/core/queries.zig:8-60).
// Wall time of the last proof's proof-of-work grind (reported beside the CPU baseline).
double& last_pow_seconds() { static thread_local double s = 0; return s; }

struct FriInner { MerkleTree tree; std::vector<uint32_t> coords[4]; };
struct FriRun {
  MerkleTree first_tree;
  std::vector<FriInner> inner;
  std::vector<QM31> last_coeffs;
  uint64_t nonce = 0;
  std::vector<size_t> queries;
  bool ok = true;  // false: the last layer exceeds its degree bound
};

FriRun fri_pow_queries(Channel& ch, std::vector<uint32_t> qcol[4], uint32_t lifting, const oracle_pcs_config& cfg,
                       int n_threads) {
  FriRun fr;
  const uint32_t B = cfg.log_blowup_factor;
  CircleDomain qdom = canonic_domain(lifting);
  std::vector<ColRef> fcols;
  for (int k = 0; k < 4; ++k) fcols.push_back({qcol[k].data(), lifting});
  fr.first_tree = merkle_commit(fcols);
  ch.mix_root(fr.first_tree.root());
  QM31 alpha = ch.draw_secure_felt();
  // fold_circle_into_line (src/core/fri/folding.zig:558-602).
  uint32_t line_log = lifting - 1;
  Coset line_coset = qdom.half;  // LineDomain(halfOdds(lifting-1))
  std::vector<uint32_t> cur[4];
  for (int k = 0; k < 4; ++k) cur[k].assign((size_t)1 << line_log, 0);
  {
    size_t m = (size_t)1 << line_log;
    std::vector<PointM> pts = qdom.half.points(m);
    std::vector<uint32_t> py(m);
    for (size_t i = 0; i < m; ++i) py[bit_reverse_index(i, line_log)] = pts[i].y;
    QM31 a2 = qsq(alpha);
    for (size_t i = 0; i < m; ++i) {
      QM31 f0 = qfrom(qcol[0][2 * i], qcol[1][2 * i], qcol[2][2 * i], qcol[3][2 * i]);
      QM31 f1 = qfrom(qcol[0][2 * i + 1], qcol[1][2 * i + 1], qcol[2][2 * i + 1], qcol[3][2 * i + 1]);
      qibutterfly(f0, f1, minv(py[i]));
      QM31 r = qadd(qmul(qzero(), a2), qadd(qmul(alpha, f1), f0));
      uint32_t w[4]; qstore(r, w);
      for (int k = 0; k < 4; ++k) cur[k][i] = w[k];
    }
  }
  const uint32_t last_log = cfg.log_last_layer_degree_bound + B;
  while (line_log > last_log) {
    FriInner L;
    for (int k = 0; k < 4; ++k) L.coords[k] = cur[k];
    std::vector<ColRef> lcols;
    for (int k = 0; k < 4; ++k) lcols.push_back({L.coords[k].data(), line_log});
    L.tree = merkle_commit(lcols);
    ch.mix_root(L.tree.root());
    QM31 a = ch.draw_secure_felt();
    // fold_line (src/core/fri/folding.zig:352-384).
    size_t m = (size_t)1 << (line_log - 1);
    std::vector<PointM> pts = line_coset.points(m);
    std::vector<uint32_t> xs(m);
    for (size_t i = 0; i < m; ++i) xs[bit_reverse_index(i, line_log - 1)] = pts[i].x;
    std::vector<uint32_t> nxt[4];
    for (int k = 0; k < 4; ++k) nxt[k].resize(m);
    for (size_t i = 0; i < m; ++i) {
      QM31 f0 = qfrom(cur[0][2 * i], cur[1][2 * i], cur[2][2 * i], cur[3][2 * i]);
      QM31 f1 = qfrom(cur[0][2 * i + 1], cur[1][2 * i + 1], cur[2][2 * i + 1], cur[3][2 * i + 1]);
      qibutterfly(f0, f1, minv(xs[i]));
      QM31 r = qadd(f0, qmul(a, f1));
      uint32_t w[4]; qstore(r, w);
      for (int k = 0; k < 4; ++k) nxt[k][i] = w[k];
    }
    for (int k = 0; k < 4; ++k) cur[k].swap(nxt[k]);
    fr.inner.push_back(std::move(L));
    line_coset = line_coset.dbl();
    line_log -= 1;
  }
  // Last layer: line IFFT (src/backend/line_evaluation.zig:97-145), degree check, truncate, mix.
  {
    size_t m = (size_t)1 << line_log;
    std::vector<QM31> v(m);
    for (size_t i = 0; i < m; ++i) v[i] = qfrom(cur[0][i], cur[1][i], cur[2][i], cur[3][i]);
    bit_reverse(v);
    Coset d = line_coset;
    while (d.size() > 1) {
      size_t chunk = d.size(), half = chunk / 2;
      std::vector<PointM> pts = d.points(half);
      for (size_t st = 0; st < m; st += chunk)
        for (size_t i = 0; i < half; ++i) qibutterfly(v[st + i], v[st + half + i], minv(pts[i].x));
      d = d.dbl();
    }
    uint32_t li = minv((uint32_t)(m % P));
    for (QM31& x : v) x = qmulm(x, li);
    bit_reverse(v);  // ordered coefficients
    size_t bound = (size_t)1 << cfg.log_last_layer_degree_bound;
    for (size_t i = bound; i < m; ++i)
      if (!qiszero(v[i])) { fr.ok = false; return fr; }  // InvalidLastLayerDegree
    fr.last_coeffs.assign(v.begin(), v.begin() + bound);
    bit_reverse(fr.last_coeffs);
    ch.mix_felts(fr.last_coeffs);
  }
  const auto t_pow = std::chrono::steady_clock::now();
  fr.nonce = pow_grind(ch.digest, cfg.pow_bits, n_threads);
  last_pow_seconds() = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_pow).count();
  ch.mix_u64(fr.nonce);
  uint32_t mask = (1u << lifting) - 1;
  while (fr.queries.size() < cfg.n_queries) {
    auto w = ch.draw_u32s();
    for (uint32_t x : w) { fr.queries.push_back(x & mask); if (fr.queries.size() == cfg.n_queries) break; }
  }
  std::sort(fr.queries.begin(), fr.queries.end());
  fr.queries.erase(std::unique(fr.queries.begin(), fr.queries.end()), fr.queries.end());
  return fr;
}

// Trace-tree decommitments and the FRI proof in wire order: "decommitments", "queried_values",
// "proof_of_work", "fri_proof" (src/interop/proof_wire.zig:19-77, src/prover/fri.zig:624-850).
void json_decommit_and_fri(Json& j, const std::vector<const Decommitment*>& ds, FriRun& fr,
                           std::vector<uint32_t> qcol[4]) {
  j.s += "\"decommitments\":[";
  for (size_t t = 0; t < ds.size(); ++t) { if (t) j.s += ','; j.s += "{\"hash_witness\":"; j.hashes(ds[t]->witness); j.s += '}'; }
  j.s += "],\"queried_values\":[";
  for (size_t t = 0; t < ds.size(); ++t) {
    if (t) j.s += ',';
    j.s += '[';
    for (size_t c = 0; c < ds[t]->queried.size(); ++c) {
      if (c) j.s += ',';
      j.s += '[';
      for (size_t q = 0; q < ds[t]->queried[c].size(); ++q) { if (q) j.s += ','; j.u(ds[t]->queried[c][q]); }
      j.s += ']';
    }
    j.s += ']';
  }
  j.s += "],\"proof_of_work\":"; j.u(fr.nonce);
  FriLayerProof first_proof = fri_decommit_layer(fr.first_tree, qcol, fr.queries);
  std::vector<FriLayerProof> inner_proofs;
  std::vector<size_t> lq = fold_queries(fr.queries);
  for (FriInner& L : fr.inner) { inner_proofs.push_back(fri_decommit_layer(L.tree, L.coords, lq)); lq = fold_queries(lq); }
  auto layer = [&](const FriLayerProof& L) {
    j.s += "{\"fri_witness\":"; j.qms(L.witness);
    j.s += ",\"decommitment\":{\"hash_witness\":"; j.hashes(L.hash_witness);
    j.s += "},\"commitment\":"; j.hash(L.commitment); j.s += '}';
  };
  j.s += ",\"fri_proof\":{\"first_layer\":"; layer(first_proof);
  j.s += ",\"inner_layers\":[";
  for (size_t i = 0; i < inner_proofs.size(); ++i) { if (i) j.s += ','; layer(inner_proofs[i]); }
  j.s += "],\"last_layer_poly\":"; j.qms(fr.last_coeffs);
  j.s += "}";
}

struct ProveParams {
  uint32_t log_n, W;
  oracle_pcs_config cfg;
  bool has_channel_seed;
  uint64_t channel_seed;
  int n_threads;
};

// The full wide-Fibonacci proof. Transaction order: src/examples/common/prover_transaction.zig:222-340;
// driver src/prover/prove.zig:209-389; PCS opening src/prover/pcs/scheme.zig:633-799;
// FRI src/prover/fri.zig:163-850.
std::string prove_wide_fib(const ProveParams& pp, const uint32_t* trace) {
  const uint32_t n = pp.log_n, W = pp.W, B = pp.cfg.log_blowup_factor;
  const size_t N = (size_t)1 << n;
  const uint32_t LDE = n + B;
  const size_t NL = (size_t)1 << LDE;

  Channel ch;
  // PcsConfig.mixInto (src/core/pcs/mod.zig:32-52), fold_step 1 and no lifting override.
  ch.mix_felts({qfrom(pp.cfg.pow_bits, pp.cfg.log_blowup_factor, pp.cfg.n_queries, pp.cfg.log_last_layer_degree_bound)});

  // Tree 0: preprocessed, empty for wide-Fibonacci.
  MerkleTree t0 = merkle_commit({});
  ch.mix_root(t0.root());

  // Tree 1: main trace -> interpolate on CanonicCoset(n), extend to CanonicCoset(n+B), commit.
  Twiddles tw_n = make_twiddles(canonic_domain(n).half);
  Twiddles tw_l = make_twiddles(canonic_domain(LDE).half);
  std::vector<std::vector<uint32_t>> coeffs(W, std::vector<uint32_t>(N)), lde(W, std::vector<uint32_t>(NL));
#pragma omp parallel for schedule(dynamic)
  for (long long c = 0; c < (long long)W; ++c) {
    std::memcpy(coeffs[c].data(), trace + (size_t)c * N, N * 4);
    circle_interpolate(coeffs[c].data(), canonic_domain(n), tw_n);
    circle_extend(coeffs[c].data(), n, B, lde[c].data(), tw_l);
  }
  std::vector<ColRef> main_cols;
  for (uint32_t c = 0; c < W; ++c) main_cols.push_back({lde[c].data(), LDE});
  MerkleTree t1 = merkle_commit(main_cols);
  ch.mix_root(t1.root());

  // Statement mix (src/examples/wide_fibonacci.zig:496-498), then the optional channel seed.
  ch.mix_u32s({n, W});
  if (pp.has_channel_seed) ch.mix_u64(pp.channel_seed);

  // Composition (src/examples/wide_fibonacci/component.zig:138-236) on CanonicCoset(n+1).
  QM31 random_coeff = ch.draw_secure_felt();
  const uint32_t CL = n + 1;
  const size_t NC = (size_t)1 << CL;
  const uint32_t n_cons = W - 2;
  std::vector<QM31> powers(n_cons);
  { QM31 cur = qone(); for (uint32_t i = 0; i < n_cons; ++i) { powers[i] = cur; cur = qmul(cur, random_coeff); } }
  std::vector<std::vector<uint32_t>> eval_cols;  // trace evaluated on CanonicCoset(n+1)
  const std::vector<std::vector<uint32_t>>* ev = &lde;
  Twiddles tw_c = make_twiddles(canonic_domain(CL).half);
  if (LDE != CL) {
    eval_cols.assign(W, std::vector<uint32_t>(NC));
#pragma omp parallel for schedule(dynamic)
    for (long long c = 0; c < (long long)W; ++c) circle_extend(coeffs[c].data(), n, 1, eval_cols[c].data(), tw_c);
    ev = &eval_cols;
  }
  CircleDomain cdom = canonic_domain(CL);
  Coset trace_coset = coset_odds(n);
  uint32_t den_inv[2] = {minv(coset_vanishing_m(trace_coset, cdom.at(0))), minv(coset_vanishing_m(trace_coset, cdom.at(1)))};
  std::vector<uint32_t> comp[4];
  for (int k = 0; k < 4; ++k) comp[k].resize(NC);
#pragma omp parallel for schedule(static)
  for (long long row = 0; row < (long long)NC; ++row) {
    uint32_t a = (*ev)[0][row], b = (*ev)[1][row];
    QM31 acc = qzero();
    for (uint32_t k = 0; k < n_cons; ++k) {
      uint32_t c = (*ev)[k + 2][row];
      uint32_t cons = msub(c, madd(mmul(a, a), mmul(b, b)));
      acc = qadd(acc, qmulm(powers[n_cons - 1 - k], cons));
      a = b; b = c;
    }
    acc = qmulm(acc, den_inv[row >> n]);
    uint32_t w[4]; qstore(acc, w);
    for (int k = 0; k < 4; ++k) comp[k][row] = w[k];
  }
  // Interpolate, split at mid into left/right (secure_poly.zig:77-105, poly.zig:302-317), commit.
  std::vector<std::vector<uint32_t>> comp_coeffs(8, std::vector<uint32_t>(N)), comp_lde(8, std::vector<uint32_t>(NL));
  for (int k = 0; k < 4; ++k) {
    std::vector<uint32_t> tmp = comp[k];
    circle_interpolate(tmp.data(), cdom, tw_c);
    std::memcpy(comp_coeffs[k].data(), tmp.data(), N * 4);
    std::memcpy(comp_coeffs[4 + k].data(), tmp.data() + N, N * 4);
  }
#pragma omp parallel for schedule(dynamic)
  for (int k = 0; k < 8; ++k) circle_extend(comp_coeffs[k].data(), n, B, comp_lde[k].data(), tw_l);
  std::vector<ColRef> comp_cols;
  for (int k = 0; k < 8; ++k) comp_cols.push_back({comp_lde[k].data(), LDE});
  MerkleTree t2 = merkle_commit(comp_cols);
  ch.mix_root(t2.root());

  // OODS point and sampled values (src/prover/prove.zig:329-364, pcs/sampled_values.zig).
  PointQ oods = random_secure_point(ch);
  const uint32_t lifting = LDE;  // max committed log size
  std::vector<QM31> sampled_main(W), sampled_comp(8);
#pragma omp parallel for schedule(dynamic)
  for (long long c = 0; c < (long long)W; ++c) sampled_main[c] = eval_at_point(coeffs[c].data(), n, oods);
  for (int k = 0; k < 8; ++k) sampled_comp[k] = eval_at_point(comp_coeffs[k].data(), n, oods);
  {
    std::vector<QM31> flat(sampled_main);
    flat.insert(flat.end(), sampled_comp.begin(), sampled_comp.end());
    ch.mix_felts(flat);
  }
  QM31 quot_coeff = ch.draw_secure_felt();

  // DEEP quotients on the lifting domain: one batch at the OODS point with all W+8 columns,
  // powers 1, a, a^2, ... in column order.
  std::vector<QuotientBatch> batches;
  {
    QM31 rp = qone();
    QuotientBatch& b = batch_for(batches, oods);
    for (uint32_t c = 0; c < W; ++c) { b.samples.push_back({lde[c].data(), LDE, sampled_main[c], rp}); rp = qmul(rp, quot_coeff); }
    for (int k = 0; k < 8; ++k) { b.samples.push_back({comp_lde[k].data(), LDE, sampled_comp[k], rp}); rp = qmul(rp, quot_coeff); }
  }
  std::vector<uint32_t> qcol[4];
  quotient_columns(batches, lifting, qcol);

  FriRun fr = fri_pow_queries(ch, qcol, lifting, pp.cfg, pp.n_threads);
  if (!fr.ok) return std::string();

  // Trace decommit (tree 0 has no columns and no positions).
  Decommitment d0 = merkle_decommit(t0, {}, {});
  Decommitment d1 = merkle_decommit(t1, main_cols, fr.queries);
  Decommitment d2 = merkle_decommit(t2, comp_cols, fr.queries);

  // Wire encoding.
  Json j;
  j.s += "{\"config\":{\"pow_bits\":"; j.u(pp.cfg.pow_bits);
  j.s += ",\"fri_config\":{\"log_blowup_factor\":"; j.u(B);
  j.s += ",\"log_last_layer_degree_bound\":"; j.u(pp.cfg.log_last_layer_degree_bound);
  j.s += ",\"n_queries\":"; j.u(pp.cfg.n_queries);
  j.s += ",\"fold_step\":1},\"lifting_log_size\":null},\"commitments\":[";
  j.hash(t0.root()); j.s += ','; j.hash(t1.root()); j.s += ','; j.hash(t2.root());
  j.s += "],\"sampled_values\":[[],[";
  for (uint32_t c = 0; c < W; ++c) { if (c) j.s += ','; j.s += '['; j.qm(sampled_main[c]); j.s += ']'; }
  j.s += "],[";
  for (int c = 0; c < 8; ++c) { if (c) j.s += ','; j.s += '['; j.qm(sampled_comp[c]); j.s += ']'; }
  j.s += "]],";
  json_decommit_and_fri(j, {&d0, &d1, &d2}, fr, qcol);
  j.s += "}";

  // Prover self-check of the composition OODS value (src/prover/prove.zig:366-386).
  {
    QM31 left = qzero(), right = qzero();
    const QM31 basis[4] = {qone(), qfrom(0, 1, 0, 0), qfrom(0, 0, 1, 0), qfrom(0, 0, 0, 1)};
    for (int k = 0; k < 4; ++k) { left = qadd(left, qmul(sampled_comp[k], basis[k])); right = qadd(right, qmul(sampled_comp[4 + k], basis[k])); }
    PointQ p = oods;
    for (uint32_t i = 0; i < CL - 2; ++i) p = qpdbl(p);
    QM31 comp_oods = qadd(left, qmul(p.x, right));
    QM31 dinv = qinv(coset_vanishing_q(trace_coset, oods));
    QM31 acc = qzero();
    QM31 a = sampled_main[0], b = sampled_main[1];
    for (uint32_t k = 2; k < W; ++k) {
      QM31 c = sampled_main[k];
      acc = qadd(qmul(acc, random_coeff), qmul(qsub(c, qadd(qsq(a), qsq(b))), dinv));
      a = b; b = c;
    }
    if (!qeq(acc, comp_oods)) return std::string("CONSTRAINTS_NOT_SATISFIED");
  }
  return j.s;
}

// ---------------------------------------------------------------------------
// LogUp XOR-lookup AIR (no reference AIR exists; it is built from the reference's pieces): a main
// component of 2^n lookups (a, b, c = a ^ b of w = t/2-bit operands) and a table component of 2^t
// rows (ta, tb, ta ^ tb with multiplicities m), each at its own size under the lifted PCS
// (columns of several sizes in one tree, src/prover/vcs_lifted/leaves.zig:104-115). The LogUp
// columns are the coset-order cumulative sums with the total/N shift of
// src/tests/metal/backend/commitment_test.zig:73-154 (oracle_logup_interaction below); the PCS
// samples, quotient batches and periodicity samples follow src/core/pcs/quotients/samples.zig:
// 163-300; the preprocessed tree is queried at src/core/pcs/utils.zig:292-314's positions; the FRI,
// proof-of-work, query and decommitment tail is the wide-Fibonacci one. Transcript:
//   config; tree 0 (ta, tb, tc); tree 1 (a, b, c, m); statement (n, t); [channel seed];
//   z, alpha; tree 2 (S_M, S_T: 4 coordinate columns each); claimed sums;
//   random_coeff; tree 3 (composition halves); OODS point; sampled values; quotient coefficient;
//   FRI; last layer; PoW; queries.
// Constraints (cyclic thanks to the shift), with d = a + alpha b + alpha^2 c - z at a row and
// S(x g^-1) the previous row at the component's size:
//   C_M = (S_M(x) - S_M(x g^-1) + claimed_M / 2^n) d_M(x) - 1
//   C_T = (S_T(x) - S_T(x g^-1) + claimed_T / 2^t) d_T(x) + m(x)
// composed as random_coeff C_M / Z_M + C_T / Z_T on CanonicCoset(L + 1), L = max(n, t), each
// component entering through the lifting map.
// ---------------------------------------------------------------------------
struct XorParams {
  uint32_t log_n, log_table;
  oracle_pcs_config cfg;
  uint64_t seed;
  bool has_channel_seed;
  uint64_t channel_seed;
  int n_threads;
};

// Storage position (bit-reversed circle order) of logical coset row k at size 2^log.
inline size_t storage_of_row(size_t k, uint32_t log) {
  size_t n = (size_t)1 << log;
  size_t ci = (k & 1) == 0 ? k / 2 : n - 1 - k / 2;
  return bit_reverse_index(ci, log);
}

std::string prove_logup_xor(const XorParams& xp) {
  const uint32_t n = xp.log_n, t = xp.log_table, B = xp.cfg.log_blowup_factor;
  const uint32_t L = std::max(n, t), LDE = L + B, CL = L + 1;
  const size_t NC = (size_t)1 << CL;
  const uint32_t w = t / 2, wmask = (1u << w) - 1;
  // Columns: tree 0 (0-2: ta, tb, tc), tree 1 (3-5: a, b, c; 6: m), tree 2 (7-10: S_M; 11-14: S_T).
  enum { TA = 0, A = 3, M = 6, SM = 7, ST = 11, NCOLS = 15 };
  struct Col { uint32_t log; std::vector<uint32_t> vals, coeffs, lde, evc; };
  std::vector<Col> col(NCOLS);
  for (int c = 0; c < NCOLS; ++c) col[c].log = (c < A || c == M || c >= ST) ? t : n;
  for (Col& c : col) c.vals.assign((size_t)1 << c.log, 0);

  // Trace: main rows are seeded by their logical (coset-order) row k: SplitMix64 of
  // seed ^ (0xD6E8FEB86659FD93 (k + 1)), a = low w bits, b = w bits from bit 8; table row k holds
  // ta = k >> w, tb = k & (2^w - 1) (the bitwise table layout of
  // src/frontends/riscv/air/preprocessed/bitwise.zig:17-35) and the count of main rows (ta, tb).
  std::vector<uint32_t> hist((size_t)1 << t, 0);
  for (size_t s = 0; s < ((size_t)1 << n); ++s) {
    uint64_t state = xp.seed ^ (0xD6E8FEB86659FD93ull * ((uint64_t)logical_row(n, s) + 1));
    uint64_t x = splitmix64(state);
    uint32_t a = (uint32_t)x & wmask, b = (uint32_t)(x >> 8) & wmask;
    col[A].vals[s] = a; col[A + 1].vals[s] = b; col[A + 2].vals[s] = a ^ b;
    ++hist[(a << w) | b];
  }
  for (size_t s = 0; s < ((size_t)1 << t); ++s) {
    size_t k = logical_row(t, s);
    uint32_t ta = (uint32_t)(k >> w), tb = (uint32_t)k & wmask;
    col[TA].vals[s] = ta; col[TA + 1].vals[s] = tb; col[TA + 2].vals[s] = ta ^ tb;
    col[M].vals[s] = hist[k];
  }

  std::vector<Twiddles> tw(LDE + 2);
  std::vector<bool> have(LDE + 2, false);
  auto twiddles = [&](uint32_t log) -> const Twiddles& {
    if (!have[log]) { tw[log] = make_twiddles(canonic_domain(log).half); have[log] = true; }
    return tw[log];
  };
  // Coefficients, own-size LDE (blowup B) and own-size evaluation on CanonicCoset(log + 1).
  auto prepare = [&](int first, int count) {
    for (int c = first; c < first + count; ++c) {
      Col& k = col[c];
      k.coeffs = k.vals;
      circle_interpolate(k.coeffs.data(), canonic_domain(k.log), twiddles(k.log));
      k.lde.resize((size_t)1 << (k.log + B));
      circle_extend(k.coeffs.data(), k.log, B, k.lde.data(), twiddles(k.log + B));
      if (B == 1) { k.evc = k.lde; continue; }
      k.evc.resize((size_t)2 << k.log);
      circle_extend(k.coeffs.data(), k.log, 1, k.evc.data(), twiddles(k.log + 1));
    }
  };
  auto refs = [&](int first, int count) {
    std::vector<ColRef> r;
    for (int c = first; c < first + count; ++c) r.push_back({col[c].lde.data(), col[c].log + B});
    return r;
  };

  Channel ch;
  ch.mix_felts({qfrom(xp.cfg.pow_bits, B, xp.cfg.n_queries, xp.cfg.log_last_layer_degree_bound)});
  prepare(TA, 3);
  MerkleTree t0 = merkle_commit(refs(TA, 3));
  ch.mix_root(t0.root());
  prepare(A, 4);
  MerkleTree t1 = merkle_commit(refs(A, 4));
  ch.mix_root(t1.root());
  ch.mix_u32s({n, t});
  if (xp.has_channel_seed) ch.mix_u64(xp.channel_seed);

  // Interaction: each component's LogUp column at its own size.
  const QM31 z = ch.draw_secure_felt();
  const QM31 alpha = ch.draw_secure_felt();
  const QM31 alpha2 = qsq(alpha);
  QM31 claimed[2];
  {
    uint32_t alphas[12];
    qstore(qone(), alphas); qstore(alpha, alphas + 4); qstore(alpha2, alphas + 8);
    uint32_t zw[4]; qstore(z, zw);
    for (int comp = 0; comp < 2; ++comp) {
      const int words0 = comp == 0 ? A : TA, out0 = comp == 0 ? SM : ST;
      const uint32_t log = col[words0].log;
      oracle_logup_use u{};
      u.n_words = 3;
      for (int j = 0; j < 3; ++j) u.words[j] = col[words0 + j].vals.data();
      u.multiplicity = comp == 0 ? nullptr : col[M].vals.data();
      u.negate = comp == 0 ? 0 : 1;
      std::vector<uint32_t> out((size_t)4 << log);
      uint32_t cw[4];
      int rc = oracle_logup_interaction(log, 1, &u, alphas, zw, 1, 1, out.data(), cw);
      if (rc != 0) return std::string("DIVISION_BY_ZERO");
      claimed[comp] = qload(cw);
      for (int k = 0; k < 4; ++k)
        col[out0 + k].vals.assign(out.begin() + ((size_t)k << log), out.begin() + ((size_t)(k + 1) << log));
    }
  }
  prepare(SM, 8);
  MerkleTree t2 = merkle_commit(refs(SM, 8));
  ch.mix_root(t2.root());
  ch.mix_felts({claimed[0], claimed[1]});

  // Composition on CanonicCoset(L + 1).
  const QM31 random_coeff = ch.draw_secure_felt();
  std::vector<uint32_t> comp[4];
  for (int k = 0; k < 4; ++k) comp[k].resize(NC);
  {
    const QM31 shift[2] = {qmulm(claimed[0], minv((uint32_t)(((size_t)1 << n) % P))),
                           qmulm(claimed[1], minv((uint32_t)(((size_t)1 << t) % P)))};
    uint32_t den[2][2];
    for (int c = 0; c < 2; ++c) {
      const uint32_t k = c == 0 ? n : t;
      CircleDomain cd = canonic_domain(k + 1);
      Coset trace = coset_odds(k);
      den[c][0] = minv(coset_vanishing_m(trace, cd.at(0)));
      den[c][1] = minv(coset_vanishing_m(trace, cd.at(1)));
    }
    auto at = [&](int c, size_t r) { return col[c].evc[lifted_index(r, CL, col[c].log + 1)]; };
    auto sec = [&](int c0, size_t r) { return qfrom(at(c0, r), at(c0 + 1, r), at(c0 + 2, r), at(c0 + 3, r)); };
#pragma omp parallel for schedule(static)
    for (long long rr = 0; rr < (long long)NC; ++rr) {
      const size_t r = (size_t)rr;
      const size_t rp = storage_of_row((logical_row(CL, r) + NC - 2) % NC, CL);  // x g_L^-1
      const QM31 d_main = qsub(qadd(qadd(qbase(at(A, r)), qmulm(alpha, at(A + 1, r))), qmulm(alpha2, at(A + 2, r))), z);
      const QM31 d_table =
          qsub(qadd(qadd(qbase(at(TA, r)), qmulm(alpha, at(TA + 1, r))), qmulm(alpha2, at(TA + 2, r))), z);
      const QM31 c_main = qsub(qmul(qadd(qsub(sec(SM, r), sec(SM, rp)), shift[0]), d_main), qone());
      const QM31 c_table = qadd(qmul(qadd(qsub(sec(ST, r), sec(ST, rp)), shift[1]), d_table), qbase(at(M, r)));
      const size_t h = r >> L;
      const QM31 q = qadd(qmulm(qmul(random_coeff, c_main), den[0][h]), qmulm(c_table, den[1][h]));
      uint32_t wq[4]; qstore(q, wq);
      for (int k = 0; k < 4; ++k) comp[k][r] = wq[k];
    }
  }
  // Interpolate, split at mid (left = first 2^L coefficients), extend, commit as tree 3.
  std::vector<std::vector<uint32_t>> comp_coeffs(8, std::vector<uint32_t>((size_t)1 << L)),
      comp_lde(8, std::vector<uint32_t>((size_t)1 << LDE));
  for (int k = 0; k < 4; ++k) {
    std::vector<uint32_t> tmp = comp[k];
    circle_interpolate(tmp.data(), canonic_domain(CL), twiddles(CL));
    std::memcpy(comp_coeffs[k].data(), tmp.data(), ((size_t)4) << L);
    std::memcpy(comp_coeffs[4 + k].data(), tmp.data() + ((size_t)1 << L), ((size_t)4) << L);
  }
  for (int k = 0; k < 8; ++k) circle_extend(comp_coeffs[k].data(), L, B, comp_lde[k].data(), twiddles(LDE));
  std::vector<ColRef> comp_cols;
  for (int k = 0; k < 8; ++k) comp_cols.push_back({comp_lde[k].data(), LDE});
  MerkleTree t3 = merkle_commit(comp_cols);
  ch.mix_root(t3.root());

  // Samples: every column at the OODS point P, tree 2 also at P - g_L (the previous row,
  // src/frontends/riscv/air/logup.zig:45-48); a column of 2^k rows at those points doubled L - k
  // times (its lifted polynomial).
  const PointQ oods = random_secure_point(ch);
  const PointQ prev = qpadd(oods, qpneg(qpfromm(index_to_point(subgroup_gen(L)))));
  auto doubled = [&](PointQ p, uint32_t k) { for (uint32_t i = k; i < L; ++i) p = qpdbl(p); return p; };
  std::vector<QM31> cur(NCOLS), before(NCOLS), sampled_comp(8);
  for (int c = 0; c < NCOLS; ++c) {
    cur[c] = eval_at_point(col[c].coeffs.data(), col[c].log, doubled(oods, col[c].log));
    if (c >= SM) before[c] = eval_at_point(col[c].coeffs.data(), col[c].log, doubled(prev, col[c].log));
  }
  for (int k = 0; k < 8; ++k) sampled_comp[k] = eval_at_point(comp_coeffs[k].data(), L, oods);
  {
    std::vector<QM31> flat;
    for (int c = 0; c < SM; ++c) flat.push_back(cur[c]);
    for (int c = SM; c < NCOLS; ++c) { flat.push_back(before[c]); flat.push_back(cur[c]); }
    flat.insert(flat.end(), sampled_comp.begin(), sampled_comp.end());
    ch.mix_felts(flat);
  }
  const QM31 quot_coeff = ch.draw_secure_felt();

  // Quotient batches: random powers over (tree, column, sample); a two-sample column first takes
  // its periodicity sample at its second point plus the lifting domain's generator doubled to the
  // column's committed log size; batches by point in order of first appearance.
  std::vector<QuotientBatch> batches;
  {
    QM31 rp = qone();
    auto next = [&]() { QM31 r = rp; rp = qmul(rp, quot_coeff); return r; };
    const PointM lifting_gen = index_to_point(subgroup_gen(LDE));  // CanonicCoset(LDE).step()
    for (int c = 0; c < SM; ++c) batch_for(batches, oods).samples.push_back({col[c].lde.data(), col[c].log + B, cur[c], next()});
    for (int c = SM; c < NCOLS; ++c) {
      PointM g = lifting_gen;
      for (uint32_t i = 0; i < col[c].log + B; ++i) g = pdbl(g);
      const uint32_t lg = col[c].log + B;
      batch_for(batches, qpadd(oods, qpfromm(g))).samples.push_back({col[c].lde.data(), lg, cur[c], next()});
      batch_for(batches, prev).samples.push_back({col[c].lde.data(), lg, before[c], next()});
      batch_for(batches, oods).samples.push_back({col[c].lde.data(), lg, cur[c], next()});
    }
    for (int k = 0; k < 8; ++k) batch_for(batches, oods).samples.push_back({comp_lde[k].data(), LDE, sampled_comp[k], next()});
  }
  std::vector<uint32_t> qcol[4];
  quotient_columns(batches, LDE, qcol);

  FriRun fr = fri_pow_queries(ch, qcol, LDE, xp.cfg, xp.n_threads);
  if (!fr.ok) return std::string();

  // Decommitments: tree 0 at the lifting domain's positions mapped to its own size.
  std::vector<size_t> pre_q;
  for (size_t q : fr.queries) pre_q.push_back(((q >> (LDE - (t + B) + 1)) << 1) + (q & 1));
  Decommitment d0 = merkle_decommit(t0, refs(TA, 3), pre_q);
  Decommitment d1 = merkle_decommit(t1, refs(A, 4), fr.queries);
  Decommitment d2 = merkle_decommit(t2, refs(SM, 8), fr.queries);
  Decommitment d3 = merkle_decommit(t3, comp_cols, fr.queries);

  // Self-checks: the lookup balances and the composition matches the constraints at P.
  if (!qiszero(qadd(claimed[0], claimed[1]))) return std::string("CONSTRAINTS_NOT_SATISFIED");
  {
    const QM31 basis[4] = {qone(), qfrom(0, 1, 0, 0), qfrom(0, 0, 1, 0), qfrom(0, 0, 0, 1)};
    auto secure = [&](const std::vector<QM31>& v, int c0) {
      QM31 r = qzero();
      for (int k = 0; k < 4; ++k) r = qadd(r, qmul(v[c0 + k], basis[k]));
      return r;
    };
    QM31 left = qzero(), right = qzero();
    for (int k = 0; k < 4; ++k) { left = qadd(left, qmul(sampled_comp[k], basis[k])); right = qadd(right, qmul(sampled_comp[4 + k], basis[k])); }
    PointQ pp = oods;
    for (uint32_t i = 0; i + 2 < CL; ++i) pp = qpdbl(pp);
    const QM31 comp_oods = qadd(left, qmul(pp.x, right));
    const QM31 d_main = qsub(qadd(qadd(cur[A], qmul(alpha, cur[A + 1])), qmul(alpha2, cur[A + 2])), z);
    const QM31 d_table = qsub(qadd(qadd(cur[TA], qmul(alpha, cur[TA + 1])), qmul(alpha2, cur[TA + 2])), z);
    const QM31 c_main = qsub(qmul(qadd(qsub(secure(cur, SM), secure(before, SM)),
                                       qmulm(claimed[0], minv((uint32_t)(((size_t)1 << n) % P)))), d_main), qone());
    const QM31 c_table = qadd(qmul(qadd(qsub(secure(cur, ST), secure(before, ST)),
                                        qmulm(claimed[1], minv((uint32_t)(((size_t)1 << t) % P)))), d_table), cur[M]);
    const QM31 expect = qadd(qmul(qmul(random_coeff, c_main), qinv(coset_vanishing_q(coset_odds(n), doubled(oods, n)))),
                             qmul(c_table, qinv(coset_vanishing_q(coset_odds(t), doubled(oods, t)))));
    if (!qeq(expect, comp_oods)) return std::string("CONSTRAINTS_NOT_SATISFIED");
  }

  Json j;
  j.s += "{\"config\":{\"pow_bits\":"; j.u(xp.cfg.pow_bits);
  j.s += ",\"fri_config\":{\"log_blowup_factor\":"; j.u(B);
  j.s += ",\"log_last_layer_degree_bound\":"; j.u(xp.cfg.log_last_layer_degree_bound);
  j.s += ",\"n_queries\":"; j.u(xp.cfg.n_queries);
  j.s += ",\"fold_step\":1},\"lifting_log_size\":null},\"statement\":{\"log_n\":"; j.u(n);
  j.s += ",\"log_table\":"; j.u(t);
  j.s += "},\"commitments\":[";
  j.hash(t0.root()); j.s += ','; j.hash(t1.root()); j.s += ','; j.hash(t2.root()); j.s += ','; j.hash(t3.root());
  j.s += "],\"claimed_sums\":["; j.qm(claimed[0]); j.s += ','; j.qm(claimed[1]);
  j.s += "],\"sampled_values\":[[";
  for (int c = TA; c < A; ++c) { if (c != TA) j.s += ','; j.s += '['; j.qm(cur[c]); j.s += ']'; }
  j.s += "],[";
  for (int c = A; c < SM; ++c) { if (c != A) j.s += ','; j.s += '['; j.qm(cur[c]); j.s += ']'; }
  j.s += "],[";
  for (int c = SM; c < NCOLS; ++c) { if (c != SM) j.s += ','; j.s += '['; j.qm(before[c]); j.s += ','; j.qm(cur[c]); j.s += ']'; }
  j.s += "],[";
  for (int k = 0; k < 8; ++k) { if (k) j.s += ','; j.s += '['; j.qm(sampled_comp[k]); j.s += ']'; }
  j.s += "]],";
  json_decommit_and_fri(j, {&d0, &d1, &d2, &d3}, fr, qcol);
  j.s += "}";
  return j.s;
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points.
// ---------------------------------------------------------------------------
// Montgomery batch inversion, batchInverseClassic (src/core/fields/mod.zig:178-200): prefix products,
// one inversion of the total, backward pass. Returns -2 (DivisionByZero) when an element is zero.
template <class F, class Mul, class Inv, class IsZero>
int batch_inverse_classic(std::vector<F>& col, Mul mul, Inv inv, IsZero is_zero) {
  size_t n = col.size();
  if (n == 0) return 0;
  std::vector<F> dst(n);
  dst[0] = col[0];
  for (size_t i = 1; i < n; ++i) dst[i] = mul(dst[i - 1], col[i]);
  if (is_zero(dst[n - 1])) return -2;
  F cur = inv(dst[n - 1]);
  for (size_t i = n; i-- > 1;) {
    dst[i] = mul(dst[i - 1], cur);
    cur = mul(cur, col[i]);
  }
  dst[0] = cur;
  col.swap(dst);
  return 0;
}

QM31 qinv_oracle(QM31 x) { return qinv(x); }

extern "C" {

int oracle_gen_trace(uint32_t log_n_rows, uint32_t sequence_len, int trace_kind, uint64_t seed, uint32_t* out) {
  if (log_n_rows == 0 || log_n_rows >= 31 || sequence_len < 2 || !out) return -1;
  gen_trace(log_n_rows, sequence_len, trace_kind, seed, out);
  return 0;
}

int oracle_prove_wide_fib(uint32_t log_n_rows, uint32_t sequence_len, const oracle_pcs_config* cfg,
                          const uint32_t* trace, int trace_kind, uint64_t trace_seed, int has_channel_seed,
                          uint64_t channel_seed, int n_threads, uint8_t* out, size_t out_cap, size_t* out_len) {
  if (!cfg || log_n_rows < 1 || log_n_rows > 26 || sequence_len < 2 || cfg->log_blowup_factor < 1 ||
      cfg->log_blowup_factor > 4 || cfg->n_queries == 0)
    return -1;
  if (log_n_rows + cfg->log_blowup_factor < cfg->log_last_layer_degree_bound + cfg->log_blowup_factor + 1) return -1;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  std::vector<uint32_t> own;
  if (!trace) {
    own.resize((size_t)sequence_len << log_n_rows);
    gen_trace(log_n_rows, sequence_len, trace_kind, trace_seed, own.data());
    trace = own.data();
  }
  ProveParams pp{log_n_rows, sequence_len, *cfg, has_channel_seed != 0, channel_seed, n_threads};
  std::string s = prove_wide_fib(pp, trace);
  if (s.empty()) return -3;
  if (s == "CONSTRAINTS_NOT_SATISFIED") return -4;
  if (out_len) *out_len = s.size();
  if (!out || out_cap < s.size()) return -2;
  std::memcpy(out, s.data(), s.size());
  return 0;
}

int oracle_prove_logup_xor(uint32_t log_n, uint32_t log_table, const oracle_pcs_config* cfg, uint64_t seed,
                           int has_channel_seed, uint64_t channel_seed, int n_threads, uint8_t* out, size_t out_cap,
                           size_t* out_len) {
  if (!cfg || log_n < 1 || log_n > 24 || (log_table != 8 && log_table != 16) || cfg->log_blowup_factor < 1 ||
      cfg->log_blowup_factor > 4 || cfg->n_queries == 0)
    return -1;
  if (cfg->log_last_layer_degree_bound + cfg->log_blowup_factor + 1 > std::max(log_n, log_table) + cfg->log_blowup_factor)
    return -1;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  XorParams xp{log_n, log_table, *cfg, seed, has_channel_seed != 0, channel_seed, n_threads};
  std::string s = prove_logup_xor(xp);
  if (s.empty()) return -3;
  if (s == "CONSTRAINTS_NOT_SATISFIED") return -4;
  if (s == "DIVISION_BY_ZERO") return -5;
  if (out_len) *out_len = s.size();
  if (!out || out_cap < s.size()) return -2;
  std::memcpy(out, s.data(), s.size());
  return 0;
}

double oracle_last_pow_seconds(void) { return last_pow_seconds(); }

int oracle_interpolate(uint32_t log_size, uint32_t* values) {
  if (log_size < 1 || log_size > 28 || !values) return -1;
  CircleDomain d = canonic_domain(log_size);
  circle_interpolate(values, d, make_twiddles(d.half));
  return 0;
}

int oracle_evaluate(uint32_t log_size, uint32_t* values) {
  if (log_size < 1 || log_size > 28 || !values) return -1;
  CircleDomain d = canonic_domain(log_size);
  circle_evaluate(values, d, make_twiddles(d.half));
  return 0;
}

int oracle_extend(uint32_t log_size, uint32_t log_blowup, const uint32_t* coeffs, uint32_t* evals) {
  if (log_size < 1 || log_size + log_blowup > 28 || !coeffs || !evals) return -1;
  circle_extend(coeffs, log_size, log_blowup, evals, make_twiddles(canonic_domain(log_size + log_blowup).half));
  return 0;
}

int oracle_merkle_root(uint32_t n_cols, const uint32_t* log_sizes, const uint32_t* const* cols, uint8_t root[32]) {
  std::vector<ColRef> c;
  for (uint32_t i = 0; i < n_cols; ++i) c.push_back({cols[i], log_sizes[i]});
  MerkleTree t = merkle_commit(c);
  std::memcpy(root, t.root().data(), 32);
  return 0;
}

int oracle_merkle_layers(uint32_t n_cols, const uint32_t* log_sizes, const uint32_t* const* cols, uint8_t* out_layers) {
  std::vector<ColRef> c;
  for (uint32_t i = 0; i < n_cols; ++i) c.push_back({cols[i], log_sizes[i]});
  MerkleTree t = merkle_commit(c);
  size_t at = 0;
  for (int k = (int)t.max_log; k >= 0; --k)
    for (const Hash& h : t.layers[k]) { std::memcpy(out_layers + at, h.data(), 32); at += 32; }
  return 0;
}

int oracle_fold_circle_into_line(uint32_t src_log_size, const uint32_t* src, const uint32_t alpha_in[4], uint32_t* dst) {
  if (src_log_size < 2 || src_log_size > 28) return -1;
  size_t n = (size_t)1 << src_log_size, m = n / 2;
  CircleDomain dom = canonic_domain(src_log_size);
  std::vector<PointM> pts = dom.half.points(m);
  QM31 alpha = qload(alpha_in), a2 = qsq(alpha);
  for (size_t i = 0; i < m; ++i) {
    uint32_t py = pts[bit_reverse_index(i, src_log_size - 1)].y;
    QM31 f0 = qfrom(src[2 * i], src[n + 2 * i], src[2 * n + 2 * i], src[3 * n + 2 * i]);
    QM31 f1 = qfrom(src[2 * i + 1], src[n + 2 * i + 1], src[2 * n + 2 * i + 1], src[3 * n + 2 * i + 1]);
    qibutterfly(f0, f1, minv(py));
    QM31 d = qfrom(dst[i], dst[m + i], dst[2 * m + i], dst[3 * m + i]);
    QM31 r = qadd(qmul(d, a2), qadd(qmul(alpha, f1), f0));
    uint32_t w[4]; qstore(r, w);
    for (int k = 0; k < 4; ++k) dst[k * m + i] = w[k];
  }
  return 0;
}

int oracle_fold_line(uint32_t src_log_size, uint32_t first_line_log_size, const uint32_t* src, const uint32_t alpha_in[4], uint32_t* dst) {
  if (src_log_size < 1 || src_log_size > first_line_log_size || first_line_log_size > 28) return -1;
  Coset c = coset_half_odds(first_line_log_size);
  for (uint32_t k = src_log_size; k < first_line_log_size; ++k) c = c.dbl();
  size_t n = (size_t)1 << src_log_size, m = n / 2;
  std::vector<PointM> pts = c.points(m);
  QM31 alpha = qload(alpha_in);
  for (size_t i = 0; i < m; ++i) {
    uint32_t x = pts[bit_reverse_index(i, src_log_size - 1)].x;
    QM31 f0 = qfrom(src[2 * i], src[n + 2 * i], src[2 * n + 2 * i], src[3 * n + 2 * i]);
    QM31 f1 = qfrom(src[2 * i + 1], src[n + 2 * i + 1], src[2 * n + 2 * i + 1], src[3 * n + 2 * i + 1]);
    qibutterfly(f0, f1, minv(x));
    QM31 r = qadd(f0, qmul(alpha, f1));
    uint32_t w[4]; qstore(r, w);
    for (int k = 0; k < 4; ++k) dst[k * m + i] = w[k];
  }
  return 0;
}

int oracle_eval_at_point(uint32_t log_size, const uint32_t* coeffs, const uint32_t px[4], const uint32_t py[4], uint32_t out[4]) {
  if (log_size > 28) return -1;
  qstore(eval_at_point(coeffs, log_size, {qload(px), qload(py)}), out);
  return 0;
}

int oracle_blake2s(const uint8_t* data, size_t len, uint8_t out[32]) {
  Hash h = b2s(data, len);
  std::memcpy(out, h.data(), 32);
  return 0;
}

int oracle_pow_grind(const uint8_t digest[32], uint32_t n_bits, int n_threads, uint64_t* nonce) {
  Hash d; std::memcpy(d.data(), digest, 32);
  *nonce = pow_grind(d, n_bits, n_threads);
  return 0;
}

int oracle_batch_inverse(uint32_t degree, uint64_t n, const uint32_t* src, uint32_t* dst) {
  if (degree == 1) {
    std::vector<uint32_t> v(src, src + n);
    int r = batch_inverse_classic(v, mmul, minv, [](uint32_t a) { return a == 0; });
    if (r == 0) std::copy(v.begin(), v.end(), dst);
    return r;
  }
  if (degree == 2) {
    std::vector<CM31> v(n);
    for (uint64_t i = 0; i < n; ++i) v[i] = {src[i], src[n + i]};
    int r = batch_inverse_classic(v, cmul, cinv, czero);
    if (r == 0)
      for (uint64_t i = 0; i < n; ++i) { dst[i] = v[i].a; dst[n + i] = v[i].b; }
    return r;
  }
  if (degree == 4) {
    std::vector<QM31> v(n);
    for (uint64_t i = 0; i < n; ++i) v[i] = qfrom(src[i], src[n + i], src[2 * n + i], src[3 * n + i]);
    int r = batch_inverse_classic(v, qmul, qinv_oracle, qiszero);
    if (r == 0)
      for (uint64_t i = 0; i < n; ++i) {
        uint32_t w[4]; qstore(v[i], w);
        for (int k = 0; k < 4; ++k) dst[k * n + i] = w[k];
      }
    return r;
  }
  return -1;
}

// LogUp interaction columns. Fractions per use: relation_combine / relation_multiplicity
// (src/backends/metal/shaders/core/relation.metal:54-90): denominator = sum_j alpha_j word_j - z,
// numerator = +/- multiplicity; a column of two uses is (n_a d_b + n_b d_a) / (d_a d_b)
// (relation.metal:77-90). Column c holds the running sum over columns 0..c of the row's fractions
// (stwo_zig_relation_fused, relation.metal:131-158). The last column is then summed over rows:
// order 1 in coset order with the total/N shift, the scalar law of
// src/tests/metal/backend/commitment_test.zig:140-152; order 0 in storage order without shift
// (cumulativeColumn, src/frontends/riscv/air/logup.zig:83-105).
int oracle_logup_interaction(uint32_t log_rows, uint32_t n_uses, const oracle_logup_use* uses,
                             const uint32_t* alphas, const uint32_t z_in[4], uint32_t batch, uint32_t order,
                             uint32_t* out, uint32_t claimed_out[4]) {
  if (log_rows > 24 || n_uses == 0 || (batch != 1 && batch != 2) || order > 1) return -1;
  const size_t rows = (size_t)1 << log_rows;
  const uint32_t n_cols = (n_uses + batch - 1) / batch;
  const QM31 z = qload(z_in);
  auto den = [&](const oracle_logup_use& u, size_t r) {
    QM31 acc = qneg(z);
    for (uint32_t j = 0; j < u.n_words; ++j) {
      uint32_t w = u.words[j] ? u.words[j][r] : u.constants[j];
      acc = qadd(acc, qmulm(qload(alphas + 4 * j), w));
    }
    return acc;
  };
  auto num = [&](const oracle_logup_use& u, size_t r) {
    uint32_t m = u.multiplicity ? u.multiplicity[r] : 1u;
    return u.negate ? mneg(m) : m;
  };
  std::vector<QM31> last(rows);
  for (size_t r = 0; r < rows; ++r) {
    QM31 acc = qzero();
    for (uint32_t c = 0; c < n_cols; ++c) {
      uint32_t u0 = c * batch;
      QM31 n, d;
      if (batch == 2 && u0 + 1 < n_uses) {
        QM31 da = den(uses[u0], r), db = den(uses[u0 + 1], r);
        n = qadd(qmulm(da, num(uses[u0 + 1], r)), qmulm(db, num(uses[u0], r)));
        d = qmul(da, db);
      } else {
        n = qbase(num(uses[u0], r));
        d = den(uses[u0], r);
      }
      if (qiszero(d)) return -2;
      acc = qadd(acc, qmul(n, qinv(d)));
      uint32_t w[4]; qstore(acc, w);
      for (int k = 0; k < 4; ++k) out[(4 * (size_t)c + k) * rows + r] = w[k];
    }
    last[r] = acc;
  }
  QM31 total = qzero();
  for (size_t r = 0; r < rows; ++r) total = qadd(total, last[r]);
  uint32_t* lc = out + 4 * (size_t)(n_cols - 1) * rows;
  QM31 acc = qzero();
  if (order == 0) {
    for (size_t r = 0; r < rows; ++r) {
      acc = qadd(acc, last[r]);
      uint32_t w[4]; qstore(acc, w);
      for (int k = 0; k < 4; ++k) lc[k * rows + r] = w[k];
    }
  } else {
    QM31 shift = qmulm(total, minv((uint32_t)(rows % P)));
    for (size_t s = 0; s < rows; ++s) {
      size_t ci = (s & 1) == 0 ? s / 2 : rows - 1 - s / 2;
      size_t r = bit_reverse_index(ci, log_rows);
      acc = qadd(acc, qsub(last[r], shift));
      uint32_t w[4]; qstore(acc, w);
      for (int k = 0; k < 4; ++k) lc[k * rows + r] = w[k];
    }
  }
  qstore(total, claimed_out);
  return 0;
}

// XOR-lookup trace (the device kernel k_xor_trace restated): SplitMix64 of
// seed ^ (0xD6E8FEB86659FD93 * (row + 1)), a = low byte, b = next byte, c = a ^ b; the
// table follows the reference's bitwise table layout (row a * 256 + b,
// src/frontends/riscv/air/preprocessed/bitwise.zig:17-35); mult counts each (a, b).
int oracle_xor_lookup_trace(uint32_t log_n, uint64_t seed, uint32_t* main_cols, uint32_t* table, uint32_t* mult) {
  if (log_n > 26) return -1;
  const uint64_t rows = 1ull << log_n;
  std::fill(mult, mult + 65536, 0u);
  for (uint64_t r = 0; r < rows; ++r) {
    uint64_t z = (seed ^ (0xD6E8FEB86659FD93ull * (r + 1))) + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    uint32_t a = (uint32_t)z & 255u, b = (uint32_t)(z >> 8) & 255u;
    main_cols[r] = a;
    main_cols[rows + r] = b;
    main_cols[2 * rows + r] = a ^ b;
    ++mult[a << 8 | b];
  }
  for (uint32_t i = 0; i < 65536; ++i) {
    table[i] = i >> 8;
    table[65536 + i] = i & 255u;
    table[2 * 65536 + i] = (i >> 8) ^ (i & 255u);
  }
  return 0;
}

}  // extern "C"
