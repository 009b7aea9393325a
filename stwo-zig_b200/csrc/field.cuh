// M31 / CM31 / QM31 arithmetic in 32-bit lanes, usable from host and device.
//
// M31: p = 2^31 - 1, canonical representatives in [0, p) (src/core/fields/m31.zig:49-75).
// CM31 = M31[i]/(i^2 + 1) (src/core/fields/cm31.zig:97).
// QM31 = CM31[u]/(u^2 - (2 + i)), stored as (c0.a, c0.b, c1.a, c1.b)
// (src/core/fields/qm31.zig:13,153-206).
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define SB_HD __host__ __device__ __forceinline__
#else
#define SB_HD inline
#endif

namespace sb {

constexpr uint32_t P = 0x7fffffffu;

// Unsigned min: for s in [0, 2p) picks s or s - p without a branch.
SB_HD uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

SB_HD uint32_t madd(uint32_t a, uint32_t b) { uint32_t s = a + b; return umin32(s, s - P); }
SB_HD uint32_t msub(uint32_t a, uint32_t b) { uint32_t d = a - b; return umin32(d, d + P); }
SB_HD uint32_t mneg(uint32_t a) { return a == 0 ? 0 : P - a; }

// Product of two canonical values. With a, b < p the 62-bit product splits into
// lo = bits [0,31) and hi = bits [31,62), lo + hi <= 2p - 3, so one conditional
// subtraction lands in [0, p).
SB_HD uint32_t mmul(uint32_t a, uint32_t b) {
  uint64_t x = (uint64_t)a * b;
  uint32_t s = ((uint32_t)x & P) + (uint32_t)(x >> 31);
  return umin32(s, s - P);
}

// Reduction of a lazily accumulated 64-bit sum of products.
SB_HD uint32_t mreduce64(uint64_t x) {
  uint64_t r = (x & P) + (x >> 31);          // < 2^34
  uint32_t s = (uint32_t)(r & P) + (uint32_t)(r >> 31);  // < 2^31 + 8
  return umin32(s, s - P);
}
// Partial fold that keeps a sum of products small enough to keep accumulating:
// input < 2^64, output < 2^34.
SB_HD uint64_t mfold64(uint64_t x) { return (x & P) + (x >> 31); }

SB_HD uint32_t mpow(uint32_t a, uint32_t e) {
  uint32_t acc = 1;
  while (e) { if (e & 1) acc = mmul(acc, a); a = mmul(a, a); e >>= 1; }
  return acc;
}
SB_HD uint32_t minv(uint32_t a) { return mpow(a, P - 2); }

struct CM31 { uint32_t a, b; };
SB_HD CM31 cadd(CM31 x, CM31 y) { return {madd(x.a, y.a), madd(x.b, y.b)}; }
SB_HD CM31 csub(CM31 x, CM31 y) { return {msub(x.a, y.a), msub(x.b, y.b)}; }
SB_HD CM31 cneg(CM31 x) { return {mneg(x.a), mneg(x.b)}; }
SB_HD CM31 cmul(CM31 x, CM31 y) {
  return {msub(mmul(x.a, y.a), mmul(x.b, y.b)), madd(mmul(x.a, y.b), mmul(x.b, y.a))};
}
SB_HD CM31 cmulm(CM31 x, uint32_t m) { return {mmul(x.a, m), mmul(x.b, m)}; }
SB_HD CM31 cinv(CM31 x) {
  uint32_t d = minv(madd(mmul(x.a, x.a), mmul(x.b, x.b)));
  return {mmul(x.a, d), mmul(mneg(x.b), d)};
}
SB_HD bool ceq(CM31 x, CM31 y) { return x.a == y.a && x.b == y.b; }

struct QM31 { CM31 c0, c1; };
SB_HD QM31 qmake(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return {{a, b}, {c, d}}; }
SB_HD QM31 qbase(uint32_t a) { return {{a, 0}, {0, 0}}; }
SB_HD QM31 qzero() { return qbase(0); }
SB_HD QM31 qone() { return qbase(1); }
SB_HD QM31 qadd(QM31 x, QM31 y) { return {cadd(x.c0, y.c0), cadd(x.c1, y.c1)}; }
SB_HD QM31 qsub(QM31 x, QM31 y) { return {csub(x.c0, y.c0), csub(x.c1, y.c1)}; }
SB_HD QM31 qneg(QM31 x) { return {cneg(x.c0), cneg(x.c1)}; }
// x * (2 + i)
SB_HD CM31 mul_by_r(CM31 x) { return {msub(madd(x.a, x.a), x.b), madd(x.a, madd(x.b, x.b))}; }
SB_HD QM31 qmul(QM31 x, QM31 y) {
  CM31 ac = cmul(x.c0, y.c0), bd = cmul(x.c1, y.c1);
  CM31 cross = csub(csub(cmul(cadd(x.c0, x.c1), cadd(y.c0, y.c1)), ac), bd);
  return {cadd(ac, mul_by_r(bd)), cross};
}
SB_HD QM31 qmulm(QM31 x, uint32_t m) { return {cmulm(x.c0, m), cmulm(x.c1, m)}; }
SB_HD QM31 qmulc(QM31 x, CM31 c) { return {cmul(x.c0, c), cmul(x.c1, c)}; }
SB_HD QM31 qsq(QM31 x) { return qmul(x, x); }
SB_HD QM31 qconj(QM31 x) { return {x.c0, cneg(x.c1)}; }
SB_HD bool qeq(QM31 x, QM31 y) { return ceq(x.c0, y.c0) && ceq(x.c1, y.c1); }
SB_HD bool qiszero(QM31 x) { return x.c0.a == 0 && x.c0.b == 0 && x.c1.a == 0 && x.c1.b == 0; }
SB_HD QM31 qinv(QM31 x) {
  CM31 denom = csub(cmul(x.c0, x.c0), mul_by_r(cmul(x.c1, x.c1)));
  CM31 di = cinv(denom);
  return {cmul(x.c0, di), cmul(cneg(x.c1), di)};
}
SB_HD void qstore4(QM31 v, uint32_t* o) { o[0] = v.c0.a; o[1] = v.c0.b; o[2] = v.c1.a; o[3] = v.c1.b; }
SB_HD QM31 qload4(const uint32_t* i) { return qmake(i[0], i[1], i[2], i[3]); }

// Circle points over M31 (src/core/circle.zig:8-60).
struct PointM { uint32_t x, y; };
SB_HD PointM padd(PointM a, PointM b) {
  return {msub(mmul(a.x, b.x), mmul(a.y, b.y)), madd(mmul(a.x, b.y), mmul(a.y, b.x))};
}
SB_HD PointM pconj(PointM a) { return {a.x, mneg(a.y)}; }

struct PointQ { QM31 x, y; };
SB_HD PointQ qpadd(PointQ a, PointQ b) {
  return {qsub(qmul(a.x, b.x), qmul(a.y, b.y)), qadd(qmul(a.x, b.y), qmul(a.y, b.x))};
}
SB_HD QM31 qdouble_x(QM31 x) { QM31 s = qsq(x); return qsub(qadd(s, s), qone()); }
SB_HD uint32_t double_x(uint32_t x) { uint32_t s = mmul(x, x); return msub(madd(s, s), 1); }

// Butterflies (src/core/fft.zig:8-18).
SB_HD void butterfly(uint32_t& v0, uint32_t& v1, uint32_t t) {
  uint32_t m = mmul(v1, t);
  v1 = msub(v0, m);
  v0 = madd(v0, m);
}
SB_HD void ibutterfly(uint32_t& v0, uint32_t& v1, uint32_t it) {
  uint32_t a = v0;
  v0 = madd(a, v1);
  v1 = mmul(msub(a, v1), it);
}

}  // namespace sb
