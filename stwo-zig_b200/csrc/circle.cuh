// Circle-group indexing, cosets, domains and the twiddle tower, host and device.
//
// A point of the order-2^31 circle group is named by its index u (u * G, G the
// generator (2, 1268011823), src/core/circle.zig:137-141). Any point is one
// addition of two table entries: u = hi * 2^16 + lo.
// Cosets and canonic circle domains: src/core/circle.zig:245-375,
// src/core/poly/circle/canonic.zig:12-27, src/core/poly/circle/domain.zig:23-60.
// Twiddle tower: src/prover/poly/twiddles.zig:37-91, twiddle_tower.zig:29-81.
#pragma once
#include <cstdint>
#include <vector>

#include "field.cuh"

namespace sb {

constexpr uint32_t CIRCLE_LOG_ORDER = 31;
constexpr uint32_t INDEX_MASK = (1u << 31) - 1;
constexpr uint32_t POINT_TABLE_LO_BITS = 16;
constexpr uint32_t POINT_TABLE_LO = 1u << POINT_TABLE_LO_BITS;          // lo * G
constexpr uint32_t POINT_TABLE_HI = 1u << (31 - POINT_TABLE_LO_BITS);   // (hi * 2^16) * G

SB_HD uint32_t subgroup_gen(uint32_t log_size) { return 1u << (CIRCLE_LOG_ORDER - log_size); }

// Device/host view of the point table: table[0 .. LO) = lo * G, table[LO .. LO + HI) = (hi 2^16) G.
struct PointTable {
  const PointM* t;
  SB_HD PointM at(uint32_t idx) const {
    idx &= INDEX_MASK;
    PointM lo = t[idx & (POINT_TABLE_LO - 1)];
    PointM hi = t[POINT_TABLE_LO + (idx >> POINT_TABLE_LO_BITS)];
    return padd(lo, hi);
  }
};

inline std::vector<PointM> build_point_table() {
  std::vector<PointM> t(POINT_TABLE_LO + POINT_TABLE_HI);
  const PointM g = {2, 1268011823};
  PointM cur = {1, 0};
  for (uint32_t i = 0; i < POINT_TABLE_LO; ++i) { t[i] = cur; cur = padd(cur, g); }
  // cur = 2^16 * G now.
  PointM step = cur;
  cur = {1, 0};
  for (uint32_t i = 0; i < POINT_TABLE_HI; ++i) { t[POINT_TABLE_LO + i] = cur; cur = padd(cur, step); }
  return t;
}

// Coset {initial + k * step}, indices mod 2^31.
struct Coset {
  uint32_t initial, step, log_size;
  SB_HD uint32_t index_at(uint64_t i) const { return (uint32_t)((initial + (uint64_t)step * i) & INDEX_MASK); }
  SB_HD Coset dbl() const { return {(initial * 2) & INDEX_MASK, (step * 2) & INDEX_MASK, log_size - 1}; }
};
SB_HD Coset coset_new(uint32_t initial, uint32_t log_size) { return {initial, subgroup_gen(log_size), log_size}; }
SB_HD Coset coset_odds(uint32_t log_size) { return coset_new(subgroup_gen(log_size + 1), log_size); }
SB_HD Coset coset_half_odds(uint32_t log_size) { return coset_new(subgroup_gen(log_size + 2), log_size); }

// CanonicCoset(n).circleDomain(): the half coset halfOdds(n-1) then its conjugate.
struct CircleDomain {
  Coset half;
  SB_HD uint32_t log_size() const { return half.log_size + 1; }
  SB_HD uint32_t index_at(uint64_t i) const {
    uint64_t hs = 1ull << half.log_size;
    if (i < hs) return half.index_at(i);
    return (0u - half.index_at(i - hs)) & INDEX_MASK;
  }
};
SB_HD CircleDomain canonic_domain(uint32_t log_size) { return {coset_half_odds(log_size - 1)}; }

SB_HD uint32_t bitrev(uint32_t i, uint32_t log_size) {
#if defined(__CUDA_ARCH__)
  return log_size == 0 ? i : (__brev(i) >> (32 - log_size));
#else
  if (log_size == 0) return i;
  uint32_t r = 0;
  for (uint32_t k = 0; k < log_size; ++k) { r = (r << 1) | (i & 1); i >>= 1; }
  return r;
#endif
}

// Twiddle tower for the root half coset halfOdds(R). Layer k (0 <= k < R) is
// the x-coordinates of the first half of halfOdds(R - k), bit-reversed, with
// 2^(R-1-k) entries at offset 2^R - 2^(R-k); the last word is 1. The inverse
// tower holds the inverses. A domain whose half coset is halfOdds(L), L <= R,
// reads tower layers R-L .. R-1.
struct TwiddleView {
  const uint32_t* tower;  // forward or inverse
  const uint32_t* tower2; // the same tower's entries doubled (2t < 2^32, not reduced mod p)
  uint32_t root_log;      // R
  uint32_t line_log;      // L
  uint32_t y0;            // y (or 1/y) of halfOdds(L)'s first point, for L <= 1
  // Line layer j = s - 1 (butterfly distance 2^s, s >= 1), pair block h.
  SB_HD uint32_t line(uint32_t s, uint32_t h) const {
    return tower[(1u << root_log) - (1u << (line_log - s + 1)) + h];
  }
  // Circle layer (distance 1), pair h: [y, -y, -x, x] from line layer 0's (x, y)
  // pairs (src/prover/poly/circle/transforms.zig:233-247).
  SB_HD uint32_t circ(uint32_t h) const {
    if (line_log <= 1) return (h & 1) ? mneg(y0) : y0;
    const uint32_t* l0 = tower + (1u << root_log) - (1u << line_log);
    uint32_t m = h >> 2;
    uint32_t x = l0[2 * m], y = l0[2 * m + 1];
    switch (h & 3) {
      case 0: return y;
      case 1: return mneg(y);
      case 2: return mneg(x);
      default: return x;
    }
  }
};

}  // namespace sb
