// Blake2s-256 compression (RFC 7693), host and device.
//
// Used by the lifted Merkle hasher ("leaf"/"node" 64-byte domain prefixes,
// src/core/vcs_lifted/blake2_merkle.zig:9-10,193-262), the Fiat-Shamir channel
// (src/core/channel/blake2s.zig) and the proof-of-work grind (:135-240).
// The state of a 64-byte prefix block is a constant seed, so every leaf or node
// costs the compressions of its payload only.
#pragma once
#include <cstdint>
#include <cstring>

#include "field.cuh"

namespace sb {

SB_HD uint32_t rotr32(uint32_t x, int n) {
#if defined(__CUDA_ARCH__)
  return __funnelshift_r(x, x, n);
#else
  return (x >> n) | (x << (32 - n));
#endif
}

struct B2sIv {
  static constexpr uint32_t v0 = 0x6A09E667u, v1 = 0xBB67AE85u, v2 = 0x3C6EF372u, v3 = 0xA54FF53Au,
                            v4 = 0x510E527Fu, v5 = 0x9B05688Cu, v6 = 0x1F83D9ABu, v7 = 0x5BE0CD19u;
};

// Additions can be issued on the FMA pipe as IMAD x*one+y with a runtime `one`
// (the XOR/rotate half of G keeps the ALU pipe busy; splitting the adds off
// balances the two pipes). On the host `one` is ignored.
SB_HD uint32_t b2s_fadd(uint32_t a, uint32_t b, uint32_t one) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(one), "r"(b));
  return r;
#else
  (void)one;
  return a + b;
#endif
}
#if defined(__CUDA_ARCH__)
#define SB_ADD(a, b) b2s_fadd((a), (b), one)
#else
#define SB_ADD(a, b) ((a) + (b))
#endif

#define SB_B2S_G(a, b, c, d, x, y)                         \
  do {                                                     \
    a = SB_ADD(SB_ADD(a, b), (x)); d = rotr32(d ^ a, 16);  \
    c = SB_ADD(c, d);              b = rotr32(b ^ c, 12);  \
    a = SB_ADD(SB_ADD(a, b), (y)); d = rotr32(d ^ a, 8);   \
    c = SB_ADD(c, d);              b = rotr32(b ^ c, 7);   \
  } while (0)

// One round with the message schedule written out (sigma of RFC 7693 section 2.7).
#define SB_B2S_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  do {                                                                                     \
    SB_B2S_G(v0, v4, v8, v12, m[s0], m[s1]);                                               \
    SB_B2S_G(v1, v5, v9, v13, m[s2], m[s3]);                                               \
    SB_B2S_G(v2, v6, v10, v14, m[s4], m[s5]);                                              \
    SB_B2S_G(v3, v7, v11, v15, m[s6], m[s7]);                                              \
    SB_B2S_G(v0, v5, v10, v15, m[s8], m[s9]);                                              \
    SB_B2S_G(v1, v6, v11, v12, m[s10], m[s11]);                                            \
    SB_B2S_G(v2, v7, v8, v13, m[s12], m[s13]);                                             \
    SB_B2S_G(v3, v4, v9, v14, m[s14], m[s15]);                                             \
  } while (0)

// Rounds 2..10 on the working state v0..v15 and message m (the proof-of-work
// grind runs the first round itself, most of it precomputed per prefix).
#define SB_B2S_ROUNDS_2_TO_10()                                            \
  do {                                                                     \
    SB_B2S_ROUND(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3);    \
    SB_B2S_ROUND(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4);    \
    SB_B2S_ROUND(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8);    \
    SB_B2S_ROUND(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13);    \
    SB_B2S_ROUND(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9);    \
    SB_B2S_ROUND(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11);    \
    SB_B2S_ROUND(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10);    \
    SB_B2S_ROUND(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5);    \
    SB_B2S_ROUND(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0);    \
  } while (0)

// h <- compress(h, m, t, last). All indices are compile-time constants so the
// message and state stay in registers.
SB_HD void b2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t_lo, bool last, uint32_t one = 1) {
  uint32_t v0 = h[0], v1 = h[1], v2 = h[2], v3 = h[3], v4 = h[4], v5 = h[5], v6 = h[6], v7 = h[7];
  uint32_t v8 = B2sIv::v0, v9 = B2sIv::v1, v10 = B2sIv::v2, v11 = B2sIv::v3;
  uint32_t v12 = B2sIv::v4 ^ t_lo, v13 = B2sIv::v5, v14 = last ? ~B2sIv::v6 : B2sIv::v6, v15 = B2sIv::v7;
  SB_B2S_ROUND(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
  SB_B2S_ROUNDS_2_TO_10();
  h[0] ^= v0 ^ v8; h[1] ^= v1 ^ v9; h[2] ^= v2 ^ v10; h[3] ^= v3 ^ v11;
  h[4] ^= v4 ^ v12; h[5] ^= v5 ^ v13; h[6] ^= v6 ^ v14; h[7] ^= v7 ^ v15;
}

SB_HD void b2s_init(uint32_t h[8]) {
  h[0] = B2sIv::v0 ^ 0x01010020u; h[1] = B2sIv::v1; h[2] = B2sIv::v2; h[3] = B2sIv::v3;
  h[4] = B2sIv::v4; h[5] = B2sIv::v5; h[6] = B2sIv::v6; h[7] = B2sIv::v7;
}

// Streaming hasher for host-side transcript work. Counters above 2^32 bytes
// never occur on this path.
struct Blake2sHost {
  uint32_t h[8];
  uint8_t buf[64];
  uint32_t buflen = 0, t = 0;
  Blake2sHost() { b2s_init(h); }
  void block(bool last) {
    uint32_t m[16];
    std::memcpy(m, buf, 64);
    b2s_compress(h, m, t, last);
  }
  void update(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    while (len > 0) {
      if (buflen == 64) { t += 64; block(false); buflen = 0; }
      size_t take = len < 64 - buflen ? len : 64 - buflen;
      std::memcpy(buf + buflen, p, take);
      buflen += (uint32_t)take; p += take; len -= take;
    }
  }
  void finalize(uint8_t out[32]) {
    t += buflen;
    std::memset(buf + buflen, 0, 64 - buflen);
    block(true);
    std::memcpy(out, h, 32);
  }
};

// State after absorbing one 64-byte prefix block (not final), the Merkle seeds.
inline void b2s_prefix_seed(const char* tag, uint32_t out[8]) {
  uint8_t block[64] = {0};
  std::memcpy(block, tag, std::strlen(tag));
  b2s_init(out);
  uint32_t m[16];
  std::memcpy(m, block, 64);
  b2s_compress(out, m, 64, false);
}

}  // namespace sb
