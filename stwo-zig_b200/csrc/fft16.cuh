// Register radix-16 circle-FFT building blocks (used by fft.cu for domains of
// 2^16 .. 2^22 words).
//
// A thread holds 16 elements whose indices differ only in a 4-bit window of
// the transform index, applies up to 4 butterfly layers of that window in
// registers, and exchanges elements with other threads through shared memory
// between windows. Twiddles of one window come from one to two vector loads
// per layer (the elements of a window share consecutive twiddle blocks), read
// from the doubled tower (TwiddleView::tower2): with t2 = 2t the 64-bit
// product a * t2 = 2at holds at >> 31 in its high word and (at mod 2^31) << 1
// in its low word, so the product's reduction needs no mask and no 64-bit
// shift.
//
// Shared-memory positions are swizzled by swz(i) = i ^ (16*parity(i>>5) ^ ((i>>5)&15)).
// swz is linear over GF(2), so the position of element k of a thread is
// swz(base) ^ swz(k << W) with the second term a per-k constant, and every
// window mapping used here puts the 32 threads of a warp on 32 distinct banks.
#pragma once
#include "circle.cuh"
#include "field.cuh"

namespace sb {
namespace fft16 {

__host__ __device__ __forceinline__ uint32_t swz(uint32_t i) {
  uint32_t v = i >> 5;
#if defined(__CUDA_ARCH__)
  uint32_t par = __popc(v) & 1;
#else
  uint32_t par = __builtin_popcount(v) & 1;
#endif
  return i ^ ((par << 4) ^ (v & 15));
}

// a * t mod p for a < p and t2 = 2t, t < p. With 2at = hi * 2^32 + lo (lo even),
// at = hi * 2^31 + lo / 2 = hi + lo / 2 (mod p); hi <= 2^31 - 4 and lo / 2 < 2^31,
// so the sum is below 2p and one conditional subtraction makes it canonical.
__device__ __forceinline__ uint32_t mmul2(uint32_t a, uint32_t t2) {
  const uint64_t x = (uint64_t)a * t2;
  const uint32_t s = (uint32_t)(x >> 32) + ((uint32_t)x >> 1);
  return umin32(s, s - P);
}
// Negation of a doubled twiddle: 2(p - t) = 2p - 2t, and 0 for t = 0.
__device__ __forceinline__ uint32_t mneg2(uint32_t t2) { return t2 == 0 ? 0 : 2 * P - t2; }

// The butterflies of field.cuh with the twiddle given doubled.
__device__ __forceinline__ void butterfly2(uint32_t& v0, uint32_t& v1, uint32_t t2) {
  const uint32_t m = mmul2(v1, t2);
  v1 = msub(v0, m);
  v0 = madd(v0, m);
}
__device__ __forceinline__ void ibutterfly2(uint32_t& v0, uint32_t& v1, uint32_t it2) {
  const uint32_t a = v0;
  v0 = madd(a, v1);
  v1 = mmul2(msub(a, v1), it2);
}

// `n` consecutive doubled twiddles of line layer s (s >= 1) starting at block h0
// (h0 is a multiple of n, the layer offset a multiple of 16 bytes).
template <int N>
__device__ __forceinline__ void load_line(const TwiddleView& tv, uint32_t s, uint64_t h0, uint32_t (&tw)[8]) {
  const uint32_t* p = tv.tower2 + ((1u << tv.root_log) - (1u << (tv.line_log - s + 1))) + h0;
  if (N == 8) {
    uint4 a = __ldg(reinterpret_cast<const uint4*>(p)), b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
    tw[0] = a.x; tw[1] = a.y; tw[2] = a.z; tw[3] = a.w; tw[4] = b.x; tw[5] = b.y; tw[6] = b.z; tw[7] = b.w;
  } else if (N == 4) {
    uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    tw[0] = a.x; tw[1] = a.y; tw[2] = a.z; tw[3] = a.w;
  } else if (N == 2) {
    uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
    tw[0] = a.x; tw[1] = a.y;
  } else {
    tw[0] = __ldg(p);
  }
}

// Doubled circle-layer twiddles of 8 consecutive pairs h0 .. h0+7 (h0 a multiple of 8):
// pattern [y, -y, -x, x] over the (x, y) pairs of line layer 0.
__device__ __forceinline__ void load_circle8(const TwiddleView& tv, uint64_t h0, uint32_t (&tw)[8]) {
  const uint32_t* l0 = tv.tower2 + ((1u << tv.root_log) - (1u << tv.line_log));
  uint4 q = __ldg(reinterpret_cast<const uint4*>(l0 + (h0 >> 1)));
  tw[0] = q.y; tw[1] = mneg2(q.y); tw[2] = mneg2(q.x); tw[3] = q.x;
  tw[4] = q.w; tw[5] = mneg2(q.w); tw[6] = mneg2(q.z); tw[7] = q.z;
}

// Applies window layers j in [JLO, JHI) to x (element k at transform index
// base + (k << w0) in the window's index space). Layer j is global layer
// s = sbase + w0 + j; its pair (k, k + 2^j) uses twiddle block
// (hb >> (w0 + j + 1)) + (k >> (j + 1)), hb being the index of element 0 in the
// space where twiddle blocks are counted.
template <bool INV, int J>
__device__ __forceinline__ void layer16(uint32_t (&x)[16], const TwiddleView& tv, uint32_t sbase, uint32_t w0,
                                        uint64_t hb) {
  const uint32_t s = sbase + w0 + J;
  uint32_t tw[8];
  const uint64_t h0 = hb >> (w0 + J + 1);
  if (s == 0) {
    load_circle8(tv, h0, tw);
  } else {
    load_line<(8 >> J)>(tv, s, h0, tw);
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if (k & (1 << J)) continue;
    const uint32_t t = tw[k >> (J + 1)];
    if (INV) ibutterfly2(x[k], x[k | (1 << J)], t);
    else butterfly2(x[k], x[k | (1 << J)], t);
  }
}

template <bool INV, int JLO, int JHI>
__device__ __forceinline__ void radix16(uint32_t (&x)[16], const TwiddleView& tv, uint32_t sbase, uint32_t w0,
                                        uint64_t hb) {
  if constexpr (JLO < JHI) {
    if constexpr (INV) {
      layer16<INV, JLO>(x, tv, sbase, w0, hb);
      radix16<INV, JLO + 1, JHI>(x, tv, sbase, w0, hb);
    } else {
      layer16<INV, JHI - 1>(x, tv, sbase, w0, hb);
      radix16<INV, JLO, JHI - 1>(x, tv, sbase, w0, hb);
    }
  }
}

template <bool INV>
__device__ __forceinline__ void radix16_dyn(uint32_t (&x)[16], const TwiddleView& tv, uint32_t sbase, uint32_t w0,
                                            uint64_t hb, uint32_t nl) {
  switch (nl) {
    case 4: radix16<INV, 0, 4>(x, tv, sbase, w0, hb); break;
    case 3: radix16<INV, 0, 3>(x, tv, sbase, w0, hb); break;
    case 2: radix16<INV, 0, 2>(x, tv, sbase, w0, hb); break;
    default: radix16<INV, 0, 1>(x, tv, sbase, w0, hb); break;
  }
}

// Inserts 4 zero bits at position w0 of q.
__device__ __forceinline__ uint32_t spread(uint32_t q, uint32_t w0) {
  return ((q >> w0) << (w0 + 4)) | (q & ((1u << w0) - 1));
}

}  // namespace fft16
}  // namespace sb
