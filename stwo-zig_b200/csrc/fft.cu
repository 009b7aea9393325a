// Circle FFT over M31 columns, B200 layout.
//
// Semantics: the reference's butterfly network (src/prover/poly/circle/transforms.zig:
// evaluate :132-248, interpolate :249-362, first-layer [y,-y,-x,x] twiddles
// :233-247/:309-321, extension :132-147). A transform of 2^D words has D layers;
// layer s pairs indices at distance 2^s (s = 0 is the circle layer, s >= 1 line
// layer s-1) and uses twiddle block h = i >> (s+1).
//
// Decomposition: with b = min(D, LOW_BITS), layers s < b act inside aligned
// blocks of 2^b words (k_fft_low: one CTA per block, shared memory), layers
// s >= b act on the strided sets {g*T + t + m*2^b} (k_fft_high: one CTA per
// group of T adjacent low indices, all m). Both passes apply two layers per
// shared-memory round trip (radix-4 quads in registers).
// interpolate_extend fuses, per strided set: inverse high layers -> 1/n scale ->
// store coefficients -> extension to the blown-up domain -> forward high layers,
// so coefficients and the blown-up evaluations come out of one pass.
#include <cuda.h>  // CUtensorMap and the tiled tensor-map encoder's types

#include <algorithm>
#include <cstring>

#include "fft16.cuh"
#include "kernels.cuh"
#include "tuner.hpp"

namespace sb {

namespace {

constexpr uint32_t LOW_BITS = 11;          // low-pass block: 2^11 words = 8 KiB
constexpr uint32_t LOW_THREADS = 256;
constexpr uint32_t HIGH_T_BITS = 3;        // T = 8 adjacent columns of the strided view (32 B rows)
constexpr uint32_t HIGH_T = 1u << HIGH_T_BITS;
constexpr uint32_t HIGH_THREADS = 512;

__device__ __forceinline__ uint32_t twiddle(const TwiddleView& tv, uint32_t s, uint32_t gi) {
  return s == 0 ? tv.circ(gi >> 1) : tv.line(s, gi >> (s + 1));
}

// Applies layers [s_lo, s_hi) to a shared array of 2^local_bits words whose
// local index l maps to global index base + l (low pass).
template <bool INV>
__device__ void low_layers(uint32_t* sm, uint32_t local_bits, uint64_t base, const TwiddleView& tv,
                           uint32_t s_lo, uint32_t s_hi) {
  const uint32_t n = 1u << local_bits;
  uint32_t nl = s_hi - s_lo;
  // Radix-2 leftover layer first (forward: the top one; inverse: the bottom one).
  if (nl & 1) {
    uint32_t s = INV ? s_lo : s_hi - 1;
    for (uint32_t q = threadIdx.x; q < n / 2; q += blockDim.x) {
      uint32_t l0 = ((q >> s) << (s + 1)) | (q & ((1u << s) - 1));
      uint32_t l1 = l0 + (1u << s);
      uint32_t t = twiddle(tv, s, (uint32_t)(base + l0));
      uint32_t a = sm[l0], b = sm[l1];
      if (INV) ibutterfly(a, b, t); else butterfly(a, b, t);
      sm[l0] = a; sm[l1] = b;
    }
    __syncthreads();
    if (INV) s_lo += 1; else s_hi -= 1;
    nl -= 1;
  }
  for (uint32_t k = 0; k < nl / 2; ++k) {
    uint32_t s = INV ? s_lo + 2 * k : s_hi - 2 - 2 * k;  // pair (s, s+1)
    for (uint32_t q = threadIdx.x; q < n / 4; q += blockDim.x) {
      uint32_t l0 = ((q >> s) << (s + 2)) | (q & ((1u << s) - 1));
      uint32_t l1 = l0 + (1u << s), l2 = l0 + (2u << s), l3 = l2 + (1u << s);
      uint32_t g0 = (uint32_t)(base + l0), g2 = (uint32_t)(base + l2);
      uint32_t tb = twiddle(tv, s + 1, g0);
      uint32_t ta0 = twiddle(tv, s, g0), ta2 = twiddle(tv, s, g2);
      uint32_t v0 = sm[l0], v1 = sm[l1], v2 = sm[l2], v3 = sm[l3];
      if (INV) {
        ibutterfly(v0, v1, ta0); ibutterfly(v2, v3, ta2);
        ibutterfly(v0, v2, tb); ibutterfly(v1, v3, tb);
      } else {
        butterfly(v0, v2, tb); butterfly(v1, v3, tb);
        butterfly(v0, v1, ta0); butterfly(v2, v3, ta2);
      }
      sm[l0] = v0; sm[l1] = v1; sm[l2] = v2; sm[l3] = v3;
    }
    __syncthreads();
  }
}

// Low pass: grid (n_blocks, n_cols). Loads block blockIdx.x of 2^block_bits words
// (a source column holding only 2^src_valid_bits words is zero-extended), applies
// layers [0, block_bits) and an optional scale, stores to dst.
template <bool INV>
__global__ void k_fft_low(const uint32_t* __restrict__ src, uint64_t src_stride, uint32_t src_valid_bits,
                          uint32_t* dst, uint64_t dst_stride, uint32_t block_bits, TwiddleView tv,
                          uint32_t scale) {
  extern __shared__ uint32_t sm[];
  const uint32_t n = 1u << block_bits;
  const uint64_t base = (uint64_t)blockIdx.x << block_bits;
  const uint32_t* s = src + blockIdx.y * src_stride;
  const uint32_t valid = src_valid_bits >= block_bits ? n : (1u << src_valid_bits);
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sm[i] = i < valid ? s[base + i] : 0u;
  __syncthreads();
  low_layers<INV>(sm, block_bits, base, tv, 0, block_bits);
  uint32_t* d = dst + blockIdx.y * dst_stride;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    uint32_t v = sm[i];
    if (scale) v = mmul(v, scale);
    d[base + i] = v;
  }
}

// High-pass shared layout: sm[m * T + t] is global index m*2^b + g*T + t.
// Applies layers [s_lo, s_hi) (global s >= b) over rows [0, 2^(row_bits)).
template <bool INV>
__device__ void high_layers(uint32_t* sm, uint32_t row_bits, uint32_t b, const TwiddleView& tv,
                            uint32_t s_lo, uint32_t s_hi) {
  const uint32_t rows = 1u << row_bits;
  uint32_t nl = s_hi - s_lo;
  if (nl & 1) {
    uint32_t s = INV ? s_lo : s_hi - 1;
    uint32_t r = s - b;  // row distance 2^r
    for (uint32_t q = threadIdx.x; q < (rows / 2) * HIGH_T; q += blockDim.x) {
      uint32_t t = q & (HIGH_T - 1), p = q >> HIGH_T_BITS;
      uint32_t m0 = ((p >> r) << (r + 1)) | (p & ((1u << r) - 1));
      uint32_t m1 = m0 + (1u << r);
      uint32_t tw = tv.line(s, m0 >> (r + 1));
      uint32_t a = sm[m0 * HIGH_T + t], c = sm[m1 * HIGH_T + t];
      if (INV) ibutterfly(a, c, tw); else butterfly(a, c, tw);
      sm[m0 * HIGH_T + t] = a; sm[m1 * HIGH_T + t] = c;
    }
    __syncthreads();
    if (INV) s_lo += 1; else s_hi -= 1;
    nl -= 1;
  }
  for (uint32_t k = 0; k < nl / 2; ++k) {
    uint32_t s = INV ? s_lo + 2 * k : s_hi - 2 - 2 * k;
    uint32_t r = s - b;
    for (uint32_t q = threadIdx.x; q < (rows / 4) * HIGH_T; q += blockDim.x) {
      uint32_t t = q & (HIGH_T - 1), p = q >> HIGH_T_BITS;
      uint32_t m0 = ((p >> r) << (r + 2)) | (p & ((1u << r) - 1));
      uint32_t m1 = m0 + (1u << r), m2 = m0 + (2u << r), m3 = m2 + (1u << r);
      uint32_t tb = tv.line(s + 1, m0 >> (r + 2));
      uint32_t ta0 = tv.line(s, m0 >> (r + 1)), ta2 = tv.line(s, m2 >> (r + 1));
      uint32_t v0 = sm[m0 * HIGH_T + t], v1 = sm[m1 * HIGH_T + t], v2 = sm[m2 * HIGH_T + t], v3 = sm[m3 * HIGH_T + t];
      if (INV) {
        ibutterfly(v0, v1, ta0); ibutterfly(v2, v3, ta2);
        ibutterfly(v0, v2, tb); ibutterfly(v1, v3, tb);
      } else {
        butterfly(v0, v2, tb); butterfly(v1, v3, tb);
        butterfly(v0, v1, ta0); butterfly(v2, v3, ta2);
      }
      sm[m0 * HIGH_T + t] = v0; sm[m1 * HIGH_T + t] = v1; sm[m2 * HIGH_T + t] = v2; sm[m3 * HIGH_T + t] = v3;
    }
    __syncthreads();
  }
}

struct HighParams {
  const uint32_t* src; uint64_t src_stride; uint32_t src_log;  // 2^(src_log - b) rows valid
  uint32_t b;
  // inverse phase (optional): layers [b, src_log), then scale, then store to coef
  int do_inverse; TwiddleView itv; uint32_t scale; uint32_t* coef; uint64_t coef_stride;
  // forward phase (optional): domain out_log >= src_log, rows beyond src rows are
  // duplicated when out_log == src_log + 1 (top layer skipped) and zero otherwise.
  int do_forward; TwiddleView ftv; uint32_t out_log; uint32_t* out; uint64_t out_stride;
};

// Grid (2^b / T groups, n_cols).
__global__ void k_fft_high(HighParams p) {
  extern __shared__ uint32_t sm[];
  const uint32_t g = blockIdx.x, col = blockIdx.y;
  const uint32_t in_rows = 1u << (p.src_log - p.b);
  const uint32_t* s = p.src + col * p.src_stride + g * HIGH_T;
  for (uint32_t i = threadIdx.x; i < in_rows * HIGH_T; i += blockDim.x) {
    uint32_t m = i >> HIGH_T_BITS, t = i & (HIGH_T - 1);
    sm[i] = s[((uint64_t)m << p.b) + t];
  }
  __syncthreads();
  if (p.do_inverse) {
    high_layers<true>(sm, p.src_log - p.b, p.b, p.itv, p.b, p.src_log);
    if (p.scale) {
      for (uint32_t i = threadIdx.x; i < in_rows * HIGH_T; i += blockDim.x) sm[i] = mmul(sm[i], p.scale);
      __syncthreads();
    }
    if (p.coef) {
      uint32_t* c = p.coef + col * p.coef_stride + g * HIGH_T;
      for (uint32_t i = threadIdx.x; i < in_rows * HIGH_T; i += blockDim.x) {
        uint32_t m = i >> HIGH_T_BITS, t = i & (HIGH_T - 1);
        c[((uint64_t)m << p.b) + t] = sm[i];
      }
    }
  }
  if (p.do_forward) {
    const uint32_t out_rows = 1u << (p.out_log - p.b);
    uint32_t s_hi = p.out_log;
    if (p.out_log == p.src_log + 1) {
      // The top layer pairs each value with a zero: it duplicates the lower half.
      for (uint32_t i = threadIdx.x; i < in_rows * HIGH_T; i += blockDim.x) sm[in_rows * HIGH_T + i] = sm[i];
      s_hi = p.src_log;
    } else {
      for (uint32_t i = in_rows * HIGH_T + threadIdx.x; i < out_rows * HIGH_T; i += blockDim.x) sm[i] = 0;
    }
    __syncthreads();
    high_layers<false>(sm, p.out_log - p.b, p.b, p.ftv, p.b, s_hi);
    uint32_t* o = p.out + col * p.out_stride + g * HIGH_T;
    for (uint32_t i = threadIdx.x; i < out_rows * HIGH_T; i += blockDim.x) {
      uint32_t m = i >> HIGH_T_BITS, t = i & (HIGH_T - 1);
      o[((uint64_t)m << p.b) + t] = sm[i];
    }
  } else if (!p.coef) {
    // pure forward/inverse in place without extension: store back to src layout
    uint32_t* o = p.out + col * p.out_stride + g * HIGH_T;
    for (uint32_t i = threadIdx.x; i < in_rows * HIGH_T; i += blockDim.x) {
      uint32_t m = i >> HIGH_T_BITS, t = i & (HIGH_T - 1);
      o[((uint64_t)m << p.b) + t] = sm[i];
    }
  }
}

// Entries 2^R .. 2^(R+1) of tw and itw are the doubled copies (tw2, itw2).
__global__ void k_build_tower(PointTable pts, uint32_t R, uint32_t* tw, uint32_t* itw) {
  // Entry e < 2^R - 1 belongs to layer k with offset 2^R - 2^(R-k).
  uint64_t total = 1ull << R;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    if (e == total - 1) { tw[e] = 1; itw[e] = 1; tw[total + e] = 2; itw[total + e] = 2; continue; }
    // k = number of leading ones of e in R bits
    uint32_t k = 0;
    while ((e >> (R - 1 - k)) & 1) ++k;
    uint64_t off = total - (total >> k);
    uint32_t i = (uint32_t)(e - off);
    uint32_t len_log = R - 1 - k;  // layer has 2^len_log entries
    Coset c = coset_half_odds(R - k);
    uint32_t nat = bitrev(i, len_log);
    uint32_t x = pts.at(c.index_at(nat)).x;
    const uint32_t ix = minv(x);
    tw[e] = x;
    itw[e] = ix;
    tw[total + e] = 2 * x;
    itw[total + e] = 2 * ix;
  }
}


// ---------------------------------------------------------------------------
// Radix-16 register kernels (domains 2^16 .. 2^22).
// ---------------------------------------------------------------------------
using fft16::radix16;
using fft16::radix16_dyn;
using fft16::spread;
using fft16::swz;

constexpr uint32_t B12 = 12;  // low pass: blocks of 4096 words, 256 threads x 16

template <uint32_t WA, uint32_t WB>
__device__ __forceinline__ void exchange12(uint32_t* sm, uint32_t (&x)[16], uint32_t ia, uint32_t ib) {
  const uint32_t a = swz(ia);
#pragma unroll
  for (int k = 0; k < 16; ++k) sm[a ^ swz((uint32_t)k << WA)] = x[k];
  __syncthreads();
  const uint32_t b = swz(ib);
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = sm[b ^ swz((uint32_t)k << WB)];
}

// Layers 0..11 of blocks of 4096 words. Forward: windows [8,12) -> [4,8) -> [0,4);
// inverse: the reverse, then the optional scale.
// With TMA (forward only) the block leaves through shared memory: each thread writes its 16 words
// as four 16-byte vectors into the 128-byte swizzled layout of `out_map` (rows of 32 words, the
// 16-byte chunk c of row r at chunk c ^ (r & 7), so that the eight lanes of each vector phase hit
// distinct banks), and one thread stores the block with a tensor copy. The plain path's 16-byte
// global stores are 64 bytes apart across a warp: four times the memory wavefronts of a
// contiguous store. (The inverse pass's 16-byte loads of the same pattern staged through shared
// memory by coalesced asynchronous copies measured slower: 497 -> 510 us for 100 columns of 2^20.)
template <bool INV, bool TMA>
__global__ void __launch_bounds__(256) k_fft_low12(const uint32_t* __restrict__ src, uint64_t ss, uint32_t* dst,
                                                   uint64_t ds, TwiddleView tv, uint32_t scale,
                                                   const __grid_constant__ CUtensorMap out_map) {
  static_assert(!(INV && TMA), "the tensor store serves the forward pass");
  __shared__ __align__(1024) uint32_t sm[1 << B12];
  const uint32_t th = threadIdx.x;
  const uint64_t blk = (uint64_t)blockIdx.x << B12;
  const uint32_t* s = src + blockIdx.y * ss + blk;
  uint32_t* d = dst + blockIdx.y * ds + blk;
  const uint32_t ib2 = th;                            // elements ib2 + 256 k
  const uint32_t ib1 = ((th >> 4) << 8) | (th & 15);  // elements ib1 + 16 k
  const uint32_t ib0 = th << 4;                       // elements ib0 + k
  uint32_t x[16];
  if (!INV) {
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = __ldg(s + ib2 + 256 * k);
    radix16<false, 0, 4>(x, tv, 0, 8, blk + ib2);
    exchange12<8, 4>(sm, x, ib2, ib1);
    radix16<false, 0, 4>(x, tv, 0, 4, blk + ib1);
    __syncthreads();
    exchange12<4, 0>(sm, x, ib1, ib0);
    radix16<false, 0, 4>(x, tv, 0, 0, blk + ib0);
    // The swizzled layout assumes a 1024-byte aligned buffer (the alignment declared above); a
    // buffer placed otherwise takes the plain stores.
    if (TMA && (((uint32_t)__cvta_generic_to_shared(sm)) & 1023u) == 0) {
      __syncthreads();  // every thread has read its words of the last exchange
      // Words ib0 .. ib0 + 15: row th >> 1, 16-byte chunks 4 * (th & 1) + q.
      const uint32_t r = th >> 1;
      uint8_t* row = reinterpret_cast<uint8_t*>(sm) + 128 * r;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        *reinterpret_cast<uint4*>(row + (((4 * (th & 1) + q) ^ (r & 7)) << 4)) =
            make_uint4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
      // The tensor copy reads shared memory through the async proxy.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (th == 0) {
        asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
                     ::"l"(reinterpret_cast<uint64_t>(&out_map)), "r"(0), "r"(blockIdx.x << (B12 - 5)),
                       "r"(blockIdx.y), "r"((uint32_t)__cvta_generic_to_shared(sm))
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // Shared memory stays allocated until the copy has read it.
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      }
    } else {
      uint4* o = reinterpret_cast<uint4*>(d + ib0);
#pragma unroll
      for (int q = 0; q < 4; ++q) o[q] = make_uint4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
    }
  } else {
    const uint4* in = reinterpret_cast<const uint4*>(s + ib0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint4 v = __ldg(in + q);
      x[4 * q] = v.x; x[4 * q + 1] = v.y; x[4 * q + 2] = v.z; x[4 * q + 3] = v.w;
    }
    radix16<true, 0, 4>(x, tv, 0, 0, blk + ib0);
    exchange12<0, 4>(sm, x, ib0, ib1);
    radix16<true, 0, 4>(x, tv, 0, 4, blk + ib1);
    __syncthreads();
    exchange12<4, 8>(sm, x, ib1, ib2);
    radix16<true, 0, 4>(x, tv, 0, 8, blk + ib2);
#pragma unroll
    for (int k = 0; k < 16; ++k) d[ib2 + 256 * k] = scale ? mmul(x[k], scale) : x[k];
  }
}

struct High16Params {
  const uint32_t* src; uint64_t ss; uint32_t rows_in;  // 2^rows_in rows of 16 words per tile are loaded
  int do_inverse; TwiddleView itv; uint32_t scale; uint32_t* coef; uint64_t cs;
  int do_forward; TwiddleView ftv; uint32_t rows_out; uint32_t fwd_layers; int dup;
  uint32_t* out; uint64_t os;
};

// Tile of the high pass: 2^rows rows x 16 adjacent low indices; tile element
// i = (m << 4) | t is transform index (m << 12) + g*16 + t. A window stage gives
// thread (q, t) the 16 rows spread(q, W0) + (k << W0).
//
// SRC: 0 = shared memory, 1 = global source rows (rows beyond the source are
// duplicates when DUP, zeros otherwise); DST: 0 = shared memory, 1 = global
// output, 2 = scale, store coefficients to global and to shared memory (also at
// row + 2^rows_src when DUP).
struct HighIo {
  const uint32_t* src; uint32_t src_rows;  // source rows (log)
  uint32_t* out;                           // global destination tile base (column + g*16)
  uint32_t scale;
  int dup;
};

template <bool INV, int W0, int NL, int SRC, int DST>
__device__ __noinline__ void high_stage(uint32_t* sm, const TwiddleView tv, uint32_t rows, const HighIo io) {
  const uint32_t th = threadIdx.x;
  if (th < (1u << rows)) {
    const uint32_t t = th & 15, q = th >> 4;
    const uint32_t mb = spread(q, W0);
    const uint32_t a = swz((mb << 4) | t);
    uint32_t x[16];
    if (SRC == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) x[k] = sm[a ^ swz((uint32_t)k << (W0 + 4))];
    } else {
      const uint32_t src_n = 1u << io.src_rows;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        uint32_t m = mb + ((uint32_t)k << W0);
        uint32_t v = 0;
        if (m < src_n) v = __ldg(io.src + ((uint64_t)m << B12) + t);
        else if (io.dup) v = __ldg(io.src + ((uint64_t)(m - src_n) << B12) + t);
        x[k] = v;
      }
    }
    radix16<INV, 0, NL>(x, tv, B12, W0, mb);
    if (DST == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) sm[a ^ swz((uint32_t)k << (W0 + 4))] = x[k];
    } else if (DST == 1) {
#pragma unroll
      for (int k = 0; k < 16; ++k) io.out[((uint64_t)(mb + ((uint32_t)k << W0)) << B12) + t] = x[k];
    } else {
      const uint32_t dup_off = swz((1u << rows) << 4);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        uint32_t v = io.scale ? mmul(x[k], io.scale) : x[k];
        io.out[((uint64_t)(mb + ((uint32_t)k << W0)) << B12) + t] = v;
        uint32_t pos = a ^ swz((uint32_t)k << (W0 + 4));
        sm[pos] = v;
        if (io.dup) sm[pos ^ dup_off] = v;
      }
    }
  }
  __syncthreads();
}

template <bool INV, int W0, int NL>
__device__ __forceinline__ void high_stage_io(uint32_t* sm, const TwiddleView& tv, uint32_t rows, const HighIo& io,
                                              int src, int dst) {
  if (src == 0 && dst == 0) high_stage<INV, W0, NL, 0, 0>(sm, tv, rows, io);
  else if (src == 0 && dst == 1) high_stage<INV, W0, NL, 0, 1>(sm, tv, rows, io);
  else if (src == 0 && dst == 2) high_stage<INV, W0, NL, 0, 2>(sm, tv, rows, io);
  else if (src == 1 && dst == 0) high_stage<INV, W0, NL, 1, 0>(sm, tv, rows, io);
  else if (src == 1 && dst == 1) high_stage<INV, W0, NL, 1, 1>(sm, tv, rows, io);
  else high_stage<INV, W0, NL, 1, 2>(sm, tv, rows, io);
}

// Runtime (w0, nl) -> compiled stage. Windows used: w0 in [0, 6], nl = 4 except
// the short stage at w0 = 0.
template <bool INV>
__device__ void high_stage_dyn(uint32_t* sm, const TwiddleView& tv, uint32_t rows, const HighIo& io, uint32_t w0,
                               uint32_t nl, int src, int dst) {
  if (nl == 4) {
    switch (w0) {
      case 0: high_stage_io<INV, 0, 4>(sm, tv, rows, io, src, dst); break;
      case 1: high_stage_io<INV, 1, 4>(sm, tv, rows, io, src, dst); break;
      case 2: high_stage_io<INV, 2, 4>(sm, tv, rows, io, src, dst); break;
      case 3: high_stage_io<INV, 3, 4>(sm, tv, rows, io, src, dst); break;
      case 4: high_stage_io<INV, 4, 4>(sm, tv, rows, io, src, dst); break;
      case 5: high_stage_io<INV, 5, 4>(sm, tv, rows, io, src, dst); break;
      default: high_stage_io<INV, 6, 4>(sm, tv, rows, io, src, dst); break;
    }
  } else if (nl == 3) {
    high_stage_io<INV, 0, 3>(sm, tv, rows, io, src, dst);
  } else if (nl == 2) {
    high_stage_io<INV, 0, 2>(sm, tv, rows, io, src, dst);
  } else {
    high_stage_io<INV, 0, 1>(sm, tv, rows, io, src, dst);
  }
}

// Grid (256 tiles of 16 adjacent low indices, n_cols); blockDim = 2^max(rows) threads.
// Phases: inverse layers [12, 12 + rows_in) then 1/n scale and coefficient store;
// forward layers of the extended tile. Every stage keeps its 16 elements in
// registers; only the first stage reads global memory and only the last writes it.
// Tiles of up to 512 threads are built for three resident CTAs per SM (42 registers a
// thread), the 1024-thread tile for one: on 2^20 x 100 columns the forward pass measured
// 1.686 ms against 1.713 ms with a single 1024-thread build, bit-identical output.
template <int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_fft_high16(High16Params p) {
  extern __shared__ uint32_t sm[];
  const uint32_t g = blockIdx.x, col = blockIdx.y;
  HighIo io;
  io.src = p.src + col * p.ss + g * 16;
  io.src_rows = p.rows_in;
  io.scale = p.scale;
  io.dup = p.dup;
  if (p.do_inverse) {
    const uint32_t RL = p.rows_in, rem = RL & 3;
    const uint32_t n_st = (RL >> 2) + (rem ? 1 : 0);
    io.out = p.coef + col * p.cs + g * 16;
    uint32_t w0 = 0;
    for (uint32_t st = 0; st < n_st; ++st) {
      const uint32_t nl = (st == 0 && rem) ? rem : 4;
      const int src = st == 0 ? 1 : 0;
      const int dst = st + 1 == n_st ? 2 : 0;
      // a pure inverse transform (no forward phase) needs no shared copy at the end
      high_stage_dyn<true>(sm, p.itv, RL, io, w0, nl, src, dst);
      w0 += nl;
    }
  }
  if (p.do_forward) {
    const uint32_t RL = p.fwd_layers, rem = RL & 3;
    const uint32_t n_st = (RL >> 2) + (rem ? 1 : 0);
    io.out = p.out + col * p.os + g * 16;
    if (p.do_inverse && !p.dup && p.rows_out > p.rows_in) {
      // zero extension after an inverse phase: rows beyond the coefficients are zero
      for (uint32_t i = (16u << p.rows_in) + threadIdx.x; i < (16u << p.rows_out); i += blockDim.x) sm[swz(i)] = 0;
      __syncthreads();
    }
    int w0 = (int)RL - 4;
    for (uint32_t st = 0; st < n_st; ++st) {
      const bool short_st = rem && st + 1 == n_st;
      const uint32_t nl = short_st ? rem : 4;
      const uint32_t ww = short_st ? 0 : (uint32_t)w0;
      const int src = (st == 0 && !p.do_inverse) ? 1 : 0;
      const int dst = st + 1 == n_st ? 1 : 0;
      high_stage_dyn<false>(sm, p.ftv, p.rows_out, io, ww, nl, src, dst);
      w0 -= 4;
    }
  }
}

// Windows of the high pass over R row bits: an optional short window [0, R % 4) first, then
// full 4-bit windows. Window i covers row bits [win_w0(i), win_w0(i) + 4) of which it applies
// win_nl(i) layers.
template <int R>
__host__ __device__ constexpr int win_count() { return R / 4 + (R % 4 ? 1 : 0); }
template <int R>
__host__ __device__ constexpr uint32_t win_w0(int i) { return R % 4 ? (i == 0 ? 0u : (uint32_t)(R % 4 + 4 * (i - 1))) : 4u * i; }
template <int R>
__host__ __device__ constexpr uint32_t win_nl(int i) { return (R % 4 && i == 0) ? (uint32_t)(R % 4) : 4u; }

// Interpolation's high layers fused with the blow-up-2 extension, for columns of 2^(12 + R)
// words (R = 5..10): one CTA of 2^R threads per tile of 2^R rows x 16 adjacent low indices
// (row m, low index t is transform index (m << 12) + g * 16 + t), each thread 16 rows of one low
// index per window. The inverse windows run bottom-up; the last one, which covers the top row
// bits [R - 4, R), also scales by 1/n, stores the coefficients, and applies the extension's
// forward window over the same row bits to two copies of its 16 coefficients: the extension's
// top layer pairs every coefficient with a zero row, so it only copies row m to m + 2^R (the
// reference skips it the same way, src/prover/poly/circle/transforms.zig:132-147), and the two
// copies then differ only in their twiddles. The remaining forward windows run top-down on both
// halves. One shared-memory exchange and barrier per window boundary; the generic kernel pays a
// zero fill, a 9th layer of butterflies on zeros and three more exchanges on 2^20 -> 2^21.
template <int R>
__global__ void __launch_bounds__(1 << R, R <= 8 ? (1024 >> R) : 1) k_fft_high16_lde1(High16Params p) {
  static_assert(R >= 5 && R <= 10, "tile rows");
  constexpr int NW = win_count<R>();
  extern __shared__ uint32_t sm[];  // 16 << (R + 1) words: both halves of the extended tile
  const uint32_t th = threadIdx.x, t = th & 15, q = th >> 4;
  const uint32_t g = blockIdx.x, col = blockIdx.y;
  // Row m of low index t is word (m << 12) + t past these (the tile's 16 low indices are adjacent).
  const uint32_t* src = p.src + col * p.ss + g * 16 + t;
  uint32_t* coef = p.coef + col * p.cs + g * 16 + t;
  uint32_t* out = p.out + col * p.os + g * 16 + t;
  const uint32_t hoff = swz((1u << R) << 4);  // shared position of row m + 2^R relative to row m
  uint32_t x[16], y[16];
#pragma unroll
  for (int i = 0; i < NW; ++i) {
    const uint32_t w0 = win_w0<R>(i), nl = win_nl<R>(i);
    const uint32_t mb = spread(q, w0);
    const uint32_t a = swz((mb << 4) | t);
    if (i == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) x[k] = __ldg(src + ((uint64_t)(mb + ((uint32_t)k << w0)) << B12));
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) x[k] = sm[a ^ swz((uint32_t)k << (w0 + 4))];
    }
    radix16_dyn<true>(x, p.itv, B12, w0, mb, nl);
    if (i + 1 < NW) {
#pragma unroll
      for (int k = 0; k < 16; ++k) sm[a ^ swz((uint32_t)k << (w0 + 4))] = x[k];
      __syncthreads();
    }
  }
  {
    constexpr uint32_t w0 = R - 4;
    const uint32_t mb = spread(q, w0);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t v = mmul(x[k], p.scale);
      coef[(uint64_t)(mb + ((uint32_t)k << w0)) << B12] = v;
      x[k] = v;
      y[k] = v;
    }
    radix16<false, 0, 4>(x, p.ftv, B12, w0, mb);
    radix16<false, 0, 4>(y, p.ftv, B12, w0, mb | (1u << R));
    const uint32_t a = swz((mb << 4) | t);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t pos = a ^ swz((uint32_t)k << (w0 + 4));
      sm[pos] = x[k];
      sm[pos ^ hoff] = y[k];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = NW - 2; i >= 0; --i) {
    const uint32_t w0 = win_w0<R>(i), nl = win_nl<R>(i);
    const uint32_t mb = spread(q, w0);
    const uint32_t a = swz((mb << 4) | t);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t pos = a ^ swz((uint32_t)k << (w0 + 4));
      x[k] = sm[pos];
      y[k] = sm[pos ^ hoff];
    }
    radix16_dyn<false>(x, p.ftv, B12, w0, mb, nl);
    radix16_dyn<false>(y, p.ftv, B12, w0, mb | (1u << R), nl);
    if (i > 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint32_t pos = a ^ swz((uint32_t)k << (w0 + 4));
        sm[pos] = x[k];
        sm[pos ^ hoff] = y[k];
      }
      __syncthreads();
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint64_t m = mb + ((uint32_t)k << w0);
        out[m << B12] = x[k];
        out[(m + (1u << R)) << B12] = y[k];
      }
    }
  }
}

inline uint32_t inv_pow2(uint32_t log) { return minv(1u << log); }

}  // namespace

TwiddleView DeviceTables::view(uint32_t domain_log, bool inverse) const {
  TwiddleView v;
  v.tower = inverse ? itw : tw;
  v.tower2 = inverse ? itw2 : tw2;
  v.root_log = tower_log;
  v.line_log = domain_log - 1;
  v.y0 = 0;
  if (domain_log <= 2) {
    // y of halfOdds(L)'s first point, from the host point table.
    static std::vector<PointM> host_pts = build_point_table();
    PointTable pt{host_pts.data()};
    Coset c = coset_half_odds(domain_log - 1);
    uint32_t y = pt.at(c.initial).y;
    v.y0 = inverse ? minv(y) : y;
  }
  return v;
}

cudaError_t build_twiddle_tower(DeviceTables& t, uint32_t root_log, cudaStream_t stream) {
  k_build_tower<<<1024, 256, 0, stream>>>(PointTable{t.points}, root_log, t.tw, t.itw); note_launch();
  t.tower_log = root_log;
  return cudaGetLastError();
}

static cudaError_t launch_low(const DeviceTables& t, bool inverse, uint32_t domain_log, uint32_t n_cols,
                              const uint32_t* src, uint64_t src_stride, uint32_t src_valid_log, uint32_t* dst,
                              uint64_t dst_stride, uint32_t scale, cudaStream_t stream) {
  uint32_t b = std::min(domain_log, LOW_BITS);
  dim3 grid(1u << (domain_log - b), n_cols);
  size_t smem = (size_t)4 << b;
  TwiddleView tv = t.view(domain_log, inverse);
  if (inverse)
    k_fft_low<true><<<grid, LOW_THREADS, smem, stream>>>(src, src_stride, src_valid_log, dst, dst_stride, b, tv, scale);
  else
    k_fft_low<false><<<grid, LOW_THREADS, smem, stream>>>(src, src_stride, src_valid_log, dst, dst_stride, b, tv, scale);
  note_launch();
  return cudaGetLastError();
}

static cudaError_t launch_high(const HighParams& p, uint32_t n_cols, cudaStream_t stream) {
  uint32_t rows_log = std::max(p.src_log, p.do_forward ? p.out_log : p.src_log) - p.b;
  size_t smem = ((size_t)HIGH_T * 4) << rows_log;
  static const bool attr_set = [] {  // once per process (thread-safe static initialisation)
    cudaFuncSetAttribute(k_fft_high, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    return true;
  }();
  (void)attr_set;
  dim3 grid((1u << p.b) / HIGH_T, n_cols);
  k_fft_high<<<grid, HIGH_THREADS, smem, stream>>>(p); note_launch();
  return cudaGetLastError();
}


// ---- radix-16 path launchers ----------------------------------------------
// The radix-16 kernels read and write 16-byte vectors: columns must start 16-byte aligned.
static bool aligned16(const void* p, uint64_t stride) { return ((uintptr_t)p & 15) == 0 && (stride & 3) == 0; }
static bool use16(uint32_t log_in, uint32_t log_out, const void* a, uint64_t sa, const void* b, uint64_t sb_) {
  return log_in >= 16 && log_out <= 22 && aligned16(a, sa) && aligned16(b, sb_);
}

// cuTensorMapEncodeTiled, looked up once through the runtime (null if the driver lacks it).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// The forward low pass's output as a tensor: rows of 32 words (128 bytes, the swizzle span),
// 2^(log-5) rows per column, n_cols columns `stride` words apart; a box is one 4096-word block
// (128 rows). The caller has checked 16-byte alignment of the base and the stride.
static bool low12_store_map(CUtensorMap* m, uint32_t* dst, uint32_t log, uint32_t n_cols, uint64_t stride) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc || log < B12) return false;
  const cuuint64_t dims[3] = {32, 1ull << (log - 5), n_cols};
  const cuuint64_t strides[2] = {128, stride * 4};
  const cuuint32_t box[3] = {32, 1u << (B12 - 5), 1};
  const cuuint32_t elem[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, dst, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static cudaError_t launch_low12(const DeviceTables& t, bool inverse, uint32_t domain_log, uint32_t n_cols,
                                const uint32_t* src, uint64_t ss, uint32_t* dst, uint64_t ds, uint32_t scale,
                                cudaStream_t stream) {
  dim3 grid(1u << (domain_log - B12), n_cols);
  TwiddleView tv = t.view(domain_log, inverse);
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if (inverse) k_fft_low12<true, false><<<grid, 256, 0, stream>>>(src, ss, dst, ds, tv, scale, map);
  else if (low12_store_map(&map, dst, domain_log, n_cols, ds))
    k_fft_low12<false, true><<<grid, 256, 0, stream>>>(src, ss, dst, ds, tv, scale, map);
  else k_fft_low12<false, false><<<grid, 256, 0, stream>>>(src, ss, dst, ds, tv, scale, map);
  note_launch();
  return cudaGetLastError();
}

static cudaError_t launch_high16(const High16Params& p, uint32_t n_cols, cudaStream_t stream) {
  uint32_t rows = p.do_forward ? std::max(p.rows_in, p.rows_out) : p.rows_in;
  size_t smem = (size_t)64 << rows;
  static const bool attr_set = [] {  // once per process (thread-safe static initialisation)
    cudaFuncSetAttribute(k_fft_high16<512, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 32 * 1024);
    cudaFuncSetAttribute(k_fft_high16<1024, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    return true;
  }();
  (void)attr_set;
  dim3 grid(1u << (B12 - 4), n_cols);
  if (rows <= 9) k_fft_high16<512, 3><<<grid, 1u << rows, smem, stream>>>(p);
  else k_fft_high16<1024, 1><<<grid, 1u << rows, smem, stream>>>(p);
  note_launch();
  return cudaGetLastError();
}

template <int R>
static cudaError_t launch_lde1_rows(const High16Params& p, uint32_t n_cols, cudaStream_t stream) {
  const size_t smem = (size_t)64 << (R + 1);
  static const bool attr_set = [] {  // once per process (thread-safe static initialisation)
    cudaFuncSetAttribute(k_fft_high16_lde1<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)((size_t)64 << (R + 1)));
    return true;
  }();
  (void)attr_set;
  k_fft_high16_lde1<R><<<dim3(1u << (B12 - 4), n_cols), 1u << R, smem, stream>>>(p);
  note_launch();
  return cudaGetLastError();
}

// The fused interpolate + blow-up-2 extension high pass (rows_in in [5, 10]).
static cudaError_t launch_high16_lde1(const High16Params& p, uint32_t n_cols, cudaStream_t stream) {
  switch (p.rows_in) {
    case 5: return launch_lde1_rows<5>(p, n_cols, stream);
    case 6: return launch_lde1_rows<6>(p, n_cols, stream);
    case 7: return launch_lde1_rows<7>(p, n_cols, stream);
    case 8: return launch_lde1_rows<8>(p, n_cols, stream);
    case 9: return launch_lde1_rows<9>(p, n_cols, stream);
    default: return launch_lde1_rows<10>(p, n_cols, stream);
  }
}

cudaError_t fft_columns(const DeviceTables& t, bool inverse, uint32_t log_size, uint32_t n_cols, uint32_t* cols,
                        uint64_t stride, cudaStream_t stream) {
  if (n_cols == 0) return cudaSuccess;
  if (use16(log_size, log_size, cols, stride, cols, stride)) {
    High16Params p{};
    p.src = cols; p.ss = stride; p.rows_in = log_size - B12;
    if (inverse) {
      cudaError_t e = launch_low12(t, true, log_size, n_cols, cols, stride, cols, stride, 0, stream);
      if (e != cudaSuccess) return e;
      p.do_inverse = 1; p.itv = t.view(log_size, true); p.scale = inv_pow2(log_size); p.coef = cols; p.cs = stride;
      return launch_high16(p, n_cols, stream);
    }
    p.do_forward = 1; p.ftv = t.view(log_size, false); p.rows_out = p.rows_in; p.fwd_layers = p.rows_in;
    p.out = cols; p.os = stride;
    cudaError_t e = launch_high16(p, n_cols, stream);
    if (e != cudaSuccess) return e;
    return launch_low12(t, false, log_size, n_cols, cols, stride, cols, stride, 0, stream);
  }
  const uint32_t b = std::min(log_size, LOW_BITS);
  const uint32_t scale = inverse ? inv_pow2(log_size) : 0;
  if (log_size <= b)
    return launch_low(t, inverse, log_size, n_cols, cols, stride, log_size, cols, stride, scale, stream);
  HighParams p{};
  p.src = cols; p.src_stride = stride; p.src_log = log_size; p.b = b;
  p.out = cols; p.out_stride = stride;
  if (inverse) {
    cudaError_t e = launch_low(t, true, log_size, n_cols, cols, stride, log_size, cols, stride, 0, stream);
    if (e != cudaSuccess) return e;
    p.do_inverse = 1; p.itv = t.view(log_size, true); p.scale = scale; p.coef = cols; p.coef_stride = stride;
    return launch_high(p, n_cols, stream);
  }
  p.do_forward = 1; p.ftv = t.view(log_size, false); p.out_log = log_size;
  // out_log == src_log: no duplication, all layers [b, log_size)
  cudaError_t e = launch_high(p, n_cols, stream);
  if (e != cudaSuccess) return e;
  return launch_low(t, false, log_size, n_cols, cols, stride, log_size, cols, stride, 0, stream);
}

cudaError_t extend(const DeviceTables& t, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                   const uint32_t* coeffs, uint64_t co_stride, uint32_t* lde, uint64_t lde_stride,
                   cudaStream_t stream) {
  if (n_cols == 0) return cudaSuccess;
  const uint32_t out_log = log_size + log_blowup;
  if (use16(log_size, out_log, coeffs, co_stride, lde, lde_stride)) {
    High16Params p{};
    p.src = coeffs; p.ss = co_stride; p.rows_in = log_size - B12;
    p.do_forward = 1; p.ftv = t.view(out_log, false); p.rows_out = out_log - B12;
    p.dup = log_blowup == 1; p.fwd_layers = p.dup ? p.rows_in : p.rows_out;
    p.out = lde; p.os = lde_stride;
    cudaError_t e = launch_high16(p, n_cols, stream);
    if (e != cudaSuccess) return e;
    return launch_low12(t, false, out_log, n_cols, lde, lde_stride, lde, lde_stride, 0, stream);
  }
  const uint32_t b = std::min(out_log, LOW_BITS);
  if (out_log <= b)  // single low pass with zero extension
    return launch_low(t, false, out_log, n_cols, coeffs, co_stride, log_size, lde, lde_stride, 0, stream);
  HighParams p{};
  p.b = b;
  if (log_size >= b) {
    p.src = coeffs; p.src_stride = co_stride; p.src_log = log_size;
  } else {
    // Tiny source: zero-extend to 2^b first through a low pass of the identity (no layers).
    p.src = coeffs; p.src_stride = co_stride; p.src_log = log_size;
  }
  if (log_size < b) {
    // Route: treat the coefficient column as rows of the strided view with only
    // the first 2^log_size words non-zero. Build a zero-extended copy in lde.
    // lde[0 .. 2^b) = coeffs, rest zero; then forward high + low on lde.
    cudaError_t e = cudaMemset2DAsync(lde, lde_stride * 4, 0, (size_t)4 << out_log, n_cols, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemcpy2DAsync(lde, lde_stride * 4, coeffs, co_stride * 4, (size_t)4 << log_size, n_cols,
                          cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return e;
    return fft_columns(t, false, out_log, n_cols, lde, lde_stride, stream);
  }
  p.do_forward = 1; p.ftv = t.view(out_log, false); p.out_log = out_log; p.out = lde; p.out_stride = lde_stride;
  cudaError_t e = launch_high(p, n_cols, stream);
  if (e != cudaSuccess) return e;
  return launch_low(t, false, out_log, n_cols, lde, lde_stride, out_log, lde, lde_stride, 0, stream);
}

cudaError_t interpolate_extend(const DeviceTables& t, uint32_t log_size, uint32_t log_blowup, uint32_t n_cols,
                               const uint32_t* evals, uint64_t ev_stride, uint32_t* coeffs, uint64_t co_stride,
                               uint32_t* lde, uint64_t lde_stride, cudaStream_t stream) {
  if (n_cols == 0) return cudaSuccess;
  const uint32_t out_log = log_size + log_blowup;
  if (use16(log_size, out_log, evals, ev_stride, lde, lde_stride) && aligned16(coeffs, co_stride)) {
    // Variant 0: the fused high pass (blow-up 2, 2^17 .. 2^22); variant 1: the generic one.
    auto chain = [&](int variant) -> cudaError_t {
      cudaError_t e = launch_low12(t, true, log_size, n_cols, evals, ev_stride, coeffs, co_stride, 0, stream);
      if (e != cudaSuccess) return e;
      High16Params p{};
      p.src = coeffs; p.ss = co_stride; p.rows_in = log_size - B12;
      p.do_inverse = 1; p.itv = t.view(log_size, true); p.scale = inv_pow2(log_size); p.coef = coeffs; p.cs = co_stride;
      p.do_forward = 1; p.ftv = t.view(out_log, false); p.rows_out = out_log - B12;
      p.dup = log_blowup == 1; p.fwd_layers = p.dup ? p.rows_in : p.rows_out;
      p.out = lde; p.os = lde_stride;
      e = log_blowup == 1 && p.rows_in >= 5 && variant == 0 ? launch_high16_lde1(p, n_cols, stream)
                                                             : launch_high16(p, n_cols, stream);
      if (e != cudaSuccess) return e;
      return launch_low12(t, false, out_log, n_cols, lde, lde_stride, lde, lde_stride, 0, stream);
    };
    const bool fusable = log_blowup == 1 && log_size - B12 >= 5;
    // The chain reads evals only, so it can run again for timing unless evals is also an output.
    const bool rerunnable = evals != coeffs && evals != lde;
    return tuned_run(TUNE_LDE1, log_size, n_cols, fusable ? 2 : 1, rerunnable, stream, chain);
  }
  const uint32_t b = std::min(log_size, LOW_BITS);
  if (log_size <= b || out_log > LOW_BITS + 12) {
    // Small domains (or unsupported fused sizes): separate transforms.
    if (coeffs != evals) {
      cudaError_t e = cudaMemcpy2DAsync(coeffs, co_stride * 4, evals, ev_stride * 4, (size_t)4 << log_size, n_cols,
                                        cudaMemcpyDeviceToDevice, stream);
      if (e != cudaSuccess) return e;
    }
    cudaError_t e = fft_columns(t, true, log_size, n_cols, coeffs, co_stride, stream);
    if (e != cudaSuccess) return e;
    return extend(t, log_size, log_blowup, n_cols, coeffs, co_stride, lde, lde_stride, stream);
  }
  // 1. inverse low layers: evals -> coeffs (partial)
  cudaError_t e = launch_low(t, true, log_size, n_cols, evals, ev_stride, log_size, coeffs, co_stride, 0, stream);
  if (e != cudaSuccess) return e;
  // 2. inverse high layers + scale -> coeffs; extension + forward high layers -> lde
  HighParams p{};
  p.src = coeffs; p.src_stride = co_stride; p.src_log = log_size; p.b = b;
  p.do_inverse = 1; p.itv = t.view(log_size, true); p.scale = inv_pow2(log_size); p.coef = coeffs; p.coef_stride = co_stride;
  p.do_forward = 1; p.ftv = t.view(out_log, false); p.out_log = out_log; p.out = lde; p.out_stride = lde_stride;
  e = launch_high(p, n_cols, stream);
  if (e != cudaSuccess) return e;
  // 3. forward low layers on lde in place
  return launch_low(t, false, out_log, n_cols, lde, lde_stride, out_log, lde, lde_stride, 0, stream);
}

}  // namespace sb
