// Montgomery batch inversion of M31 / CM31 / QM31 columns (the backend
// batchInverse, src/backend/field_ops.zig:9-15; algorithm of batchInverseClassic,
// src/core/fields/mod.zig:178-200: prefix products, one inversion, backward pass).
//
// A CTA of 256 threads owns a tile of 256 * K consecutive elements; thread t
// takes elements t, t + 256, ... so every load and store is coalesced. Each
// thread keeps its K inputs and prefix products in registers and inverts one
// product, so the field inversion (an exponentiation by p - 2) is amortised
// over K elements and HBM traffic is one read and one write per element.
#include "kernels.cuh"

namespace sb {

namespace {

constexpr int BI_THREADS = 256;

template <int DEG>
struct Elem;
template <>
struct Elem<1> {
  uint32_t v;
  static SB_HD Elem one() { return {1}; }
  SB_HD bool zero() const { return v == 0; }
  SB_HD Elem mul(const Elem& o) const { return {mmul(v, o.v)}; }
  SB_HD Elem inv() const { return {minv(v)}; }
  __device__ static Elem load(const uint32_t* s, uint64_t stride, uint64_t i) { return {s[i]}; }
  __device__ void store(uint32_t* d, uint64_t stride, uint64_t i) const { d[i] = v; }
};
template <>
struct Elem<2> {
  CM31 v;
  static SB_HD Elem one() { return {{1, 0}}; }
  SB_HD bool zero() const { return v.a == 0 && v.b == 0; }
  SB_HD Elem mul(const Elem& o) const { return {cmul(v, o.v)}; }
  SB_HD Elem inv() const { return {cinv(v)}; }
  __device__ static Elem load(const uint32_t* s, uint64_t stride, uint64_t i) { return {{s[i], s[stride + i]}}; }
  __device__ void store(uint32_t* d, uint64_t stride, uint64_t i) const {
    d[i] = v.a;
    d[stride + i] = v.b;
  }
};
template <>
struct Elem<4> {
  QM31 v;
  static SB_HD Elem one() { return {qone()}; }
  SB_HD bool zero() const { return qiszero(v); }
  SB_HD Elem mul(const Elem& o) const { return {qmul(v, o.v)}; }
  SB_HD Elem inv() const { return {qinv(v)}; }
  __device__ static Elem load(const uint32_t* s, uint64_t stride, uint64_t i) {
    return {qmake(s[i], s[stride + i], s[2 * stride + i], s[3 * stride + i])};
  }
  __device__ void store(uint32_t* d, uint64_t stride, uint64_t i) const {
    d[i] = v.c0.a;
    d[stride + i] = v.c0.b;
    d[2 * stride + i] = v.c1.a;
    d[3 * stride + i] = v.c1.b;
  }
};

template <int DEG, int K>
__global__ void __launch_bounds__(BI_THREADS) k_batch_inverse(uint64_t n, const uint32_t* src, uint64_t ss,
                                                              uint32_t* dst, uint64_t ds, uint32_t* zero_flag) {
  using E = Elem<DEG>;
  const uint64_t base = (uint64_t)blockIdx.x * BI_THREADS * K + threadIdx.x;
  E x[K], pre[K];
  E acc = E::one();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    uint64_t i = base + (uint64_t)j * BI_THREADS;
    x[j] = i < n ? E::load(src, ss, i) : E::one();  // padding with ones leaves the product unchanged
    acc = acc.mul(x[j]);
    pre[j] = acc;
  }
  if (acc.zero()) {
    atomicOr(zero_flag, 1u);
    return;
  }
  E cur = acc.inv();  // (x_0 ... x_{K-1})^-1
#pragma unroll
  for (int j = K - 1; j >= 1; --j) {
    E inv_j = pre[j - 1].mul(cur);
    cur = cur.mul(x[j]);
    uint64_t i = base + (uint64_t)j * BI_THREADS;
    if (i < n) inv_j.store(dst, ds, i);
  }
  if (base < n) cur.store(dst, ds, base);
}

template <int DEG, int K>
cudaError_t launch_bi(uint64_t n, const uint32_t* src, uint64_t ss, uint32_t* dst, uint64_t ds, uint32_t* flag,
                      cudaStream_t stream) {
  uint64_t tile = (uint64_t)BI_THREADS * K;
  uint64_t blocks = (n + tile - 1) / tile;
  if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
  k_batch_inverse<DEG, K><<<(unsigned)blocks, BI_THREADS, 0, stream>>>(n, src, ss, dst, ds, flag);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

cudaError_t batch_inverse(uint32_t degree, uint64_t n, const uint32_t* src, uint64_t src_stride, uint32_t* dst,
                          uint64_t dst_stride, uint32_t* zero_flag, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  switch (degree) {
    case 1: return launch_bi<1, 16>(n, src, src_stride, dst, dst_stride, zero_flag, stream);
    case 2: return launch_bi<2, 12>(n, src, src_stride, dst, dst_stride, zero_flag, stream);
    case 4: return launch_bi<4, 8>(n, src, src_stride, dst, dst_stride, zero_flag, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace sb
