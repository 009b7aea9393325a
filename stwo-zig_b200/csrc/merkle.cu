// Lifted Blake2s Merkle commitment on the device.
//
// Leaf = Blake2s("leaf" prefix block || LE32 of each column value at the row)
// (src/core/vcs_lifted/blake2_merkle.zig:193-262, src/prover/vcs_lifted/leaves.zig:24-115);
// node = Blake2s("node" prefix block || left || right) (blake2_merkle.zig:77-130).
// The prefix block's chaining value is a constant seed, so a leaf costs
// ceil(4 n_cols / 64) compressions and a node one compression.
//
// One thread per leaf: a warp reads 32 consecutive rows of a column as one
// 128-byte transaction; the message schedule and state stay in registers.
// Each CTA hashes 256 leaves and then folds the three node levels whose parents
// fill whole warps (128, 64, 32) in shared memory, writing every level; a tree
// that fits one CTA is folded to its root there. The layers above are folded by
// k_merkle_nodes: four levels per launch while there are more than 2^12
// children, then up to 9 levels per launch.
#include <utility>

#include "blake2s.cuh"
#include "kernels.cuh"
#include "tuner.hpp"

namespace sb {

namespace {

constexpr uint32_t LEAF_THREADS = 256;  // leaves per CTA
constexpr uint32_t LEAF_LEVELS = 8;     // node levels folded inside a leaf CTA
constexpr uint32_t FULL_WARP_LEVELS = 3;  // levels whose parents fill whole warps (128, 64, 32)
constexpr uint32_t NODE_THREADS = 256;  // parents per CTA at the first level
constexpr uint32_t NODE_FOLD_LOG = 12;  // layers up to 2^12 nodes fold inside CTAs

struct Seeds { uint32_t leaf[8], node[8]; };

// Programmatic dependent launch for the latency-bound chains (node levels, FRI layers, channel
// steps): the kernels of a chain are launched with programmatic stream serialization, so the launch
// of the next one is processed while the previous one runs, and each waits until the previous kernel
// of the stream has completed and its memory is visible (griddepcontrol.wait) before it reads
// anything. The wait is the hardware's grid dependency, not a flag. No kernel triggers its
// dependents early: early triggers let waiting CTAs hold SMs that other proofs' kernels could use
// (batched 2^20x100 proofs 156.4 -> 154.2 proofs/s), while the wait alone keeps the single-proof
// gain (6.89 -> 6.70 ms median). Chaining the large kernels too (FFT passes, leaves, OODS,
// quotients, proof-of-work rounds) measured 1% slower batched and no faster single. Launched
// without the attribute, the wait is a no-op.
__device__ __forceinline__ void chain_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... K, typename... A>
cudaError_t launch_chained(void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

Seeds make_seeds() {
  Seeds s;
  b2s_prefix_seed("leaf", s.leaf);
  b2s_prefix_seed("node", s.node);
  return s;
}

__device__ __forceinline__ void store_hash(uint8_t* layers, uint64_t node, const uint32_t h[8]) {
  uint4* d = reinterpret_cast<uint4*>(layers + node * 32);
  d[0] = make_uint4(h[0], h[1], h[2], h[3]);
  d[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

__device__ __forceinline__ void node_hash(const uint32_t seed[8], const uint32_t* l, const uint32_t* r, uint32_t h[8],
                                          uint32_t one) {
  uint32_t m[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) { m[i] = l[i]; m[8 + i] = r[i]; }
#pragma unroll
  for (int i = 0; i < 8; ++i) h[i] = seed[i];
  b2s_compress(h, m, 128, true, one);
}

// Folds `count` hashes in shared memory (sm[i*8 .. i*8+8)) `levels` times;
// level j's nodes are written to the layer of log size (top_log - j).
__device__ void fold_levels(uint32_t* sm, uint32_t count, uint32_t levels, uint8_t* layers, uint32_t max_log,
                            uint32_t child_log, uint64_t first_child, const uint32_t seed[8], uint32_t one) {
  for (uint32_t j = 1; j <= levels; ++j) {
    uint32_t n = count >> j;
    uint32_t h[8];
    bool active = threadIdx.x < n;
    if (active) node_hash(seed, sm + (2 * threadIdx.x) * 8, sm + (2 * threadIdx.x + 1) * 8, h, one);
    __syncthreads();
    if (active) {
#pragma unroll
      for (int i = 0; i < 8; ++i) sm[threadIdx.x * 8 + i] = h[i];
      uint32_t layer_log = child_log - j;
      uint64_t node = merkle_layer_offset(max_log, layer_log) + (first_child >> j) + threadIdx.x;
      store_hash(layers, node, h);
    }
    __syncthreads();
  }
}

// Five CTAs per SM (48 registers, 16 bytes spilled): a 2^21 x 100 commit took 0.765 ms,
// against 0.789 ms at six CTAs per SM (40 registers, 80 bytes spilled), 0.887 ms at four
// (64 registers, no spills) and 0.953 ms for the unconstrained 62-register build.
template <int MINB>
__global__ void __launch_bounds__(LEAF_THREADS, MINB) k_merkle_leaves(uint32_t log_size, uint32_t n_cols,
                                                                 const uint32_t* __restrict__ cols, uint64_t stride,
                                                                 uint8_t* layers, Seeds seeds, uint32_t levels,
                                                                 uint32_t one) {
  __shared__ uint32_t sm[LEAF_THREADS * 8];
  const uint64_t row = (uint64_t)blockIdx.x * LEAF_THREADS + threadIdx.x;
  const uint64_t n_rows = 1ull << log_size;
  uint32_t h[8];
  if (row < n_rows) {
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = seeds.leaf[i];
    // Blocks of 16 columns without a bounds test, then the ragged last block; the column
    // pointer advances by the stride (no per-column index product).
    const uint32_t n_full = n_cols / 16, rem = n_cols % 16;
    const uint32_t total = 64 + 4 * n_cols;
    const uint32_t* p = cols + row;
    for (uint32_t blk = 0; blk < n_full; ++blk) {
      uint32_t m[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        m[i] = __ldg(p);
        p += stride;
      }
      const bool last = rem == 0 && blk + 1 == n_full;
      b2s_compress(h, m, last ? total : 64 + 64 * (blk + 1), last, one);
    }
    if (rem) {
      uint32_t m[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) m[i] = (uint32_t)i < rem ? __ldg(p + (uint64_t)i * stride) : 0u;
      b2s_compress(h, m, total, true, one);
    }
    store_hash(layers, row, h);
#pragma unroll
    for (int i = 0; i < 8; ++i) sm[threadIdx.x * 8 + i] = h[i];
  }
  __syncthreads();
  uint32_t count = n_rows < LEAF_THREADS ? (uint32_t)n_rows : LEAF_THREADS;
  fold_levels(sm, count, levels, layers, log_size, log_size, (uint64_t)blockIdx.x * LEAF_THREADS, seeds.node, one);
}

// Leaves over columns of mixed log sizes (the lifted tree, src/prover/vcs_lifted/
// leaves.zig:104-115): leaf pos hashes, for every column in leaf order (stably
// sorted by log size ascending), its value at ((pos >> (max_log - log + 1)) << 1)
// + (pos & 1). Column pointers and log sizes are staged in shared memory.
constexpr uint32_t LIFTED_MAX_COLS = 2048;

__global__ void __launch_bounds__(LEAF_THREADS) k_merkle_leaves_lifted(uint32_t max_log, uint32_t n_cols,
                                                                       const uint32_t* const* __restrict__ col_ptrs,
                                                                       const uint32_t* __restrict__ col_logs,
                                                                       uint8_t* layers, Seeds seeds, uint32_t levels,
                                                                       uint32_t one) {
  __shared__ uint32_t sm[LEAF_THREADS * 8];
  __shared__ const uint32_t* sp[LIFTED_MAX_COLS];
  __shared__ uint8_t ssh[LIFTED_MAX_COLS];  // max_log - log + 1, or 0 for full-size columns
  for (uint32_t c = threadIdx.x; c < n_cols; c += blockDim.x) {
    sp[c] = col_ptrs[c];
    uint32_t lg = col_logs[c];
    ssh[c] = lg == max_log ? 0 : (uint8_t)(max_log - lg + 1);
  }
  __syncthreads();
  const uint64_t row = (uint64_t)blockIdx.x * LEAF_THREADS + threadIdx.x;
  const uint64_t n_rows = 1ull << max_log;
  uint32_t h[8];
  if (row < n_rows) {
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = seeds.leaf[i];
    const uint32_t n_blocks = (n_cols + 15) / 16;
    const uint32_t total = 64 + 4 * n_cols;
    for (uint32_t blk = 0; blk < n_blocks; ++blk) {
      uint32_t m[16];
      const uint32_t c0 = blk * 16;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        uint32_t c = c0 + i;
        uint32_t v = 0;
        if (c < n_cols) {
          uint32_t sh = ssh[c];
          uint64_t idx = sh == 0 ? row : (((row >> sh) << 1) | (row & 1));
          v = __ldg(sp[c] + idx);
        }
        m[i] = v;
      }
      const bool last = blk + 1 == n_blocks;
      const uint32_t t = last ? total : 64 + 64 * (blk + 1);
      b2s_compress(h, m, t, last, one);
    }
    store_hash(layers, row, h);
#pragma unroll
    for (int i = 0; i < 8; ++i) sm[threadIdx.x * 8 + i] = h[i];
  }
  __syncthreads();
  uint32_t count = n_rows < LEAF_THREADS ? (uint32_t)n_rows : LEAF_THREADS;
  fold_levels(sm, count, levels, layers, max_log, max_log, (uint64_t)blockIdx.x * LEAF_THREADS, seeds.node, one);
}

// Children layer of log size child_log -> `levels` parent levels; each CTA folds
// 2 * NODE_THREADS children (or the whole layer when smaller).
__global__ void __launch_bounds__(NODE_THREADS) k_merkle_nodes(uint8_t* layers, uint32_t max_log, uint32_t child_log,
                                                                uint32_t levels, Seeds seeds, uint32_t one) {
  chain_enter();
  __shared__ uint32_t sm[2 * NODE_THREADS * 8];
  const uint64_t n_children = 1ull << child_log;
  const uint32_t per_cta = n_children < 2 * NODE_THREADS ? (uint32_t)n_children : 2 * NODE_THREADS;
  const uint64_t first = (uint64_t)blockIdx.x * per_cta;
  const uint4* src = reinterpret_cast<const uint4*>(layers + (merkle_layer_offset(max_log, child_log) + first) * 32);
  for (uint32_t i = threadIdx.x; i < per_cta * 2; i += blockDim.x) {
    uint4 v = src[i];
    sm[i * 4 + 0] = v.x; sm[i * 4 + 1] = v.y; sm[i * 4 + 2] = v.z; sm[i * 4 + 3] = v.w;
  }
  __syncthreads();
  fold_levels(sm, per_cta, levels, layers, max_log, child_log, first, seeds.node, one);
}

// FRI fold fused with the next layer's commitment (src/core/fri/folding.zig:352-384,
// 558-602; src/prover/fri.zig:377-592): thread i folds pair (2i, 2i+1) of the source
// into line value i, stores its 4 coordinates and, when `layers` is set, hashes it
// as leaf i of the next layer's tree (4 words, one compression) and folds `levels`
// node levels inside the CTA.
__device__ __forceinline__ void fri_ibfly(QM31& f0, QM31& f1, uint32_t it) {
  QM31 a = f0;
  f0 = qadd(a, f1);
  f1 = qmulm(qsub(a, f1), it);
}

template <bool CIRCLE>
__global__ void __launch_bounds__(LEAF_THREADS) k_fri_fold_commit(TwiddleView itv, uint32_t dst_log,
                                                                   const uint32_t* __restrict__ src, uint64_t ss,
                                                                   const QM31* alpha_p, uint32_t* dst, uint64_t ds,
                                                                   uint8_t* layers, Seeds seeds, uint32_t levels,
                                                                   uint32_t one) {
  chain_enter();
  __shared__ uint32_t sm[LEAF_THREADS * 8];
  const uint64_t n = 1ull << dst_log;
  const uint64_t i = (uint64_t)blockIdx.x * LEAF_THREADS + threadIdx.x;
  if (i < n) {
    const QM31 alpha = *alpha_p;
    uint2 w0 = *reinterpret_cast<const uint2*>(src + 2 * i);
    uint2 w1 = *reinterpret_cast<const uint2*>(src + ss + 2 * i);
    uint2 w2 = *reinterpret_cast<const uint2*>(src + 2 * ss + 2 * i);
    uint2 w3 = *reinterpret_cast<const uint2*>(src + 3 * ss + 2 * i);
    QM31 f0 = qmake(w0.x, w1.x, w2.x, w3.x), f1 = qmake(w0.y, w1.y, w2.y, w3.y);
    fri_ibfly(f0, f1, CIRCLE ? itv.circ((uint32_t)i) : itv.line(1, (uint32_t)i));
    QM31 r = CIRCLE ? qadd(qmul(alpha, f1), f0) : qadd(f0, qmul(alpha, f1));
    dst[i] = r.c0.a; dst[ds + i] = r.c0.b; dst[2 * ds + i] = r.c1.a; dst[3 * ds + i] = r.c1.b;
    if (layers) {
      uint32_t h[8], m[16] = {r.c0.a, r.c0.b, r.c1.a, r.c1.b, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < 8; ++k) h[k] = seeds.leaf[k];
      b2s_compress(h, m, 80, true, one);
      store_hash(layers, i, h);
#pragma unroll
      for (int k = 0; k < 8; ++k) sm[threadIdx.x * 8 + k] = h[k];
    }
  }
  if (!layers) return;
  __syncthreads();
  uint32_t count = n < LEAF_THREADS ? (uint32_t)n : LEAF_THREADS;
  fold_levels(sm, count, levels, layers, dst_log, dst_log, (uint64_t)blockIdx.x * LEAF_THREADS, seeds.node, one);
}

constexpr int FRI_DRAW_TRIES = 64;

// One thread: the channel steps of one FRI layer (see fri_channel_step).
__device__ void fri_channel_body(FriChannelDev* c, const uint8_t* root, uint32_t slot) {
  uint32_t m[16], h[8];
  const uint32_t* r = reinterpret_cast<const uint32_t*>(root);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    m[k] = c->digest[k];
    m[8 + k] = r[k];
    c->roots[slot][k] = r[k];
  }
  b2s_init(h);
  b2s_compress(h, m, 64, true);  // digest' = H(digest || root), one final 64-byte block
  uint32_t n_draws = 0;
  // drawSecureFelt: words of H(digest || LE32 n_draws || 0), all below 2p, else draw again.
  for (int tries = 0; tries < FRI_DRAW_TRIES; ++tries) {
    uint32_t w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) m[k] = h[k];
    m[8] = n_draws;
#pragma unroll
    for (int k = 9; k < 16; ++k) m[k] = 0;
    b2s_init(w);
    b2s_compress(w, m, 37, true);
    ++n_draws;
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 8; ++k) ok &= w[k] < 2 * P;
    if (ok) {
#pragma unroll
      for (int k = 0; k < 8; ++k) c->digest[k] = h[k];
      c->n_draws = n_draws;
      c->alpha[slot] = qmake(mreduce64(w[0]), mreduce64(w[1]), mreduce64(w[2]), mreduce64(w[3]));
      return;
    }
  }
  c->status = 1;
  c->alpha[slot] = qmake(0, 0, 0, 0);
}

__global__ void k_fri_channel(FriChannelDev* c, const uint8_t* root, uint32_t slot) {
  chain_enter();
  fri_channel_body(c, root, slot);
}

// The small inner FRI layers in one CTA: for line layers k = k0 .. n_inner-1 (2^(L-1-k) values,
// at most 2^FRI_TAIL_LOG), the channel step on layer k's root (alpha into slot k + 1), the fold
// into layer k + 1 and, below the last layer, the commitment of layer k + 1: leaf hashes and every
// node level, folded in shared memory. Same arithmetic, buffers and outputs as the per-layer
// k_fri_channel + k_fri_fold_commit<false> + merkle_finish sequence.
constexpr uint32_t FRI_TAIL_LOG = 12, FRI_TAIL_THREADS = 1024;
struct FriTailParams {
  uint32_t L, k0, n_inner;
  uint32_t* line[FRI_MAX_LAYERS + 1];
  uint8_t* tree[FRI_MAX_LAYERS];
  TwiddleView tv[FRI_MAX_LAYERS];  // inverse view of line layer k's domain (log L - k)
  Seeds seeds;
};

__global__ void __launch_bounds__(FRI_TAIL_THREADS) k_fri_tail(FriChannelDev* c, const __grid_constant__ FriTailParams p,
                                                               uint32_t one) {
  chain_enter();
  extern __shared__ uint32_t tsm[];  // (2^(FRI_TAIL_LOG-1)) hashes, then alpha
  QM31* s_alpha = reinterpret_cast<QM31*>(tsm + (1u << (FRI_TAIL_LOG - 1)) * 8);
  const uint32_t t = threadIdx.x;
  for (uint32_t k = p.k0; k < p.n_inner; ++k) {
    const uint32_t lg = p.L - 1 - k;
    const uint64_t sz = 1ull << lg, n = sz >> 1;
    if (t == 0) {
      fri_channel_body(c, p.tree[k] + (2 * sz - 2) * 32, k + 1);
      *s_alpha = c->alpha[k + 1];
    }
    __syncthreads();
    const QM31 alpha = *s_alpha;
    const uint32_t* src = p.line[k];
    uint32_t* dst = p.line[k + 1];
    const bool commit = k + 1 < p.n_inner;
    for (uint32_t i = t; i < n; i += FRI_TAIL_THREADS) {
      QM31 f0 = qmake(src[2 * i], src[sz + 2 * i], src[2 * sz + 2 * i], src[3 * sz + 2 * i]);
      QM31 f1 = qmake(src[2 * i + 1], src[sz + 2 * i + 1], src[2 * sz + 2 * i + 1], src[3 * sz + 2 * i + 1]);
      fri_ibfly(f0, f1, p.tv[k].line(1, i));
      const QM31 r = qadd(f0, qmul(alpha, f1));
      dst[i] = r.c0.a; dst[n + i] = r.c0.b; dst[2 * n + i] = r.c1.a; dst[3 * n + i] = r.c1.b;
      if (commit) {
        uint32_t h[8], m[16] = {r.c0.a, r.c0.b, r.c1.a, r.c1.b, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = p.seeds.leaf[q];
        b2s_compress(h, m, 80, true, one);
        store_hash(p.tree[k + 1], i, h);
#pragma unroll
        for (int q = 0; q < 8; ++q) tsm[i * 8 + q] = h[q];
      }
    }
    __syncthreads();
    if (commit) fold_levels(tsm, (uint32_t)n, lg - 1, p.tree[k + 1], lg - 1, lg - 1, 0, p.seeds.node, one);
  }
}

__global__ void k_empty_root(uint8_t* layers, Seeds seeds) {
  // No columns: the single leaf hashes the prefix block alone, as the final block.
  uint32_t h[8];
  b2s_init(h);
  uint32_t m[16] = {0};
  m[0] = 0x6661656cu;  // "leaf" little-endian
  b2s_compress(h, m, 64, true);
  store_hash(layers, 0, h);
}

}  // namespace

static const Seeds& seeds_once() {
  static const Seeds seeds = make_seeds();
  return seeds;
}

// Folds the node layers above child layer `child_log` of a tree with 2^max_log leaves.
static cudaError_t merkle_finish(uint8_t* layers, uint32_t max_log, uint32_t child_log, cudaStream_t stream) {
  const Seeds& seeds = seeds_once();
  cudaError_t e = cudaSuccess;
  // Large layers: four levels per launch, each CTA folding 512 children (every level's
  // parents fill whole warps: 256, 128, 64, 32).
  while (child_log > NODE_FOLD_LOG) {
    uint32_t levels = child_log - NODE_FOLD_LOG < 4 ? child_log - NODE_FOLD_LOG : 4;
    uint32_t blocks = (uint32_t)((1ull << child_log) / (2 * NODE_THREADS));
    e = launch_chained(k_merkle_nodes, blocks, NODE_THREADS, 0, stream, layers, max_log, child_log, levels, seeds, 1u);
    note_launch();
    if (e != cudaSuccess) return e;
    child_log -= levels;
  }
  while (child_log > 0) {
    uint32_t levels = child_log < 9 ? child_log : 9;
    uint64_t n_children = 1ull << child_log;
    uint32_t per_cta = n_children < 2 * NODE_THREADS ? (uint32_t)n_children : 2 * NODE_THREADS;
    uint32_t blocks = (uint32_t)(n_children / per_cta);
    e = launch_chained(k_merkle_nodes, blocks, NODE_THREADS, 0, stream, layers, max_log, child_log, levels, seeds, 1u);
    note_launch();
    if (e != cudaSuccess) return e;
    child_log -= levels;
  }
  return cudaSuccess;
}

uint32_t fri_tail_first(uint32_t L, uint32_t n_inner) {
  for (uint32_t k = 0; k < n_inner; ++k)
    if (L - 1 - k <= FRI_TAIL_LOG) return k;
  return n_inner;
}

cudaError_t fri_tail(const DeviceTables& t, FriChannelDev* c, uint32_t L, uint32_t k0, uint32_t n_inner,
                     uint32_t* const* line, uint8_t* const* trees, cudaStream_t stream) {
  if (k0 >= n_inner) return cudaSuccess;
  if (n_inner > FRI_MAX_LAYERS || L - 1 - k0 > FRI_TAIL_LOG) return cudaErrorInvalidValue;
  FriTailParams p{};
  p.L = L;
  p.k0 = k0;
  p.n_inner = n_inner;
  for (uint32_t k = k0; k <= n_inner; ++k) p.line[k] = line[k];
  for (uint32_t k = k0; k < n_inner; ++k) {
    p.tree[k] = trees[k];
    p.tv[k] = t.view(L - k, true);
  }
  p.seeds = seeds_once();
  const size_t smem = (1u << (FRI_TAIL_LOG - 1)) * 32 + 16;
  static const bool attr = [&] {  // once per process (thread-safe static initialisation)
    cudaFuncSetAttribute(k_fri_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return true;
  }();
  (void)attr;
  cudaError_t e = launch_chained(k_fri_tail, 1, FRI_TAIL_THREADS, smem, stream, c, p, 1u);
  note_launch();
  return e;
}

cudaError_t fri_channel_step(FriChannelDev* c, const uint8_t* root, uint32_t slot, cudaStream_t stream) {
  if (slot >= FRI_MAX_LAYERS) return cudaErrorInvalidValue;
  cudaError_t e = launch_chained(k_fri_channel, 1, 1, 0, stream, c, root, slot);
  note_launch();
  return e;
}

cudaError_t fri_fold_commit(const DeviceTables& t, bool circle, uint32_t src_log, const uint32_t* src,
                            uint64_t src_stride, const QM31* alpha, uint32_t* dst, uint64_t dst_stride,
                            uint8_t* layers, cudaStream_t stream) {
  const Seeds& seeds = seeds_once();
  const uint32_t dst_log = src_log - 1;
  const uint64_t n = 1ull << dst_log;
  const uint32_t grid = (uint32_t)((n + LEAF_THREADS - 1) / LEAF_THREADS);
  // One compression per leaf; the CTA also folds the three full-warp node levels
  // (the whole tree when it fits one CTA).
  const uint32_t levels = layers ? (dst_log <= LEAF_LEVELS ? dst_log : FULL_WARP_LEVELS) : 0;
  cudaError_t e;
  if (circle)
    e = launch_chained(k_fri_fold_commit<true>, grid, LEAF_THREADS, 0, stream, t.view(src_log, true), dst_log, src,
                       src_stride, alpha, dst, dst_stride, layers, seeds, levels, 1u);
  else
    e = launch_chained(k_fri_fold_commit<false>, grid, LEAF_THREADS, 0, stream, t.view(src_log + 1, true), dst_log, src,
                       src_stride, alpha, dst, dst_stride, layers, seeds, levels, 1u);
  note_launch();
  if (e != cudaSuccess || !layers) return e;
  return merkle_finish(layers, dst_log, dst_log - levels, stream);
}

cudaError_t merkle_commit(uint32_t log_size, uint32_t n_cols, const uint32_t* cols, uint64_t stride,
                          uint8_t* layers, cudaStream_t stream) {
  const Seeds& seeds = seeds_once();
  if (n_cols == 0) {
    k_empty_root<<<1, 1, 0, stream>>>(layers, seeds); note_launch();
    return cudaGetLastError();
  }
  const uint64_t n_rows = 1ull << log_size;
  // A tree that fits one CTA is folded to its root in the leaf launch; larger ones
  // fold their three full-warp node levels there. Levels 4-8 inside the CTA would
  // run on partly empty warps (16, 8, .. 1 parents): for 2^21 leaves of 4 words,
  // folding 8 levels took 283 us, 3 levels 245 us and none 254 us.
  uint32_t leaf_levels = log_size <= LEAF_LEVELS ? log_size : FULL_WARP_LEVELS;
  uint32_t grid = (uint32_t)((n_rows + LEAF_THREADS - 1) / LEAF_THREADS);
  // Variants: leaf kernels built for 5, 6 and 4 resident CTAs per SM (48, 40 and 64 registers).
  auto commit = [&](int variant) -> cudaError_t {
    if (variant == 1)
      k_merkle_leaves<6><<<grid, LEAF_THREADS, 0, stream>>>(log_size, n_cols, cols, stride, layers, seeds, leaf_levels, 1u);
    else if (variant == 2)
      k_merkle_leaves<4><<<grid, LEAF_THREADS, 0, stream>>>(log_size, n_cols, cols, stride, layers, seeds, leaf_levels, 1u);
    else
      k_merkle_leaves<5><<<grid, LEAF_THREADS, 0, stream>>>(log_size, n_cols, cols, stride, layers, seeds, leaf_levels, 1u);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return merkle_finish(layers, log_size, log_size - leaf_levels, stream);
  };
  // Trees big enough for the occupancy to matter; the commit only reads the columns.
  return tuned_run(TUNE_LEAVES, log_size, n_cols, log_size >= 16 ? 3 : 1, true, stream, commit);
}

cudaError_t merkle_commit_lifted(uint32_t max_log, uint32_t n_cols, const uint32_t* const* col_ptrs,
                                 const uint32_t* col_logs, uint8_t* layers, cudaStream_t stream) {
  const Seeds& seeds = seeds_once();
  if (n_cols == 0) {
    k_empty_root<<<1, 1, 0, stream>>>(layers, seeds); note_launch();
    return cudaGetLastError();
  }
  if (n_cols > LIFTED_MAX_COLS) return cudaErrorInvalidValue;
  const uint64_t n_rows = 1ull << max_log;
  uint32_t leaf_levels = max_log <= LEAF_LEVELS ? max_log : FULL_WARP_LEVELS;
  uint32_t grid = (uint32_t)((n_rows + LEAF_THREADS - 1) / LEAF_THREADS);
  k_merkle_leaves_lifted<<<grid, LEAF_THREADS, 0, stream>>>(max_log, n_cols, col_ptrs, col_logs, layers, seeds,
                                                            leaf_levels, 1u); note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return merkle_finish(layers, max_log, max_log - leaf_levels, stream);
}

// ---------------------------------------------------------------------------
// Proof of work: lowest nonce with ctz(Blake2s(prefix_digest || LE64 nonce)[0..16]) >= n_bits.
// Each thread tests its nonces in increasing order and stops once its next nonce
// is not below the best found so far, so every nonce below the result is tested
// and the result does not depend on scheduling (src/core/channel/blake2s.zig:168-240).
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ uint32_t ctz128(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  if (a) return __ffs(a) - 1;
  if (b) return 32 + __ffs(b) - 1;
  if (c) return 64 + __ffs(c) - 1;
  if (d) return 96 + __ffs(d) - 1;
  return 128;
}

// The grind hashes prefix (32 bytes) || nonce (8 bytes) as one final block. Of
// the first round's eight G steps only G(v0, v5, v10, v15, m8, m9) reads the
// nonce; the other seven touch other state words and constant message words,
// so they run once per prefix on the host. `v` is the working state after those
// seven (v0, v5, v10, v15 as the column step left them).
struct PowPrefix { uint32_t w[8]; uint32_t v[16]; };

PowPrefix pow_prefix(const uint32_t words[8]) {
  PowPrefix p;
  const uint32_t one = 1;  // the additions' multiplier when this body is parsed for the device
  (void)one;
  uint32_t h[8], m[16] = {};
  b2s_init(h);
  for (int i = 0; i < 8; ++i) p.w[i] = m[i] = words[i];
  uint32_t v0 = h[0], v1 = h[1], v2 = h[2], v3 = h[3], v4 = h[4], v5 = h[5], v6 = h[6], v7 = h[7];
  uint32_t v8 = B2sIv::v0, v9 = B2sIv::v1, v10 = B2sIv::v2, v11 = B2sIv::v3;
  uint32_t v12 = B2sIv::v4 ^ 40u, v13 = B2sIv::v5, v14 = ~B2sIv::v6, v15 = B2sIv::v7;
  SB_B2S_G(v0, v4, v8, v12, m[0], m[1]);
  SB_B2S_G(v1, v5, v9, v13, m[2], m[3]);
  SB_B2S_G(v2, v6, v10, v14, m[4], m[5]);
  SB_B2S_G(v3, v7, v11, v15, m[6], m[7]);
  SB_B2S_G(v1, v6, v11, v12, m[10], m[11]);
  SB_B2S_G(v2, v7, v8, v13, m[12], m[13]);
  SB_B2S_G(v3, v4, v9, v14, m[14], m[15]);
  const uint32_t v[16] = {v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15};
  for (int i = 0; i < 16; ++i) p.v[i] = v[i];
  return p;
}

// The grind's message is the 32-byte prefix digest (words 0-7), the nonce (words 8 and 9) and six
// zero words. These rounds name the message words by token, so an addition of a word that is zero
// (10-15 always, 9 when every nonce of the round is below 2^32) is not issued at all: 63 additions
// of the 9 rounds that follow the first, which the generic compression issues because its message
// words are only known at run time.
#define SB_PADD_M0(t) SB_ADD(t, w0)
#define SB_PADD_M1(t) SB_ADD(t, w1)
#define SB_PADD_M2(t) SB_ADD(t, w2)
#define SB_PADD_M3(t) SB_ADD(t, w3)
#define SB_PADD_M4(t) SB_ADD(t, w4)
#define SB_PADD_M5(t) SB_ADD(t, w5)
#define SB_PADD_M6(t) SB_ADD(t, w6)
#define SB_PADD_M7(t) SB_ADD(t, w7)
#define SB_PADD_M8(t) SB_ADD(t, n_lo)
#define SB_PADD_M9(t) (HI0 ? (t) : SB_ADD(t, n_hi))
#define SB_PADD_M10(t) (t)
#define SB_PADD_M11(t) (t)
#define SB_PADD_M12(t) (t)
#define SB_PADD_M13(t) (t)
#define SB_PADD_M14(t) (t)
#define SB_PADD_M15(t) (t)

#define SB_POW_G(a, b, c, d, X, Y)                           \
  do {                                                       \
    a = SB_PADD_##X(SB_ADD(a, b)); d = rotr32(d ^ a, 16);    \
    c = SB_ADD(c, d);              b = rotr32(b ^ c, 12);    \
    a = SB_PADD_##Y(SB_ADD(a, b)); d = rotr32(d ^ a, 8);     \
    c = SB_ADD(c, d);              b = rotr32(b ^ c, 7);     \
  } while (0)

#define SB_POW_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  do {                                                                                    \
    SB_POW_G(v0, v4, v8, v12, s0, s1);                                                    \
    SB_POW_G(v1, v5, v9, v13, s2, s3);                                                    \
    SB_POW_G(v2, v6, v10, v14, s4, s5);                                                   \
    SB_POW_G(v3, v7, v11, v15, s6, s7);                                                   \
    SB_POW_G(v0, v5, v10, v15, s8, s9);                                                   \
    SB_POW_G(v1, v6, v11, v12, s10, s11);                                                 \
    SB_POW_G(v2, v7, v8, v13, s12, s13);                                                  \
    SB_POW_G(v3, v4, v9, v14, s14, s15);                                                  \
  } while (0)

// Rounds 2..10 (sigma rows 1..9 of RFC 7693 section 2.7).
#define SB_POW_ROUNDS_2_TO_10()                                                           \
  do {                                                                                    \
    SB_POW_ROUND(M14, M10, M4, M8, M9, M15, M13, M6, M1, M12, M0, M2, M11, M7, M5, M3);    \
    SB_POW_ROUND(M11, M8, M12, M0, M5, M2, M15, M13, M10, M14, M3, M6, M7, M1, M9, M4);    \
    SB_POW_ROUND(M7, M9, M3, M1, M13, M12, M11, M14, M2, M6, M5, M10, M4, M0, M15, M8);    \
    SB_POW_ROUND(M9, M0, M5, M7, M2, M4, M10, M15, M14, M1, M11, M12, M6, M8, M3, M13);    \
    SB_POW_ROUND(M2, M12, M6, M10, M0, M11, M8, M3, M4, M13, M7, M5, M15, M14, M1, M9);    \
    SB_POW_ROUND(M12, M5, M1, M15, M14, M13, M4, M10, M0, M7, M6, M3, M9, M2, M8, M11);    \
    SB_POW_ROUND(M13, M11, M7, M14, M12, M1, M3, M9, M5, M0, M15, M4, M8, M6, M2, M10);    \
    SB_POW_ROUND(M6, M15, M14, M9, M11, M3, M0, M8, M12, M2, M13, M7, M1, M4, M10, M5);    \
    SB_POW_ROUND(M10, M2, M8, M4, M7, M6, M1, M5, M15, M11, M9, M14, M3, M12, M13, M0);    \
  } while (0)

// One bounded round of the search: nonces [base, base + grid*256*per_thread).
// Rounds are enqueued in nonce order on one stream; a round starts by leaving
// at once when an earlier round already found a smaller nonce, and each thread
// stops at its first valid nonce or once the best known nonce is below its own.
// CTA b owns the contiguous nonces [base + b*256*per_thread, +256*per_thread)
// and CTAs are dispatched in index order, so the round runs in nonce order: once
// the lowest valid nonce is found, only the CTAs in flight around it still work
// (spreading each CTA's nonces over the whole round left about a quarter of a
// round of work above the hit).
// LOW32: for n_bits <= 32 the condition is that the low n_bits of the first hash
// word are zero, so only that word is live and the compiler drops the last
// round's work that only feeds the other words.
// HI0: every nonce of the round is below 2^32, so message word 9 is zero.
template <bool LOW32, bool HI0>
__global__ void __launch_bounds__(256) k_pow_round(PowPrefix pre, uint32_t n_bits, uint64_t base,
                                                   uint32_t per_thread, unsigned long long* found, uint32_t one) {
  const uint32_t stride = blockDim.x;
  uint64_t nonce = base + (uint64_t)blockIdx.x * blockDim.x * per_thread + threadIdx.x;
  const uint32_t mask = n_bits >= 32 ? 0xffffffffu : (1u << n_bits) - 1u;
  const uint32_t w0 = pre.w[0], w1 = pre.w[1], w2 = pre.w[2], w3 = pre.w[3], w4 = pre.w[4], w5 = pre.w[5],
                 w6 = pre.w[6], w7 = pre.w[7];
  unsigned long long best = *((volatile unsigned long long*)found);
  for (uint32_t k = 0; k < per_thread && nonce < best; ++k, nonce += stride) {
    const uint32_t n_lo = (uint32_t)nonce, n_hi = (uint32_t)(nonce >> 32);
    (void)n_hi;
    uint32_t v0 = pre.v[0], v1 = pre.v[1], v2 = pre.v[2], v3 = pre.v[3], v4 = pre.v[4], v5 = pre.v[5],
             v6 = pre.v[6], v7 = pre.v[7], v8 = pre.v[8], v9 = pre.v[9], v10 = pre.v[10], v11 = pre.v[11],
             v12 = pre.v[12], v13 = pre.v[13], v14 = pre.v[14], v15 = pre.v[15];
    SB_POW_G(v0, v5, v10, v15, M8, M9);
    SB_POW_ROUNDS_2_TO_10();
    const uint32_t h0 = (B2sIv::v0 ^ 0x01010020u) ^ v0 ^ v8;
    const bool ok = LOW32 ? (h0 & mask) == 0
                          : ctz128(h0, B2sIv::v1 ^ v1 ^ v9, B2sIv::v2 ^ v2 ^ v10, B2sIv::v3 ^ v3 ^ v11) >= n_bits;
    if (ok) {
      atomicMin(found, (unsigned long long)nonce);
      return;
    }
    if ((k & 3) == 3) best = *((volatile unsigned long long*)found);
  }
}

}  // namespace

uint64_t pow_round_nonces(int sm_count) { return (uint64_t)sm_count * 4 * 256 * 112; }

cudaError_t pow_round(const uint32_t prefix_words[8], uint32_t n_bits, uint64_t base, uint32_t* result_dev,
                      int sm_count, cudaStream_t stream) {
  const PowPrefix pre = pow_prefix(prefix_words);
  // Four waves of short CTAs (32 registers: eight 256-thread CTAs resident per SM;
  // 14 nonces per thread, ~0.15 ms a wave) rather than one wave of long ones, so
  // that other streams' work gets SMs between them.
  auto* res = reinterpret_cast<unsigned long long*>(result_dev);
  const bool hi0 = base + pow_round_nonces(sm_count) <= (1ull << 32);
  const uint32_t grid = sm_count * 4 * 8;
  if (n_bits <= 32) {
    if (hi0) k_pow_round<true, true><<<grid, 256, 0, stream>>>(pre, n_bits, base, 14, res, 1u);
    else k_pow_round<true, false><<<grid, 256, 0, stream>>>(pre, n_bits, base, 14, res, 1u);
  } else {
    if (hi0) k_pow_round<false, true><<<grid, 256, 0, stream>>>(pre, n_bits, base, 14, res, 1u);
    else k_pow_round<false, false><<<grid, 256, 0, stream>>>(pre, n_bits, base, 14, res, 1u);
  }
  note_launch();
  return cudaGetLastError();
}

}  // namespace sb
