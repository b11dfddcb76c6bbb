// common.cuh -- device helpers shared by the graph-build kernels (sm_100a).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tagore {

constexpr uint32_t kInv = 0xFFFFFFFFu;
constexpr float kInfDis = 10000000.0f;   // INF_DIS of the reference (include/common.cuh:29)
constexpr uint32_t kReserve = 128;       // RESERVENUM: row stride of reverse_distance
constexpr uint32_t kSelectCand = 480;    // SELECT_CAND: ring capacity of the path collect
constexpr uint32_t kSample = 32;         // SAMPLE: hybrid_list rows are 4*SAMPLE wide
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ float2 h2lo(uint32_t v) {
  return __half22float2(*reinterpret_cast<const __half2*>(&v));
}

// Packed FP32 pair arithmetic of sm_100 (PTX .f32x2): each half is its own
// IEEE operation rounded to nearest, so a pair op equals the two scalar ops.
// (x, y) += (a, b), and (x, y) = (d0*d0 + x, d1*d1 + y).
__device__ __forceinline__ void add2(float& x, float& y, float a, float b) {
  asm("{.reg .b64 p, q;\n\t"
      "mov.b64 p, {%0, %1};\n\t"
      "mov.b64 q, {%2, %3};\n\t"
      "add.rn.f32x2 p, p, q;\n\t"
      "mov.b64 {%0, %1}, p;}"
      : "+f"(x), "+f"(y)
      : "f"(a), "f"(b));
}
__device__ __forceinline__ void fma2_sq(float& x, float& y, float d0, float d1) {
  asm("{.reg .b64 p, q;\n\t"
      "mov.b64 p, {%0, %1};\n\t"
      "mov.b64 q, {%2, %3};\n\t"
      "fma.rn.f32x2 p, q, q, p;\n\t"
      "mov.b64 {%0, %1}, p;}"
      : "+f"(x), "+f"(y)
      : "f"(d0), "f"(d1));
}
// (d0, d1) = (float(a.lo) - b0, float(a.hi) - b1), one rounding each: the
// mixed f16/f32 subtract widens a exactly, as __half2float would.
__device__ __forceinline__ void sub_h2(uint32_t a, float b0, float b1, float& d0, float& d1) {
  asm("{.reg .b16 lo, hi;\n\t"
      "mov.b32 {lo, hi}, %2;\n\t"
      "sub.rn.f32.f16 %0, lo, %3;\n\t"
      "sub.rn.f32.f16 %1, hi, %4;}"
      : "=f"(d0), "=f"(d1)
      : "r"(a), "f"(b0), "f"(b1));
}

// Accumulates one 4-dim chunk into the lane's (x, y) pair exactly as the
// reference's two __hfma2 steps do (src/Tagore_src.cu:1431-1435), in FP32:
// x takes dims 0 and 2, y takes dims 1 and 3, each a fused multiply-add of the
// rounded difference.
__device__ __forceinline__ void chunk_acc(uint2 a, uint2 b, float& x, float& y) {
  const float2 b01 = h2lo(b.x), b23 = h2lo(b.y);
  float d0, d1, d2, d3;
  sub_h2(a.x, b01.x, b01.y, d0, d1);
  sub_h2(a.y, b23.x, b23.y, d2, d3);
  fma2_sq(x, y, d0, d1);
  fma2_sq(x, y, d2, d3);
}

// Reduces the per-lane pairs with the reference's shuffle-down tree (offsets
// 16..1) and returns x + y in every lane.
__device__ __forceinline__ float warp_tree(float x, float y) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    add2(x, y, __shfl_down_sync(kFull, x, off), __shfl_down_sync(kFull, y, off));
  return __shfl_sync(kFull, __fadd_rn(x, y), 0);
}

// Exact FP32 squared L2 between two FP16 rows, in the reference's lane order.
// Executed by a full warp; `dim` is a multiple of 4.
__device__ __forceinline__ float warp_dist(const __half* __restrict__ a, const __half* __restrict__ b,
                                           uint32_t dim, int lane) {
  float x = 0.0f, y = 0.0f;
  const uint32_t chunks = dim >> 2;
  for (uint32_t j = lane; j < chunks; j += 32) {
    const uint2 va = __ldg(reinterpret_cast<const uint2*>(a) + j);
    const uint2 vb = __ldg(reinterpret_cast<const uint2*>(b) + j);
    chunk_acc(va, vb, x, y);
  }
  return warp_tree(x, y);
}

// A query row's chunks as one lane holds them in the reference's lane order
// (chunk lane + 32 i in v[i]), for a width DIM fixed at compile time: loaded
// once, reused by every distance against that query.
template <uint32_t DIM>
struct QRow {
  static constexpr uint32_t kChunks = DIM / 4, kPerLane = (kChunks + 31) / 32;
  uint2 v[kPerLane];
};

template <uint32_t DIM>
__device__ __forceinline__ void load_qrow(const __half* __restrict__ q, QRow<DIM>& r, int lane) {
#pragma unroll
  for (uint32_t i = 0; i < QRow<DIM>::kPerLane; ++i) {
    const uint32_t j = lane + 32 * i;
    r.v[i] = j < QRow<DIM>::kChunks ? *(reinterpret_cast<const uint2*>(q) + j) : make_uint2(0u, 0u);
  }
}

// warp_dist4 against a preloaded query row.
template <uint32_t DIM>
__device__ __forceinline__ void warp_dist4_q(const QRow<DIM>& qr, const __half* __restrict__ base,
                                             const uint32_t ids[4], float out[4], int lane) {
  float x[4] = {0.f, 0.f, 0.f, 0.f}, y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (uint32_t i = 0; i < QRow<DIM>::kPerLane; ++i) {
    const uint32_t j = lane + 32 * i;
    if (j < QRow<DIM>::kChunks) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (ids[t] != kInv) {
          const uint2 vb = __ldg(reinterpret_cast<const uint2*>(base + (size_t)ids[t] * DIM) + j);
          chunk_acc(qr.v[i], vb, x[t], y[t]);
        }
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int t = 0; t < 4; ++t)
      add2(x[t], y[t], __shfl_down_sync(kFull, x[t], off), __shfl_down_sync(kFull, y[t], off));
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) out[t] = __shfl_sync(kFull, __fadd_rn(x[t], y[t]), 0);
}

// Four independent distances against one query, interleaving their shuffle
// trees. Rows with id kInv yield 0 and must be ignored by the caller. DIM,
// when given, fixes the width at compile time (`dim` is then DIM).
template <uint32_t DIM = 0>
__device__ __forceinline__ void warp_dist4(const __half* __restrict__ q, const __half* __restrict__ base,
                                           uint32_t dim, const uint32_t ids[4], float out[4],
                                           int lane) {
  float x[4] = {0.f, 0.f, 0.f, 0.f}, y[4] = {0.f, 0.f, 0.f, 0.f};
  if constexpr (DIM != 0) dim = DIM;
  auto chunk = [&](uint32_t j) {
    const uint2 vq = *(reinterpret_cast<const uint2*>(q) + j);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (ids[t] != kInv) {
        const uint2 vb = __ldg(reinterpret_cast<const uint2*>(base + (size_t)ids[t] * dim) + j);
        chunk_acc(vq, vb, x[t], y[t]);
      }
    }
  };
  if constexpr (DIM != 0) {
#pragma unroll
    for (uint32_t i = 0; i < (DIM / 4 + 31) / 32; ++i)
      if (lane + 32 * i < DIM / 4) chunk(lane + 32 * i);
  } else {
    const uint32_t chunks = dim >> 2;
    for (uint32_t j = lane; j < chunks; j += 32) chunk(j);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int t = 0; t < 4; ++t)
      add2(x[t], y[t], __shfl_down_sync(kFull, x[t], off), __shfl_down_sync(kFull, y[t], off));
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) out[t] = __shfl_sync(kFull, __fadd_rn(x[t], y[t]), 0);
}

// Eight independent distances against one query at 96 dims, four per
// half-warp. At 96 dims the reference's lane slots 0..23 hold one 4-half
// chunk each and slots 24..31 none, so its first tree level (offset 16)
// adds chunk l + 16 into slot l for l < 8 and adds nothing (an exact + 0) for
// l = 8..15. Lane l of each half computes slot l's leaf and, for l < 8, slot
// l + 16's leaf and their level-1 sum itself; levels 2-5 (offsets 8..1) run
// on shuffles within the half. Same operations in the same order as the
// full-warp tree, so the same values. Rows with id kInv yield 0 and must be
// ignored by the caller.
__device__ __forceinline__ void warp_dist8_d96(const __half* __restrict__ q,
                                               const __half* __restrict__ base,
                                               const uint32_t ids[8], float out[8], int lane) {
  constexpr uint32_t kDim = 96;
  const int half = lane >> 4, l = lane & 15;
  const uint2* Q = reinterpret_cast<const uint2*>(q);
  const uint2 q0 = Q[l];
  const uint2 q1 = l < 8 ? Q[l + 16] : make_uint2(0u, 0u);
  float x[4], y[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const uint32_t id = half ? ids[4 + t] : ids[t];
    x[t] = y[t] = 0.0f;
    if (id != kInv) {
      const uint2* R = reinterpret_cast<const uint2*>(base + (size_t)id * kDim);
      chunk_acc(q0, __ldg(R + l), x[t], y[t]);
      if (l < 8) {
        float x1 = 0.0f, y1 = 0.0f;
        chunk_acc(q1, __ldg(R + l + 16), x1, y1);
        add2(x[t], y[t], x1, y1);
      }
    }
  }
#pragma unroll
  for (int off = 8; off > 0; off >>= 1) {
#pragma unroll
    for (int t = 0; t < 4; ++t)
      add2(x[t], y[t], __shfl_down_sync(kFull, x[t], off, 16),
           __shfl_down_sync(kFull, y[t], off, 16));
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const float r = __fadd_rn(x[t], y[t]);
    out[t] = __shfl_sync(kFull, r, 0);
    out[4 + t] = __shfl_sync(kFull, r, 16);
  }
}

// The reference's shuffle-down tree evaluated by one thread over the 32 lane
// slots: v_L[l] = v_{L-1}[l] + v_{L-1}[l + (32 >> L)], root v_5[0]. Walking
// the tree depth-first visits the slots in bit-reversed order and keeps at
// most five partial pairs alive. `leaf(slot, x, y)` accumulates that slot's
// chunks (slot, slot + 32, ...) into (x, y) exactly as the lane would.
template <int Level, int Slot, class Leaf>
__device__ __forceinline__ void lane_tree(Leaf& leaf, float& x, float& y) {
  if constexpr (Level == 0) {
    x = 0.0f;
    y = 0.0f;
    leaf(Slot, x, y);
  } else {
    float ax, ay, bx, by;
    lane_tree<Level - 1, Slot>(leaf, ax, ay);
    lane_tree<Level - 1, Slot + (32 >> Level)>(leaf, bx, by);
    add2(ax, ay, bx, by);
    x = ax;
    y = ay;
  }
}

// Exact FP32 squared L2 in the reference's lane order by a single thread;
// chunk(j) returns the two 4-half chunks j of the operands.
template <int D, class Chunk>
__device__ __forceinline__ float serial_dist(Chunk chunk) {
  auto leaf = [&](int slot, float& x, float& y) {
#pragma unroll
    for (int j = slot; j < D / 4; j += 32) {
      const uint2 a = chunk(j, 0), b = chunk(j, 1);
      chunk_acc(a, b, x, y);
    }
  };
  float x, y;
  lane_tree<5, 0>(leaf, x, y);
  return __fadd_rn(x, y);
}

// The 128-dim tree with 16-byte loads. At 128 dims each lane slot holds one
// chunk, so level-1 node l is leaf l + leaf l+16 and level-2 node m is
// level-1 m + level-1 m+8; chunks 2p and 2p+1 share a 16-byte load. Level-2
// nodes are built in pairs (2p, 2p+1) from four loads per row and combined
// exactly as the tree combines them.
__device__ __forceinline__ void pair_acc(uint4 a, uint4 b, float& x0, float& y0, float& x1,
                                         float& y1) {
  chunk_acc(make_uint2(a.x, a.y), make_uint2(b.x, b.y), x0, y0);
  chunk_acc(make_uint2(a.z, a.w), make_uint2(b.z, b.w), x1, y1);
}

// load(p, w) returns chunks 2p and 2p+1 of operand w as one 16-byte value.
template <class Load16>
__device__ __forceinline__ void level2_pair(Load16& load, int p, float (&x)[2], float (&y)[2]) {
  // leaves 2p, 2p+1 (pair p), 2p+8.. (pair p+4), 2p+16.. (p+8), 2p+24.. (p+12)
  float lx[4][2], ly[4][2];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    lx[q][0] = ly[q][0] = lx[q][1] = ly[q][1] = 0.0f;
    pair_acc(load(p + 4 * q, 0), load(p + 4 * q, 1), lx[q][0], ly[q][0], lx[q][1], ly[q][1]);
  }
  // q indexes leaf offsets 0, 8, 16, 24: level 1 pairs (0,16) and (8,24),
  // level 2 pairs the two results.
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float ax = lx[0][h], ay = ly[0][h], bx = lx[1][h], by = ly[1][h];
    add2(ax, ay, lx[2][h], ly[2][h]);
    add2(bx, by, lx[3][h], ly[3][h]);
    add2(ax, ay, bx, by);
    x[h] = ax;
    y[h] = ay;
  }
}

template <class Load16>
__device__ __forceinline__ float dist128_pairs(Load16 load) {
  float x0[2], y0[2], x1[2], y1[2], x2[2], y2[2], x3[2], y3[2];
  level2_pair(load, 0, x0, y0);  // level-2 nodes 0, 1
  level2_pair(load, 2, x2, y2);  // 4, 5
  level2_pair(load, 1, x1, y1);  // 2, 3
  level2_pair(load, 3, x3, y3);  // 6, 7
  // level 3: m + m+4; level 4: m + m+2; level 5: 0 + 1
  add2(x0[0], y0[0], x2[0], y2[0]);
  add2(x0[1], y0[1], x2[1], y2[1]);
  add2(x1[0], y1[0], x3[0], y3[0]);
  add2(x1[1], y1[1], x3[1], y3[1]);
  add2(x0[0], y0[0], x1[0], y1[0]);
  add2(x0[1], y0[1], x1[1], y1[1]);
  add2(x0[0], y0[0], x0[1], y0[1]);
  return __fadd_rn(x0[0], y0[0]);
}

// The same tree for any width that is a multiple of 8 halves (`units`
// 16-byte units): lane slot s accumulates chunks s, s + 32, ... in order, so
// the leaves of pair p + 4q are summed over the units p + 4q, p + 4q + 16, ...
// before the level-1 and level-2 combining above. At 128 dims there is one
// round and this is dist128_pairs.
template <class Load16>
__device__ __forceinline__ void level2_pair_rounds(Load16& load, int p, uint32_t units,
                                                   float (&x)[2], float (&y)[2]) {
  float lx[4][2], ly[4][2];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    lx[q][0] = ly[q][0] = lx[q][1] = ly[q][1] = 0.0f;
    for (uint32_t u = p + 4 * q; u < units; u += 16)
      pair_acc(load(u, 0), load(u, 1), lx[q][0], ly[q][0], lx[q][1], ly[q][1]);
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float ax = lx[0][h], ay = ly[0][h], bx = lx[1][h], by = ly[1][h];
    add2(ax, ay, lx[2][h], ly[2][h]);
    add2(bx, by, lx[3][h], ly[3][h]);
    add2(ax, ay, bx, by);
    x[h] = ax;
    y[h] = ay;
  }
}

template <class Load16>
__device__ __forceinline__ float dist_pairs_rounds(Load16 load, uint32_t units) {
  float x0[2], y0[2], x1[2], y1[2], x2[2], y2[2], x3[2], y3[2];
  level2_pair_rounds(load, 0, units, x0, y0);
  level2_pair_rounds(load, 2, units, x2, y2);
  level2_pair_rounds(load, 1, units, x1, y1);
  level2_pair_rounds(load, 3, units, x3, y3);
  add2(x0[0], y0[0], x2[0], y2[0]);
  add2(x0[1], y0[1], x2[1], y2[1]);
  add2(x1[0], y1[0], x3[0], y3[0]);
  add2(x1[1], y1[1], x3[1], y3[1]);
  add2(x0[0], y0[0], x1[0], y1[0]);
  add2(x0[1], y0[1], x1[1], y1[1]);
  add2(x0[0], y0[0], x0[1], y0[1]);
  return __fadd_rn(x0[0], y0[0]);
}

// dist_pairs_rounds with the width fixed at compile time (U 16-byte units),
// so that every load of the tree is issued up front; the same operations in
// the same order.
template <uint32_t U, class Load16>
__device__ __forceinline__ void level2_pair_fixed(Load16& load, int p, float (&x)[2],
                                                  float (&y)[2]) {
  float lx[4][2], ly[4][2];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    lx[q][0] = ly[q][0] = lx[q][1] = ly[q][1] = 0.0f;
#pragma unroll
    for (uint32_t u = p + 4 * q; u < U; u += 16)
      pair_acc(load(u, 0), load(u, 1), lx[q][0], ly[q][0], lx[q][1], ly[q][1]);
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float ax = lx[0][h], ay = ly[0][h], bx = lx[1][h], by = ly[1][h];
    add2(ax, ay, lx[2][h], ly[2][h]);
    add2(bx, by, lx[3][h], ly[3][h]);
    add2(ax, ay, bx, by);
    x[h] = ax;
    y[h] = ay;
  }
}

template <uint32_t U, class Load16>
__device__ __forceinline__ float dist_pairs_fixed(Load16 load) {
  float x0[2], y0[2], x1[2], y1[2], x2[2], y2[2], x3[2], y3[2];
  level2_pair_fixed<U>(load, 0, x0, y0);
  level2_pair_fixed<U>(load, 2, x2, y2);
  level2_pair_fixed<U>(load, 1, x1, y1);
  level2_pair_fixed<U>(load, 3, x3, y3);
  add2(x0[0], y0[0], x2[0], y2[0]);
  add2(x0[1], y0[1], x2[1], y2[1]);
  add2(x1[0], y1[0], x3[0], y3[0]);
  add2(x1[1], y1[1], x3[1], y3[1]);
  add2(x0[0], y0[0], x1[0], y1[0]);
  add2(x0[1], y0[1], x1[1], y1[1]);
  add2(x0[0], y0[0], x0[1], y0[1]);
  return __fadd_rn(x0[0], y0[0]);
}

__device__ __forceinline__ float row_dist128(const __half* __restrict__ a,
                                             const __half* __restrict__ b) {
  const uint4* A = reinterpret_cast<const uint4*>(a);
  const uint4* B = reinterpret_cast<const uint4*>(b);
  return dist128_pairs([&](int p, int w) { return __ldg((w ? B : A) + p); });
}

// The same distance between two FP16 rows of `dim` halves (a multiple of 4)
// by a single thread, so that the 32 lanes of a warp score 32 rows at once.
// Kept out of line: one copy of the unrolled tree serves every call site and
// stays in the instruction cache.
static __device__ __noinline__ float row_dist(const __half* __restrict__ a,
                                              const __half* __restrict__ b, uint32_t dim) {
  const uint2* A = reinterpret_cast<const uint2*>(a);
  const uint2* B = reinterpret_cast<const uint2*>(b);
  if (dim == 128) return row_dist128(a, b);
  if (dim == 96) {
    const uint4* A4 = reinterpret_cast<const uint4*>(a);
    const uint4* B4 = reinterpret_cast<const uint4*>(b);
    return dist_pairs_fixed<12>([&](uint32_t u, int w) { return __ldg((w ? B4 : A4) + u); });
  }
  if ((dim & 7u) == 0) {
    const uint4* A4 = reinterpret_cast<const uint4*>(a);
    const uint4* B4 = reinterpret_cast<const uint4*>(b);
    return dist_pairs_rounds([&](uint32_t u, int w) { return __ldg((w ? B4 : A4) + u); }, dim >> 3);
  }
  const uint32_t chunks = dim >> 2;
  auto leaf = [&](int slot, float& x, float& y) {
    for (uint32_t j = slot; j < chunks; j += 32) chunk_acc(__ldg(A + j), __ldg(B + j), x, y);
  };
  float x, y;
  lane_tree<5, 0>(leaf, x, y);
  return __fadd_rn(x, y);
}

// distance_filter (src/Tagore_src.cu:1488-1490) as nvcc compiles it, one fused
// multiply-add, and angle_filter (:1493-1495) with IEEE-rounded operations.
__device__ __forceinline__ bool pruned_by(int metric, float res, float dis, float cur, float thre) {
  if (metric == 0) return __fmaf_rn(thre, res, -dis) < 0.0f;
  float v = __fsub_rn(__fadd_rn(dis, cur), res);
  v = __fdiv_rn(v, 2.0f);
  v = __fdiv_rn(v, __fsqrt_rn(__fmul_rn(dis, cur)));
  return __fsub_rn(thre, v) < 0.0f;
}

// The reference's block-wide bitonic network (src/Tagore_src.cu:29-44),
// executed by one warp over shared arrays: strides 1,2,4,.., steps stride..1,
// the first step of each merge mirrored, pairs past `len` skipped. Each pass
// touches disjoint pairs, so lane order inside a pass does not matter; the
// swap sequence, and therefore tie placement, equals the reference's.
template <class Gt, class Sw>
__device__ __forceinline__ void warp_network(uint32_t len, int lane, Gt gt, Sw sw) {
  for (uint32_t stride = 1; stride < len; stride <<= 1) {
    for (uint32_t step = stride; step > 0; step >>= 1) {
      const uint32_t sh = __ffs(step) - 1;
      for (uint32_t k = lane; k < (len >> 1); k += 32) {
        const uint32_t a = (k >> sh) << (sh + 1), b = k & (step - 1);
        const uint32_t u = (step == stride) ? (a + step - 1 - b) : (a + b);
        const uint32_t d = a + b + step;
        if (d < len && gt(u, d)) sw(u, d);
      }
      __syncwarp();
    }
  }
}

// Lower-bound membership test in a sorted shared array.
__device__ __forceinline__ bool sorted_contains(const uint32_t* a, uint32_t len, uint32_t key) {
  uint32_t lo = 0, hi = len;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo < len && a[lo] == key;
}

template <class T>
__device__ __forceinline__ void swap_(T& a, T& b) {
  T t = a;
  a = b;
  b = t;
}

}  // namespace tagore
