// knn_shared.cuh -- packed neighbour keys, warp sorts and the exact
// thread-serial distance shared by the kNN-graph kernels.
#pragma once
#include "common.cuh"
#include "internal.h"

namespace tagore {
namespace knn {

constexpr uint32_t kMaxS = 32;      // samples per list: join lists hold <= 4*32 ids
constexpr uint32_t kMaxList = 128;  // new + old rows of one local join
constexpr uint32_t kMaxT = 8;       // proposals kept per join row
constexpr uint32_t kPool = 128;     // hashed candidate slots per node
constexpr uint64_t kEmpty = ~0ull;

struct Work {
  uint32_t n, dim, K, S, T, P;
  const __half* data;
  const float* norms;
  uint64_t* nb;
  unsigned long long* pool;
  uint32_t *fnew, *fold, *rnew, *rold, *fcnt, *rcnt;
  uint32_t* lists;  // [n][128] join lists: new ids first, then old
  uint32_t* lcnt;   // [n][2] (new count, total)
  // [0] proposals, [1] exact pairs, [2] row updates, [3] rows gathered, [4] error flag,
  // [5..9] learned-screen measurements (16 slots)
  unsigned long long* stats;
  // [n] (norm, k-th distance of the row): the tensor-core joins' per-row
  // screen inputs in one 8-byte record, written by k_sample each iteration
  float2* meta;
  // order in which the tensor-core joins take the nodes (null: by id)
  const uint32_t* order = nullptr;
};

int join_tc(const Work& w, cudaStream_t s);
// Row widths the tensor-core join takes (one 128-row tile of K-major FP16).
inline bool tc_supported(uint32_t dim) { return dim >= 16 && dim <= 128 && dim % 16 == 0; }
// Wider rows: the Gram tile accumulated over 64-half column blocks.
int join_tc_wide(const Work& w, cudaStream_t s);
inline bool tc_wide_supported(uint32_t dim) { return dim > 128 && dim <= 1024 && dim % 8 == 0; }

__device__ __forceinline__ uint64_t make_key(float d, uint32_t id, bool is_new) {
  return ((uint64_t)__float_as_uint(d) << 32) | ((uint64_t)id << 1) | (is_new ? 1ull : 0ull);
}
__device__ __forceinline__ uint32_t key_id(uint64_t k) { return (uint32_t)(k >> 1) & 0x7FFFFFFFu; }
__device__ __forceinline__ float key_dist(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }
// k-th distance of a row; an empty slot accepts everything
__device__ __forceinline__ float kth_of(uint64_t k) {
  return k == kEmpty ? __int_as_float(0x7f800000) : key_dist(k);
}

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int m) {
  const uint32_t lo = __shfl_xor_sync(kFull, (uint32_t)v, m);
  const uint32_t hi = __shfl_xor_sync(kFull, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_u64(uint64_t v, int src) {
  const uint32_t lo = __shfl_sync(kFull, (uint32_t)v, src);
  const uint32_t hi = __shfl_sync(kFull, (uint32_t)(v >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_up_u64(uint64_t v, int d) {
  const uint32_t lo = __shfl_up_sync(kFull, (uint32_t)v, d);
  const uint32_t hi = __shfl_up_sync(kFull, (uint32_t)(v >> 32), d);
  return ((uint64_t)hi << 32) | lo;
}

// Ascending bitonic sort of 32*E keys held element-major (position t*32+lane).
template <int E>
__device__ __forceinline__ void warp_sort_keys(uint64_t (&k)[E], int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int ts = stride / 32;
#pragma unroll
        for (int t = 0; t < E; ++t) {
          const int q = t ^ ts;
          if (q > t) {
            const bool up = (((t * 32 + lane) & size) == 0);
            const uint64_t a = k[t], b = k[q];
            if (up ? (a > b) : (a < b)) {
              k[t] = b;
              k[q] = a;
            }
          }
        }
      } else {
#pragma unroll
        for (int t = 0; t < E; ++t) {
          const uint64_t o = shfl_xor_u64(k[t], stride);
          const bool up = (((t * 32 + lane) & size) == 0);
          const bool lower = (lane & stride) == 0;
          k[t] = (lower == up) ? (k[t] < o ? k[t] : o) : (k[t] > o ? k[t] : o);
        }
      }
    }
  }
}

// Writes the first K distinct keys of a sorted warp array to `row` (equal
// (distance, id) collapse to the first, which is the old copy when one is old),
// pads with kEmpty, and returns how many written keys carry the new flag.
template <int E>
__device__ __forceinline__ uint32_t dedupe_store_row(const uint64_t (&k)[E], int lane,
                                                     uint64_t* row, uint32_t K) {
  const unsigned lt = (1u << lane) - 1u;
  uint32_t base = 0, fresh = 0;
#pragma unroll
  for (int t = 0; t < E; ++t) {
    uint64_t prev = shfl_up_u64(k[t], 1);
    if (t > 0) {
      const uint64_t tail = shfl_u64(k[t - 1], 31);
      if (lane == 0) prev = tail;
    }
    const bool first = (t == 0 && lane == 0);
    const bool keep = k[t] != kEmpty && (first || (k[t] >> 1) != (prev >> 1));
    const unsigned m = __ballot_sync(kFull, keep);
    const uint32_t pos = base + __popc(m & lt);
    if (keep && pos < K) {
      row[pos] = k[t];
      fresh += (uint32_t)(k[t] & 1ull);
    }
    base += __popc(m);
  }
  for (uint32_t j = base + lane; j < K; j += 32) row[j] = kEmpty;
  return __reduce_add_sync(kFull, fresh);
}

// Hashed candidate pool: the slot keeps the smallest key (closest, then
// lowest id) proposed for it.
__device__ __forceinline__ void propose(unsigned long long* pool, uint32_t a, uint32_t P,
                                        uint32_t c, float d) {
  const uint32_t slot = (c * 0x9E3779B1u) >> 25;  // 7 bits: P == 128
  atomicMin(pool + (size_t)a * P + (slot & (P - 1)), (unsigned long long)make_key(d, c, true));
}

// Exact FP32 squared L2 of two FP16 rows held as 32-bit words, computed by one
// thread in the reference's lane order (32 lane slots, then the shuffle tree).
template <int D>
__device__ __forceinline__ float thread_dist(const uint32_t* __restrict__ a,
                                             const uint32_t* __restrict__ b, uint32_t dim_rt) {
  if constexpr (D > 0) {
    return serial_dist<D>([&](int j, int w) {
      const uint32_t* r = w ? b : a;
      return make_uint2(r[2 * j], r[2 * j + 1]);
    });
  } else {
    float x[32], y[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) {
      x[l] = 0.0f;
      y[l] = 0.0f;
    }
    for (uint32_t j = 0; j < dim_rt / 4; ++j)
      chunk_acc(make_uint2(a[2 * j], a[2 * j + 1]), make_uint2(b[2 * j], b[2 * j + 1]),
                x[j & 31], y[j & 31]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
      for (int l = 0; l < off; ++l) {
        x[l] = __fadd_rn(x[l], x[l + off]);
        y[l] = __fadd_rn(y[l], y[l + off]);
      }
    }
    return __fadd_rn(x[0], y[0]);
  }
}

}  // namespace knn
}  // namespace tagore
