// knn.cu -- GNN-Descent style kNN graph construction on sm_100a.
//
// Replaces the two phases of the reference (src/Tagore_src.cu:158-1206,
// driven from pybind.cu:103-125) by one NN-Descent loop over a packed 64-bit
// neighbour pool:
//   entry key = (float bits of the exact distance << 32) | (id << 1) | is_new
// so a row sorted by key is sorted by distance, equal ids with equal distance
// sit side by side (dedupe), and atomicMin on a key keeps the closer one.
// Per iteration:
//   sample  -- first S new and first S old entries of each row (the reference's
//              split, :536-567), new ones marked old; reverse samples appended
//              to the sampled nodes (:570-586);
//   lists   -- each node's join list: forward+reverse new ids, then old ids;
//   join    -- local join of new x (new u old); each list row keeps its
//              `per_row` closest partners and proposes those closer than its
//              current k-th entry by atomicMin into a hashed pool;
//   merge   -- pool entries merged into the sorted row with a warp bitonic sort.
// The join has two implementations: the plain one computes every pair with
// FP32 SIMT arithmetic; the chosen one (knn_tc.cu) screens pairs on tcgen05
// tensor-core tiles and re-ranks the kept ones exactly. Every stored distance
// is the exact FP32 value in the reference's lane order, the same function the
// prune stage uses.
#include <algorithm>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"
#include "knn_shared.cuh"
#include "mlp.cuh"

namespace tagore {
namespace knn {

__device__ __forceinline__ uint32_t mix32(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return (uint32_t)x;
}

// Random initial rows (the reference's initialize_graph, :158-166, seeded
// instead of clock-seeded) with exact distances, sorted, repeats removed.
__global__ void __launch_bounds__(128)
    k_init(const __half* __restrict__ data, uint32_t n, uint32_t dim, uint32_t K, uint64_t seed,
           uint64_t* __restrict__ nb) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t u = blockIdx.x * 4 + warp; u < n; u += gridDim.x * 4) {
    uint64_t keys[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const uint32_t j = lane + 32 * t;
      keys[t] = kEmpty;
      if (j < K) {
        uint32_t v = mix32(seed ^ ((uint64_t)u * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)j << 40)) % (n - 1);
        if (v >= u) ++v;  // never u itself
        keys[t] = (uint64_t)v;
      }
    }
    // one neighbour row per lane, in the reference's lane order (row_dist)
    const __half* q = data + (size_t)u * dim;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (keys[t] != kEmpty) {
        const uint32_t v = (uint32_t)keys[t];
        keys[t] = make_key(row_dist(q, data + (size_t)v * dim, dim), v, true);
      }
    }
    warp_sort_keys<4>(keys, lane);
    dedupe_store_row<4>(keys, lane, nb + (size_t)u * K, K);
  }
}

// First S new and first S old entries of each row; new ones become old.
// Reverse samples are appended to the sampled nodes' lists (capacity S).
__global__ void __launch_bounds__(128)
    k_sample(uint64_t* __restrict__ nb, const float* __restrict__ norms, float2* __restrict__ meta,
             uint32_t n, uint32_t K, uint32_t S,
             uint32_t* __restrict__ fnew, uint32_t* __restrict__ fold, uint32_t* __restrict__ fcnt,
             uint32_t* __restrict__ rnew, uint32_t* __restrict__ rold,
             uint32_t* __restrict__ rcnt) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t u = blockIdx.x * 4 + warp; u < n; u += gridDim.x * 4) {
    uint64_t* row = nb + (size_t)u * K;
    uint32_t cn = 0, co = 0;
    for (uint32_t base = 0; base < K; base += 32) {
      const uint32_t j = base + lane;
      const uint64_t k = (j < K) ? row[j] : kEmpty;
      const bool valid = k != kEmpty;
      const bool isnew = valid && (k & 1ull);
      const bool isold = valid && !(k & 1ull);
      const unsigned mn = __ballot_sync(kFull, isnew), mo = __ballot_sync(kFull, isold);
      const uint32_t rn = cn + __popc(mn & lt), ro = co + __popc(mo & lt);
      if (isnew && rn < S) {
        fnew[(size_t)u * S + rn] = key_id(k);
        row[j] = k & ~1ull;
      }
      if (isold && ro < S) fold[(size_t)u * S + ro] = key_id(k);
      if (j == K - 1) meta[u] = make_float2(norms[u], kth_of(k));
      cn += __popc(mn);
      co += __popc(mo);
    }
    cn = min(cn, S);
    co = min(co, S);
    __syncwarp();
    if (lane == 0) {
      fcnt[2 * u] = cn;
      fcnt[2 * u + 1] = co;
    }
    for (uint32_t i = lane; i < cn + co; i += 32) {
      const bool isnew = i < cn;
      const uint32_t v = isnew ? fnew[(size_t)u * S + i] : fold[(size_t)u * S + (i - cn)];
      const uint32_t slot = atomicAdd(&rcnt[2 * v + (isnew ? 0 : 1)], 1u);
      if (slot < S) (isnew ? rnew : rold)[(size_t)v * S + slot] = u;
    }
  }
}

// Join list of each node: forward new, reverse new (deduped, first kept),
// then forward old and reverse old not already present. Warp per node.
// Repeats are found with a per-warp open-addressing table of the node's up to
// 128 entries (256 slots, load <= 1/2): every entry claims its id's slot, and
// the slot's owner is the smallest position (source-major, then lane) that
// holds the id, so the first copy is the one kept whatever the order in which
// the lanes' atomics land.
constexpr uint32_t kListSlots = 256;

__device__ __forceinline__ uint32_t list_slot(uint32_t* __restrict__ key, uint32_t id) {
  uint32_t h = (id * 0x9E3779B1u) >> 24;  // 8 bits: kListSlots == 256
  for (uint32_t p = 0; p < kListSlots; ++p) {
    const uint32_t prev = atomicCAS(&key[h], kInv, id);
    if (prev == kInv || prev == id) break;
    h = (h + 1) & (kListSlots - 1);
  }
  return h;  // at most 128 ids in 256 slots: the loop ends on a free or own slot
}

__global__ void __launch_bounds__(128)
    k_build_lists(uint32_t n, uint32_t S, const uint32_t* __restrict__ fnew,
                  const uint32_t* __restrict__ fold, const uint32_t* __restrict__ fcnt,
                  const uint32_t* __restrict__ rnew, const uint32_t* __restrict__ rold,
                  const uint32_t* __restrict__ rcnt, uint32_t* __restrict__ lists,
                  uint32_t* __restrict__ lcnt) {
  __shared__ __align__(16) uint32_t key_s[4][kListSlots], owner_s[4][kListSlots];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  uint32_t* key = key_s[warp];
  uint32_t* owner = owner_s[warp];
  for (uint32_t u = blockIdx.x * 4 + warp; u < n; u += gridDim.x * 4) {
    // the four sources, one entry per lane (S <= 32): forward new, reverse
    // new, forward old, reverse old -- the order in which repeats keep their
    // first copy
    const uint32_t cnt[4] = {fcnt[2 * u], min(rcnt[2 * u], S), fcnt[2 * u + 1],
                             min(rcnt[2 * u + 1], S)};
    const uint32_t* src[4] = {fnew, rnew, fold, rold};
    uint32_t x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      x[q] = (uint32_t)lane < cnt[q] ? src[q][(size_t)u * S + lane] : kInv;
    const uint4 none = make_uint4(kInv, kInv, kInv, kInv);
#pragma unroll
    for (uint32_t t = (uint32_t)lane; t < kListSlots / 4; t += 32) {
      reinterpret_cast<uint4*>(key)[t] = none;
      reinterpret_cast<uint4*>(owner)[t] = none;
    }
    __syncwarp();
    uint32_t slot[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      slot[q] = 0;
      if (x[q] != kInv) {
        slot[q] = list_slot(key, x[q]);
        atomicMin(&owner[slot[q]], (uint32_t)(q * 32 + lane));
      }
    }
    __syncwarp();
    // an entry is kept when it is not u and is its id's first copy
    uint32_t pos = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool keep =
          x[q] != kInv && x[q] != u && owner[slot[q]] == (uint32_t)(q * 32 + lane);
      const unsigned m = __ballot_sync(kFull, keep);
      if (keep) lists[(size_t)u * kMaxList + pos + __popc(m & lt)] = x[q];
      pos += __popc(m);
      if (q == 1 && lane == 0) lcnt[2 * u] = pos;  // the new entries
    }
    if (lane == 0) lcnt[2 * u + 1] = pos;
    __syncwarp();  // every lane has read the table before the next node clears it
  }
}

// Plain local join: every pair with a new endpoint computed once with FP32
// SIMT arithmetic (thread per pair, reference lane order), kept in a shared
// distance matrix; each row then proposes its `per_row` closest partners.
// kStaged: the join-list rows are copied into shared memory first (rows up
// to about 300 dims); otherwise each pair reads its two rows from the cache
// hierarchy.
template <int D, bool kStaged>
__global__ void __launch_bounds__(128)
    k_join_plain(const uint64_t* __restrict__ nb, const __half* __restrict__ data, uint32_t n,
                 uint32_t dim_rt, uint32_t K, uint32_t T, uint32_t P,
                 const uint32_t* __restrict__ lists, const uint32_t* __restrict__ lcnt,
                 unsigned long long* __restrict__ pool, unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t dim = D > 0 ? (uint32_t)D : dim_rt;
  const uint32_t words = dim / 2 + 1;  // padded row stride in 32-bit words
  uint32_t* list = reinterpret_cast<uint32_t*>(smem);  // 128
  float* kth = reinterpret_cast<float*>(list + kMaxList);  // 128
  float* dm = kth + kMaxList;  // 128 x 129
  uint32_t* vec = reinterpret_cast<uint32_t*>(dm + kMaxList * (kMaxList + 1));
  const uint32_t tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  unsigned long long props = 0, pairs = 0, rows = 0;
  for (uint32_t u = blockIdx.x; u < n; u += gridDim.x) {
    const uint32_t nn = lcnt[2 * u], total = lcnt[2 * u + 1];
    if (nn == 0 || total < 2) continue;
    if (tid == 0) rows += total;
    if (tid < total) {
      list[tid] = lists[(size_t)u * kMaxList + tid];
      kth[tid] = kth_of(nb[(size_t)list[tid] * K + K - 1]);
    }
    __syncthreads();
    if (kStaged) {
      for (uint32_t r = warp; r < total; r += 4) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(data + (size_t)list[r] * dim);
        for (uint32_t w = lane; w < dim / 2; w += 32) vec[r * words + w] = __ldg(src + w);
      }
    }
    __syncthreads();
    for (uint32_t r = 0; r < nn; ++r) {
      for (uint32_t c = r + 1 + tid; c < total; c += blockDim.x) {
        const float d = kStaged ? thread_dist<D>(vec + r * words, vec + c * words, dim)
                                : row_dist(data + (size_t)list[r] * dim,
                                           data + (size_t)list[c] * dim, dim);
        dm[r * (kMaxList + 1) + c] = d;
        dm[c * (kMaxList + 1) + r] = d;
        ++pairs;
      }
    }
    __syncthreads();
    if (tid < total) {
      const uint32_t r = tid;
      float bd[kMaxT];
      uint32_t bc[kMaxT];
      for (uint32_t t = 0; t < T; ++t) {
        bd[t] = __int_as_float(0x7f800000);
        bc[t] = kInv;
      }
      for (uint32_t c = 0; c < total; ++c) {
        if (c == r || (r >= nn && c >= nn)) continue;
        float v = dm[r * (kMaxList + 1) + c];
        uint32_t vc = c;
        for (uint32_t t = 0; t < T; ++t)
          if (v < bd[t]) {
            swap_(v, bd[t]);
            swap_(vc, bc[t]);
          }
      }
      const uint32_t a = list[r];
      for (uint32_t t = 0; t < T; ++t) {
        if (bc[t] == kInv || !(bd[t] < kth[r])) break;
        propose(pool, a, P, list[bc[t]], bd[t]);
        ++props;
      }
    }
    __syncthreads();
  }
  atomicAdd(&stats[0], props);
  atomicAdd(&stats[1], pairs);
  if (tid == 0) atomicAdd(&stats[3], rows);
}

// Merges the pool of each node into its sorted row and clears the pool. Only
// the pool entries closer than the row's k-th (m of them, usually few) are
// sorted, in registers, and merged into the sorted row by rank; the merged
// sequence is the one a full sort of row and pool would give (keys are
// unique per pool slot, and a row key sorts before an equal pool key), and
// repeats of (distance, id) keep their first copy as before.
template <int E>
__device__ __forceinline__ void sort_fresh(uint64_t* fb, uint32_t m, int lane) {
  uint64_t k[E];
#pragma unroll
  for (int t = 0; t < E; ++t) {
    const uint32_t j = lane + 32 * t;
    k[t] = j < m ? fb[j] : kEmpty;
  }
  warp_sort_keys<E>(k, lane);
  __syncwarp();
#pragma unroll
  for (int t = 0; t < E; ++t) {
    const uint32_t j = lane + 32 * t;
    if (j < m) fb[j] = k[t];
  }
  __syncwarp();
}

__global__ void __launch_bounds__(128)
    k_merge(uint64_t* __restrict__ nb, unsigned long long* __restrict__ pool, uint32_t n,
            uint32_t K, uint32_t P, unsigned long long* __restrict__ stats) {
  __shared__ uint64_t rows_s[4][kMaxList], fresh_s[4][kPool], merged_s[4][kMaxList + kPool];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  uint64_t* rb = rows_s[warp];
  uint64_t* fb = fresh_s[warp];
  uint64_t* mb = merged_s[warp];
  unsigned long long upd = 0;
  for (uint32_t u = blockIdx.x * 4 + warp; u < n; u += gridDim.x * 4) {
    uint64_t* row = nb + (size_t)u * K;
    unsigned long long* pl = pool + (size_t)u * P;
    // the k-th key, the pool and the row are loaded together: one round trip
    const uint64_t kth = row[K - 1];
    uint64_t pk[kPool / 32], rk[kMaxList / 32];
#pragma unroll
    for (int t = 0; t < (int)(kPool / 32); ++t) {
      const uint32_t j = 32 * t + lane;
      pk[t] = j < P ? (uint64_t)pl[j] : kEmpty;
    }
#pragma unroll
    for (int t = 0; t < (int)(kMaxList / 32); ++t) {
      const uint32_t j = 32 * t + lane;
      rk[t] = j < K ? row[j] : kEmpty;
    }
    uint32_t m = 0;
#pragma unroll
    for (int t = 0; t < (int)(kPool / 32); ++t) {
      const uint64_t k = pk[t];
      if (k != kEmpty) pl[32 * t + lane] = kEmpty;
      const bool fresh = k < kth;
      const unsigned mk = __ballot_sync(kFull, fresh);
      if (fresh) fb[m + __popc(mk & lt)] = k;
      m += __popc(mk);
    }
    if (m == 0) continue;
#pragma unroll
    for (int t = 0; t < (int)(kMaxList / 32); ++t) {
      const uint32_t j = 32 * t + lane;
      if (j < K) rb[j] = rk[t];
    }
    __syncwarp();
    if (m <= 32) sort_fresh<1>(fb, m, lane);
    else if (m <= 64) sort_fresh<2>(fb, m, lane);
    else sort_fresh<4>(fb, m, lane);
    // merged rank: row i -> i + #(fresh < r_i); fresh p -> p + #(row <= f_p)
    for (uint32_t i = lane; i < K; i += 32) {
      const uint64_t r = rb[i];
      uint32_t lo = 0, hi = m;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (fb[mid] < r) lo = mid + 1;
        else hi = mid;
      }
      mb[i + lo] = r;
    }
    for (uint32_t p = lane; p < m; p += 32) {
      const uint64_t f = fb[p];
      uint32_t lo = 0, hi = K;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (rb[mid] <= f) lo = mid + 1;
        else hi = mid;
      }
      mb[p + lo] = f;
    }
    __syncwarp();
    // first K distinct (distance, id) keys back to the row
    const uint32_t total = K + m;
    uint32_t out = 0, fresh_kept = 0;
    for (uint32_t c = 0; c < total && out < K; c += 32) {
      const uint32_t i = c + lane;
      const uint64_t k = i < total ? mb[i] : kEmpty;
      const bool keep = k != kEmpty && (i == 0 || (k >> 1) != (mb[i - 1] >> 1));
      const unsigned mk = __ballot_sync(kFull, keep);
      const uint32_t pos = out + __popc(mk & lt);
      if (keep && pos < K) {
        row[pos] = k;
        fresh_kept += (uint32_t)(k & 1ull);
      }
      out += __popc(mk);
    }
    for (uint32_t j = out + lane; j < K; j += 32) row[j] = kEmpty;
    upd += __reduce_add_sync(kFull, fresh_kept);
    __syncwarp();
  }
  if (lane == 0) atomicAdd(&stats[2], upd);
}

// Splits the packed rows into the reference's graph (u32) and nei_distance
// (f32) buffers; an empty slot repeats the row's first id.
__global__ void k_finalize(const uint64_t* __restrict__ nb, uint32_t n, uint32_t K,
                           uint32_t* __restrict__ graph, float* __restrict__ nd) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * K;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = nb[e];
    const size_t r0 = e - e % K;
    if (k == kEmpty) {
      const uint64_t f = nb[r0];
      graph[e] = (f == kEmpty) ? (uint32_t)((e / K + 1) % n) : key_id(f);
      nd[e] = kInfDis;
    } else {
      graph[e] = key_id(k);
      nd[e] = key_dist(k);
    }
  }
}

// Processing order of the tensor-core joins. A node's join writes only
// proposals into the pool and reads the rows of its list, so the order in
// which nodes are taken changes no result. Taking together nodes whose lists
// overlap keeps the gathered rows resident in L2. Labels: each node takes the
// smallest label among itself and its first kOrderHops current neighbours,
// in place (labels only decrease, so concurrent updates are harmless), for
// kOrderRounds rounds; the order is the nodes sorted by label.
constexpr uint32_t kOrderHops = 4, kOrderRounds = 16;

__global__ void k_order_init(uint32_t* __restrict__ lab, uint32_t* __restrict__ ids, uint32_t n) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    lab[u] = u;
    ids[u] = u;
  }
}

__global__ void k_order_min(const uint64_t* __restrict__ nb, uint32_t K, uint32_t hops,
                            uint32_t* lab, uint32_t n) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    uint32_t m = lab[u];
    for (uint32_t j = 0; j < hops; ++j) {
      const uint64_t k = __ldg(nb + (size_t)u * K + j);
      if (k != kEmpty) m = min(m, lab[key_id(k)]);
    }
    if (m < lab[u]) lab[u] = m;
  }
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <int D>
int launch_join_plain(const Work& w, cudaStream_t s) {
  const uint32_t words = w.dim / 2 + 1;
  const size_t base = (size_t)2 * kMaxList * 4 + (size_t)kMaxList * (kMaxList + 1) * 4;
  const size_t staged = base + (size_t)kMaxList * words * 4;
  const bool stage = staged <= 227 * 1024;
  const size_t sm = stage ? staged : base;
  const void* fn = stage ? (const void*)k_join_plain<D, true> : (const void*)k_join_plain<D, false>;
  TG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int grid = sm_count() * std::max(1, (int)((227 * 1024) / (sm + 1024)));
  if (stage)
    k_join_plain<D, true><<<grid, 128, sm, s>>>(w.nb, w.data, w.n, w.dim, w.K, w.T, w.P, w.lists,
                                                w.lcnt, w.pool, w.stats);
  else
    k_join_plain<D, false><<<grid, 128, sm, s>>>(w.nb, w.data, w.n, w.dim, w.K, w.T, w.P, w.lists,
                                                 w.lcnt, w.pool, w.stats);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

// Local join screened by the learned projection z (n x 32, FP16). Each row
// keeps its T candidates closest in projected distance; the kept pairs are
// pooled per node and re-ranked with the exact reference-order FP32 distance
// of the two base rows, and a pair is proposed only when that beats the row's
// k-th entry. On every `sample_every`-th node the block also scores every
// pair exactly and counts the improving pairs (exact distance below the row's
// k-th) and how many of them the screen kept, stats[5] and stats[6], and
// the rows' exact best T candidates and how many the screen kept, stats[8]
// and stats[9].
constexpr uint32_t kLearnedMaxT = 8;
__global__ void __launch_bounds__(128)
    k_join_learned(const uint64_t* __restrict__ nb, const __half* __restrict__ data,
                   const __half* __restrict__ z, uint32_t n, uint32_t dim, uint32_t K, uint32_t T,
                   uint32_t P, const uint32_t* __restrict__ lists, const uint32_t* __restrict__ lcnt,
                   unsigned long long* __restrict__ pool, unsigned long long* __restrict__ stats,
                   uint32_t sample_every) {
  __shared__ float zs[kMaxList][mlp::kOut + 1];
  __shared__ uint32_t ids[kMaxList];
  __shared__ float kth[kMaxList];
  __shared__ uint32_t pairs[kMaxList * kLearnedMaxT];
  __shared__ uint32_t warp_cnt[4];
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  unsigned long long props = 0, exact = 0, rows = 0, improving = 0, found = 0, best = 0,
                     best_kept = 0;
  for (uint32_t u = blockIdx.x; u < n; u += gridDim.x) {
    const uint32_t nn = lcnt[2 * u], total = lcnt[2 * u + 1];
    if (nn == 0 || total < 2) continue;
    if (tid == 0) rows += total;
    const uint32_t r = tid;
    const bool live = r < total;
    if (live) {
      const uint32_t id = lists[(size_t)u * kMaxList + r];
      ids[r] = id;
      kth[r] = kth_of(nb[(size_t)id * K + K - 1]);
      const uint4* src = reinterpret_cast<const uint4*>(z + (size_t)id * mlp::kOut);
#pragma unroll
      for (int q = 0; q < mlp::kOut / 8; ++q) {
        const uint4 v = __ldg(src + q);
        const __half2* h = reinterpret_cast<const __half2*>(&v);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float2 f = __half22float2(h[e]);
          zs[r][q * 8 + 2 * e] = f.x;
          zs[r][q * 8 + 2 * e + 1] = f.y;
        }
      }
    }
    __syncthreads();
    // screen: the row's T closest columns in projected distance
    const uint32_t cmax = live ? ((r < nn) ? total : nn) : 0u;
    float zr[mlp::kOut];
#pragma unroll
    for (int o = 0; o < mlp::kOut; ++o) zr[o] = live ? zs[r][o] : 0.0f;
    float bd[kLearnedMaxT];
    uint32_t bc[kLearnedMaxT];
#pragma unroll
    for (int t = 0; t < (int)kLearnedMaxT; ++t) {
      bd[t] = (uint32_t)t < T ? INFINITY : -INFINITY;
      bc[t] = kInv;
    }
    for (uint32_t c = 0; c < total; ++c) {
      float pd = 0.0f;
#pragma unroll
      for (int o = 0; o < mlp::kOut; ++o) {
        const float e = zr[o] - zs[c][o];
        pd = fmaf(e, e, pd);
      }
      float worst = bd[0];
#pragma unroll
      for (int t = 1; t < (int)kLearnedMaxT; ++t) worst = (uint32_t)t < T ? bd[t] : worst;
      if (c < cmax && c != r && pd < worst) {
        float v = pd;
        uint32_t vc = c;
#pragma unroll
        for (int t = 0; t < (int)kLearnedMaxT; ++t)
          if (v < bd[t]) {
            swap_(v, bd[t]);
            swap_(vc, bc[t]);
          }
      }
    }
    // pooled exact re-rank of the kept pairs
    uint32_t kept = 0;
#pragma unroll
    for (int t = 0; t < (int)kLearnedMaxT; ++t) kept += bc[t] != kInv ? 1u : 0u;
    uint32_t incl = kept;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, incl, o);
      if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) warp_cnt[warp] = incl;
    __syncthreads();
    uint32_t off = incl - kept, npairs = 0;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      if ((uint32_t)w < warp) off += warp_cnt[w];
      npairs += warp_cnt[w];
    }
#pragma unroll
    for (int t = 0; t < (int)kLearnedMaxT; ++t)
      if (bc[t] != kInv) pairs[off++] = (r << 16) | bc[t];
    __syncthreads();
    for (uint32_t q = tid; q < npairs; q += blockDim.x) {
      const uint32_t pr = pairs[q], row = pr >> 16, col = pr & 0xFFFFu;
      const float d = row_dist(data + (size_t)ids[row] * dim, data + (size_t)ids[col] * dim, dim);
      ++exact;
      if (d < kth[row]) {
        propose(pool, ids[row], P, ids[col], d);
        ++props;
      }
    }
    // measurement on a sample of nodes: every pair exactly. Improving pairs
    // (exact distance below the row's k-th) and how many the screen kept steer
    // T; the row's exact best T and how many of them the screen kept measure
    // how well the projection ranks.
    if (sample_every && u % sample_every == 0 && live) {
      float ed[kLearnedMaxT];
      uint32_t ec[kLearnedMaxT];
#pragma unroll
      for (int t = 0; t < (int)kLearnedMaxT; ++t) {
        ed[t] = (uint32_t)t < T ? INFINITY : -INFINITY;
        ec[t] = kInv;
      }
      for (uint32_t c = 0; c < cmax; ++c) {
        if (c == r) continue;
        const float d = row_dist(data + (size_t)ids[r] * dim, data + (size_t)ids[c] * dim, dim);
        bool kept_c = false;
#pragma unroll
        for (int t = 0; t < (int)kLearnedMaxT; ++t) kept_c |= bc[t] == c;
        if (d < kth[r]) {
          ++improving;
          found += kept_c ? 1u : 0u;
        }
        float v = d;
        uint32_t vc = c;
#pragma unroll
        for (int t = 0; t < (int)kLearnedMaxT; ++t)
          if (v < ed[t]) {
            swap_(v, ed[t]);
            swap_(vc, ec[t]);
          }
      }
#pragma unroll
      for (int t = 0; t < (int)kLearnedMaxT; ++t) {
        if (ec[t] == kInv) continue;
        ++best;
        bool kept_c = false;
#pragma unroll
        for (int q = 0; q < (int)kLearnedMaxT; ++q) kept_c |= bc[q] == ec[t];
        best_kept += kept_c ? 1u : 0u;
      }
    }
    __syncthreads();
  }
  if (props) atomicAdd(&stats[0], props);
  if (exact) atomicAdd(&stats[1], exact);
  if (tid == 0 && rows) atomicAdd(&stats[3], rows);
  if (improving) atomicAdd(&stats[5], improving);
  if (found) atomicAdd(&stats[6], found);
  if (best) atomicAdd(&stats[8], best);
  if (best_kept) atomicAdd(&stats[9], best_kept);
}

int join_learned(const Work& w, const __half* z, uint32_t T, uint32_t sample_every,
                 cudaStream_t s) {
  const int grid = sm_count() * 8;
  k_join_learned<<<grid, 128, 0, s>>>(w.nb, w.data, z, w.n, w.dim, w.K, T, w.P, w.lists, w.lcnt,
                                      w.pool, w.stats, sample_every);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

int join_plain(const Work& w, cudaStream_t s) {
  switch (w.dim) {
    case 96: return launch_join_plain<96>(w, s);
    case 128: return launch_join_plain<128>(w, s);
    default: return launch_join_plain<0>(w, s);
  }
}

// Label bits of n nodes, and the radix sort's scratch for them.
static int order_bits(uint32_t n) {
  int end_bit = 1;
  while (end_bit < 32 && ((uint64_t)1 << end_bit) <= n) ++end_bit;
  return end_bit;
}
static size_t order_sort_bytes(uint32_t n) {
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0,
                                  order_bits(n));
  return tmp;
}

// Bytes of scratch order_nodes needs for n nodes.
size_t order_bytes(uint32_t n) { return (size_t)n * 16 + order_sort_bytes(n) + 256; }

// Writes the join order (see k_order_min) into scratch `buf` of
// order_bytes(n) bytes and points w.order at it.
int order_nodes(Work& w, void* buf, cudaStream_t s) {
  const uint32_t n = w.n, hops = std::min(kOrderHops, w.K);
  const int end_bit = order_bits(n);
  uint32_t* lab = static_cast<uint32_t*>(buf);
  uint32_t* ids = lab + n;
  uint32_t* lab2 = ids + n;
  uint32_t* out = lab2 + n;
  void* tmp_p = reinterpret_cast<char*>(out + n) + (256 - ((uintptr_t)(out + n) & 255)) % 256;
  size_t tmp = order_sort_bytes(n);
  const int g = sm_count() * 8;
  k_order_init<<<g, 256, 0, s>>>(lab, ids, n);
  count_launch();
  for (uint32_t r = 0; r < kOrderRounds; ++r) {
    k_order_min<<<g, 256, 0, s>>>(w.nb, w.K, hops, lab, n);
    count_launch();
  }
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cub::DeviceRadixSort::SortPairs(tmp_p, tmp, lab, lab2, ids, out, (int)n, 0, end_bit, s));
  w.order = out;
  return TAGORE_OK;
}

}  // namespace knn

// The exact join for a width and mode: the tensor-core tile up to 128 dims,
// the K-streamed tile up to 1024, otherwise (and in the plain mode) FP32 SIMT.
static int join_exact(const knn::Work& w, uint32_t mode, cudaStream_t s) {
  if (mode != TAGORE_KNN_PLAIN && knn::tc_supported(w.dim)) return knn::join_tc(w, s);
  if (mode != TAGORE_KNN_PLAIN && knn::tc_wide_supported(w.dim)) return knn::join_tc_wide(w, s);
  return knn::join_plain(w, s);
}

int knn_build(const Dev& d, const float* norms, const KnnArgs& a, KnnStats* st, cudaStream_t s) {
  using namespace knn;
  if (d.n < 2 || a.k == 0 || a.k >= d.n) return fail(TAGORE_EINVAL, "need POINTS > K >= 1");
  if (a.k > 128) return fail(TAGORE_EINVAL, "K must be <= 128 (got %u)", a.k);
  if (d.dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", d.dim);
  if (d.n >= 0x7FFFFFFFu) return fail(TAGORE_EINVAL, "POINTS must be < 2^31");
  if (a.mode > TAGORE_KNN_LEARNED) return fail(TAGORE_EINVAL, "unknown kNN mode %u", a.mode);
  const uint32_t S = std::min<uint32_t>(a.sample ? a.sample : 32, kMaxS);
  const uint32_t T = std::min<uint32_t>(a.per_row ? a.per_row : 2,
                                        a.mode == TAGORE_KNN_PLAIN ? kMaxT : 4u);
  const uint32_t P = kPool;
  const uint32_t K = a.k;
  Work w{};
  w.n = d.n;
  w.dim = d.dim;
  w.K = K;
  w.S = S;
  w.T = T;
  w.P = P;
  w.data = d.data;
  w.norms = norms;
  const size_t nbB = (size_t)d.n * K * 8, poolB = (size_t)d.n * P * 8;
  const size_t listB = (size_t)d.n * S * 4;
  Scratch sc(s);
  TG_TRY(sc.alloc(nbB + poolB + 4 * listB + (size_t)d.n * kMaxList * 4 + (size_t)d.n * 32 + 256));
  unsigned char* p = sc.as<unsigned char>();
  w.nb = reinterpret_cast<uint64_t*>(p);
  p += nbB;
  w.meta = reinterpret_cast<float2*>(p);
  p += (size_t)d.n * 8;
  w.pool = reinterpret_cast<unsigned long long*>(p);
  p += poolB;
  w.fnew = reinterpret_cast<uint32_t*>(p);
  w.fold = w.fnew + (size_t)d.n * S;
  w.rnew = w.fold + (size_t)d.n * S;
  w.rold = w.rnew + (size_t)d.n * S;
  w.lists = w.rold + (size_t)d.n * S;
  w.fcnt = w.lists + (size_t)d.n * kMaxList;
  w.rcnt = w.fcnt + (size_t)d.n * 2;
  w.lcnt = w.rcnt + (size_t)d.n * 2;
  w.stats = reinterpret_cast<unsigned long long*>(
      (reinterpret_cast<uintptr_t>(w.lcnt + (size_t)d.n * 2) + 15) & ~(uintptr_t)15);
  TG_CUDA(cudaMemsetAsync(w.pool, 0xFF, poolB, s));
  TG_CUDA(cudaMemsetAsync(w.stats, 0, 128, s));
  const int sms = sm_count();
  const uint64_t n64 = d.n;
  stage_begin("knn_init", s);
  k_init<<<sms * 16, 128, 0, s>>>(d.data, d.n, d.dim, K, a.seed, w.nb);
  count_launch();
  stage_end("knn_init", s, n64 * K * (2ull * d.dim + 8), n64 * K);
  TG_CUDA(cudaGetLastError());
  const bool tc_width = tc_supported(d.dim) || tc_wide_supported(d.dim);
  const char* join_name = a.mode == TAGORE_KNN_PLAIN || !tc_width ? "knn_join_plain"
                          : tc_supported(d.dim)                   ? "knn_join_tc"
                                                                  : "knn_join_tc_wide";
  // The learned screen serves the chosen path where no tensor-core tile
  // applies (and every width when asked for): the first iterations run the
  // exact join, then the MLP is trained on their rows and screens the rest.
  const bool learned = a.mode == TAGORE_KNN_LEARNED || (a.mode == TAGORE_KNN_CHOSEN && !tc_width);
  const uint32_t warm = std::min<uint32_t>(2, a.iters);
  uint32_t lt = a.per_row ? std::min<uint32_t>(std::max<uint32_t>(a.per_row, 2), kLearnedMaxT) : 4;
  const bool adapt = !(a.learn_flags & TAGORE_LEARN_FIXED_T);
  bool fallback = false;
  mlp::Net net;
  Scratch zbuf(s);
  ScreenStats sst{};
  // the tensor-core joins take the nodes in locality order from the second
  // iteration on (the first one's rows are random), recomputed once more at
  // the fourth as the rows settle
  const bool ordered = a.mode != TAGORE_KNN_PLAIN && tc_width;
  Scratch obuf(s);
  if (ordered && a.iters > 1) TG_TRY(obuf.alloc(order_bytes(d.n)));
  for (uint32_t it = 0; it < a.iters; ++it) {
    if (ordered && (it == 1 || it == 3)) {
      stage_begin("knn_order", s);
      TG_TRY(order_nodes(w, obuf.as<unsigned char>(), s));
      stage_end("knn_order", s);
    }
    TG_CUDA(cudaMemsetAsync(w.rcnt, 0, (size_t)d.n * 8, s));
    stage_begin("knn_sample", s);
    k_sample<<<sms * 16, 128, 0, s>>>(w.nb, w.norms, w.meta, d.n, K, S, w.fnew, w.fold, w.fcnt, w.rnew, w.rold,
                                       w.rcnt);
    count_launch();
    stage_end("knn_sample", s, n64 * K * 8 + n64 * 2 * S * 4 * 2 + n64 * 12, n64);
    TG_CUDA(cudaGetLastError());
    stage_begin("knn_lists", s);
    k_build_lists<<<sms * 16, 128, 0, s>>>(d.n, S, w.fnew, w.fold, w.fcnt, w.rnew, w.rold, w.rcnt,
                                           w.lists, w.lcnt);
    count_launch();
    stage_end("knn_lists", s, n64 * 4 * S * 4 + n64 * kMaxList * 4, n64);
    TG_CUDA(cudaGetLastError());
    if (learned && it == warm && !fallback) {
      stage_begin("mlp_train", s);
      TG_TRY(net.init(d.dim, a.seed ^ 0x5C4EE17ull, s));
      TG_TRY(net.center(d.data, d.n, s));
      const uint32_t steps = (a.learn_flags & TAGORE_LEARN_NO_TRAIN)
                                 ? 0u
                                 : (a.learn_steps ? a.learn_steps : 400u);
      if (steps) {
        TG_TRY(net.train(w.nb, d.n, K, d.data, steps, 4096, a.seed + it, &sst.loss_first,
                         &sst.loss_last, s));
      }
      sst.steps = steps;
      stage_end("mlp_train", s, (uint64_t)steps * 3 * 4096 * (2ull * d.dim), (uint64_t)steps * 4096);
      stage_begin("mlp_project", s);
      TG_TRY(zbuf.alloc((size_t)d.n * mlp::kOut * 2));
      TG_TRY(net.project(d.data, d.n, zbuf.as<__half>(), s));
      stage_end("mlp_project", s, n64 * (2ull * d.dim + 2ull * mlp::kOut), n64);
    }
    if (learned && it >= warm && !fallback) {
      stage_begin("knn_join_learned", s);
      TG_CUDA(cudaMemsetAsync(w.stats + 5, 0, 5 * 8, s));
      TG_TRY(join_learned(w, zbuf.as<__half>(), lt, 256, s));
      count_launch();
      stage_end("knn_join_learned", s);
      unsigned long long h2[5] = {0, 0, 0, 0, 0};
      TG_CUDA(cudaMemcpyAsync(h2, w.stats + 5, sizeof(h2), cudaMemcpyDeviceToHost, s));
      TG_CUDA(cudaStreamSynchronize(s));
      sst.last_best_kept = h2[3] ? (double)h2[4] / (double)h2[3] : 0.0;
      // miss rate of the screen on the sampled nodes steers the kept count.
      // A screen that misses most improving pairs (three in four at any
      // count, or half at the largest) hands the join to the exact path: this
      // iteration's join is run again exactly, its proposals joining the
      // screened ones in the pool, so no iteration is lost to the screen.
      const double miss = h2[0] ? 1.0 - (double)h2[1] / (double)h2[0] : 0.0;
      sst.last_miss = miss;
      sst.screened_iters += 1;
      if (adapt) {
        if (miss > 0.75 || (miss > 0.5 && lt == kLearnedMaxT)) {
          fallback = true;
          stage_begin(join_name, s);
          TG_TRY(join_exact(w, a.mode, s));
          count_launch();
          stage_end(join_name, s);
        } else if (miss > 0.10 && lt < kLearnedMaxT) {
          lt = std::min<uint32_t>(kLearnedMaxT, lt + 2);
        } else if (miss < 0.02 && lt > 2) {
          lt -= 1;
        }
      }
    } else {
      stage_begin(join_name, s);
      TG_TRY(join_exact(w, a.mode, s));
      count_launch();
      stage_end(join_name, s);
    }
    stage_begin("knn_merge", s);
    k_merge<<<sms * 16, 128, 0, s>>>(w.nb, w.pool, d.n, K, P, w.stats);
    count_launch();
    stage_end("knn_merge", s, n64 * (16ull * K + 16ull * P), n64);
    TG_CUDA(cudaGetLastError());
  }
  k_finalize<<<sms * 8, 256, 0, s>>>(w.nb, d.n, K, d.graph, d.nd);
  count_launch();
  TG_CUDA(cudaGetLastError());
  unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  TG_CUDA(cudaMemcpyAsync(h, w.stats, sizeof(h), cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  if ((uint32_t)h[4] != 0) return fail(TAGORE_ETIMEOUT, "tensor-core join: a bounded wait ran out");
  // join traffic: each gathered row (FP16 vector, 8-byte norm and k-th
  // distance record, list id), one 8-byte count pair per node, one 8-byte
  // read-modify-write per proposal
  stage_add(join_name, h[3] * (2ull * d.dim + 12) + n64 * a.iters * 8 + h[0] * 16, h[1]);
  if (st) {
    st->proposals = h[0];
    st->pairs = h[1];
  }
  sst.used = learned ? 1u : 0u;
  sst.per_row = lt;
  sst.fallback = fallback ? 1u : 0u;
  set_screen_stats(sst);
  return TAGORE_OK;
}

}  // namespace tagore
