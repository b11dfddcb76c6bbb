// prune.cu -- Collect / Filter / Store prune of a kNN graph on sm_100a.
//
// Restates the CFS framework of ZJU-DAILY/Tagore (src/Tagore_src.cu:1209-2058,
// pybind.cu:145-295) with one warp per node and results that are a function of
// the input graph only:
//  * every distance is FP32 arithmetic on the FP16 base in the reference's
//    lane order (common.cuh), every sort is the reference's bitonic network on
//    the same positions, so ties fall where the reference puts them;
//  * the Collect stage reads the kNN graph as a snapshot: pruned rows go to
//    scratch and reach `graph` only in the Store stage;
//  * reverse edges are inserted in ascending source order (a stable radix sort
//    by target), so the reference's replacement rule for full lists
//    (:1465-1475, :1697-1707) gives one defined answer;
//  * the Filter stage is evaluated lazily: a candidate is tested against the
//    kept neighbours in order and dropped at the first rule that fires, which
//    keeps exactly the set the reference's round-by-round sweep (:1416-1460)
//    keeps while computing far fewer distances.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <string>

#include "common.cuh"
#include "internal.h"
#include "knn_shared.cuh"

namespace tagore {
namespace {

constexpr int kWarps = 4;  // warps (= nodes in flight) per block


// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Beam search shared by cal_ep_gpu (:1905-2047) and collect_path (:1211-1335).
// The helpers below are __noinline__: the select kernel is latency-bound and
// its warps sit in different phases, so one copy of each sort and merge keeps
// the code they run small enough for the instruction cache (inlined copies
// at every call site cost 8 % of the select at 1M points).
struct Beam {
  uint32_t* id;
  float* dis;
  uint8_t* ex;
  uint32_t* hash;  // membership set of the W beam ids (open addressing)
  uint32_t hslots;  // hash slots
  float* sb;       // scratch (K): the fresh positions, then sorted entering distances
  float* sm;       // staging (W + 1): merged distances of positions 0..TOPM
  uint32_t* sid;   // staging (W + 1): their ids
  uint8_t* sex;    // staging (W + 1): their explored flags
};

// Hash slots: the beam at load <= 1/2 (TOPM <= 256, K <= 128). 384 slots keep a
// warp's beam region within its candidate list's, so six blocks per SM still
// fit the 132 KB shared-memory carveout and leave L1 its larger share.
__host__ __device__ inline uint32_t hash_slots(uint32_t W) { return W <= 192 ? 384u : 768u; }

__host__ __device__ inline size_t beam_bytes(uint32_t W) {
  return (size_t)hash_slots(W) * 4 + (size_t)W * 8 + 128 * 4 + (size_t)(W + 1) * 8 +
         ((W + 15u) & ~15u) + ((W + 16u) & ~15u);
}

__device__ inline Beam beam_carve(unsigned char* p, uint32_t W) {
  Beam b;
  b.hash = reinterpret_cast<uint32_t*>(p);
  b.hslots = hash_slots(W);
  b.id = b.hash + hash_slots(W);
  b.dis = reinterpret_cast<float*>(b.id + W);
  b.sb = b.dis + W;
  b.sm = b.sb + 128;
  b.sid = reinterpret_cast<uint32_t*>(b.sm + W + 1);
  b.ex = reinterpret_cast<uint8_t*>(b.sid + W + 1);
  b.sex = b.ex + ((W + 15u) & ~15u);
  return b;
}

__device__ __forceinline__ uint32_t hslot(uint32_t key, uint32_t slots) {
  return (uint32_t)(((uint64_t)(key * 0x9E3779B1u) * slots) >> 32);  // multiply-shift into [0, slots)
}

// The reference keeps the beam ids sorted (top_M_Cand2, :1253-1259) only to
// test membership (:1282-1290); a hash set of the same ids answers the same
// question without a sort.
__device__ __noinline__ void beam_rehash(Beam bm, uint32_t W, int lane) {
  for (uint32_t t = lane; t < bm.hslots; t += 32) bm.hash[t] = kInv;
  __syncwarp();
  for (uint32_t t = lane; t < W; t += 32) {
    const uint32_t key = bm.id[t];
    if (key == kInv) continue;
    uint32_t h = hslot(key, bm.hslots);
    while (true) {
      const uint32_t prev = atomicCAS(&bm.hash[h], kInv, key);
      if (prev == kInv || prev == key) break;
      h = h + 1 == bm.hslots ? 0u : h + 1;
    }
  }
  __syncwarp();
}

__device__ __forceinline__ bool beam_has(const Beam& bm, uint32_t key) {
  uint32_t h = hslot(key, bm.hslots);
  while (true) {
    const uint32_t v = bm.hash[h];
    if (v == key) return true;
    if (v == kInv) return false;
    h = h + 1 == bm.hslots ? 0u : h + 1;
  }
}

__device__ __noinline__ void beam_network(Beam bm, uint32_t off, uint32_t len, int lane) {
  float* D = bm.dis + off;
  uint32_t* I = bm.id + off;
  uint8_t* E = bm.ex + off;
  warp_network(len, lane, [&](uint32_t u, uint32_t d) { return D[u] > D[d]; },
               [&](uint32_t u, uint32_t d) {
                 swap_(D[u], D[d]);
                 swap_(I[u], I[d]);
                 swap_(E[u], E[d]);
               });
}

// Sorted (distance, position) keys of the n <= 128 entries at [off, off+n),
// element-major in four registers per lane.
__device__ __forceinline__ void sorted_keys(const Beam& bm, uint32_t off, uint32_t n, uint64_t (&key)[4],
                                            int lane) {
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const uint32_t j = lane + 32 * t;
    key[t] = j < n ? (((uint64_t)__float_as_uint(bm.dis[off + j]) << 32) | j) : ~0ull;
  }
  knn::warp_sort_keys<4>(key, lane);
}

__device__ __forceinline__ float key_dis(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }

// Merges the m entering entries, whose (distance, slot) keys sit in sm/sid
// [0, m), into the sorted prefix [0, topm) by rank, through the staging
// arrays. Returns false (nothing moved) when two merged positions 0..topm tie.
template <int E>
__device__ __noinline__ bool beam_merge(Beam bm, uint32_t topm, uint32_t m, int lane) {
  uint64_t key[E];
#pragma unroll
  for (int t = 0; t < E; ++t) {
    const uint32_t q = lane + 32 * t;
    key[t] = q < m ? (((uint64_t)__float_as_uint(bm.sm[q]) << 32) | bm.sid[q]) : ~0ull;
  }
  knn::warp_sort_keys<E>(key, lane);
#pragma unroll
  for (int t = 0; t < E; ++t) {
    const uint32_t q = lane + 32 * t;
    if (q < m) bm.sb[q] = key_dis(key[t]);
  }
  __syncwarp();
  // merged rank: prefix i -> i + #(entering < A_i); entering q -> q + #(prefix <= B_q)
  for (uint32_t i = lane; i < topm; i += 32) {
    const float a = bm.dis[i];
    uint32_t lo = 0, hi = m;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (bm.sb[mid] < a) lo = mid + 1;
      else hi = mid;
    }
    const uint32_t r = i + lo;
    if (r <= topm) {
      bm.sm[r] = a;
      bm.sid[r] = bm.id[i];
      bm.sex[r] = bm.ex[i];
    }
  }
#pragma unroll
  for (int t = 0; t < E; ++t) {
    const uint32_t q = lane + 32 * t;
    if (q < m) {
      const float v = key_dis(key[t]);
      uint32_t lo = 0, hi = topm;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (bm.dis[mid] <= v) lo = mid + 1;
        else hi = mid;
      }
      const uint32_t r = q + lo;
      if (r <= topm) {
        const uint32_t j = (uint32_t)(key[t] & 0xFFFFFFFFu);
        bm.sm[r] = v;
        bm.sid[r] = bm.id[topm + j];
        bm.sex[r] = bm.ex[topm + j];
      }
    }
  }
  __syncwarp();
  bool tie = false;
  for (uint32_t p = lane + 1; p <= topm; p += 32) tie |= bm.sm[p] == bm.sm[p - 1];
  if (__any_sync(kFull, tie)) return false;
  for (uint32_t i = lane; i < topm; i += 32) {
    bm.dis[i] = bm.sm[i];
    bm.id[i] = bm.sid[i];
    bm.ex[i] = bm.sex[i];
  }
  __syncwarp();
  return true;
}

// After an expansion: [0, topm) holds the previous sorted prefix, [topm, W)
// the K new entries, of which the `nfresh` at slots fresh[0, nfresh) were
// scored and the rest are beam members at INF_DIS. The reference sorts all W
// with its network; only [0, topm) and the set of the W ids survive into the
// next expansion (the rest is overwritten), and with strictly increasing
// distances over merged positions 0..topm that part is the same for every
// correct sort. With a full prefix only scored entries no farther than its
// last one can reach positions 0..topm, so just those are sorted and merged
// by rank; a tie there, or a prefix that is not full, runs the network.
__device__ __noinline__ void beam_update(Beam bm, uint32_t topm, uint32_t K, const uint32_t* fresh,
                            uint32_t nfresh, int lane) {
  const uint32_t W = topm + K;
  beam_rehash(bm, W, lane);  // the set of all W ids, before anything moves
  const float worst = bm.dis[topm - 1];
  if (topm > 128 || !(worst < kInfDis)) {
    beam_network(bm, 0, W, lane);
    return;
  }
  const unsigned below = (1u << lane) - 1u;
  uint32_t m = 0;
  for (uint32_t base = 0; base < nfresh; base += 32) {
    const uint32_t r = base + lane;
    bool enter = false;
    float d = 0.0f;
    uint32_t j = 0;
    if (r < nfresh) {
      j = fresh[r];
      d = bm.dis[topm + j];
      enter = d <= worst;
    }
    const unsigned mk = __ballot_sync(kFull, enter);
    if (enter) {
      const uint32_t q = m + __popc(mk & below);
      bm.sm[q] = d;
      bm.sid[q] = j;
    }
    m += __popc(mk);
  }
  if (m == 0) return;  // every scored entry lies beyond the prefix: nothing moves
  __syncwarp();
  bool ok;
  if (m <= 32) ok = beam_merge<1>(bm, topm, m, lane);
  else if (m <= 64) ok = beam_merge<2>(bm, topm, m, lane);
  else ok = beam_merge<4>(bm, topm, m, lane);
  if (!ok) beam_network(bm, 0, W, lane);
}

__device__ uint32_t warp_beam(const uint32_t* __restrict__ G, const __half* __restrict__ data,
                              uint32_t dim, uint32_t K, const __half* query, uint32_t start,
                              uint32_t topm, uint32_t iters, Beam bm, uint32_t* ring_id,
                              float* ring_dis, uint32_t* ring_count, int lane) {
  const uint32_t W = topm + K;
  for (uint32_t t = lane; t < W; t += 32) {
    bm.id[t] = kInv;
    bm.dis[t] = kInfDis;
    bm.ex[t] = 1;
  }
  __syncwarp();
  // Seeds: the start node's row, scored one row per lane; ring slots follow
  // the row order.
  for (uint32_t t = lane; t < K; t += 32) {
    const uint32_t a = __ldg(G + (size_t)start * K + t);
    const float d = row_dist(query, data + (size_t)a * dim, dim);
    bm.id[topm + t] = a;
    bm.ex[topm + t] = 0;
    bm.dis[topm + t] = d;
    if (ring_id) {
      ring_id[t % kSelectCand] = a;
      ring_dis[t % kSelectCand] = d;
    }
  }
  __syncwarp();
  // Seeds: the network's order is observable on the first min(TOPM, K)
  // positions, copied into the prefix; a tie there runs the network.
  const uint32_t keep = min(topm, K);
  bool seeded = false;
  if (K <= 128) {
    uint64_t key[4];
    sorted_keys(bm, topm, K, key, lane);
    bool tie = false;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const uint32_t p = lane + 32 * t;
      uint32_t prev = __shfl_up_sync(kFull, (uint32_t)(key[t] >> 32), 1);
      if (t > 0) {
        const uint32_t tail = __shfl_sync(kFull, (uint32_t)(key[t - 1] >> 32), 31);
        if (lane == 0) prev = tail;
      }
      if (p >= 1 && p <= keep && p < K && (uint32_t)(key[t] >> 32) == prev) tie = true;
    }
    if (!__any_sync(kFull, tie)) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const uint32_t p = lane + 32 * t;
        if (p < keep) {
          const uint32_t j = (uint32_t)(key[t] & 0xFFFFFFFFu);
          bm.id[p] = bm.id[topm + j];
          bm.dis[p] = key_dis(key[t]);
          bm.ex[p] = 0;
        }
      }
      for (uint32_t i = K + lane; i < topm; i += 32) {  // TOPM > K: empty slots
        bm.id[i] = kInv;
        bm.dis[i] = kInfDis;
        bm.ex[i] = 1;
      }
      seeded = true;
    }
  }
  if (!seeded) {
    beam_network(bm, topm, K, lane);
    for (uint32_t i = lane; i < topm; i += 32) {
      if (topm + i < W) {
        bm.id[i] = bm.id[topm + i];
        bm.dis[i] = bm.dis[topm + i];
        bm.ex[i] = bm.ex[topm + i];
      } else {  // slots past the K seeds start empty (TOPM > K)
        bm.id[i] = kInv;
        bm.dis[i] = kInfDis;
        bm.ex[i] = 1;
      }
    }
  }
  __syncwarp();
  beam_rehash(bm, W, lane);
  uint32_t curr = K, to_explore = kInv;
  for (uint32_t it = 0; it < iters; ++it) {
    // First unexplored of the top TOPM; when none is left the reference keeps
    // the previous node (its `j == TOPM` test never fires, :1270).
    for (uint32_t base = 0; base < topm; base += 32) {
      const uint32_t j = base + lane;
      const unsigned m = __ballot_sync(kFull, j < topm && !bm.ex[j]);
      if (m) {
        const uint32_t f = base + __ffs(m) - 1;
        to_explore = bm.id[f];
        __syncwarp();
        if (lane == 0) bm.ex[f] = 1;
        break;
      }
    }
    __syncwarp();
    if (to_explore == kInv) break;
    // Neighbours of the explored node: members of the beam keep INF_DIS; the
    // others are listed in ascending neighbour order (which fixes their ring
    // slots) and scored one row per lane.
    uint32_t* fresh_at = reinterpret_cast<uint32_t*>(bm.sb);  // K <= 128 slots
    uint32_t nfresh = 0;
    for (uint32_t base = 0; base < K; base += 32) {
      const uint32_t j = base + lane;
      bool fresh = false;
      if (j < K) {
        const uint32_t a = __ldg(G + (size_t)to_explore * K + j);
        fresh = !beam_has(bm, a);
        bm.id[topm + j] = a;
        bm.ex[topm + j] = 0;
        bm.dis[topm + j] = kInfDis;
      }
      const unsigned m = __ballot_sync(kFull, fresh);
      if (fresh) fresh_at[nfresh + __popc(m & ((1u << lane) - 1u))] = j;
      nfresh += __popc(m);
    }
    __syncwarp();
    for (uint32_t r = lane; r < nfresh; r += 32) {
      const uint32_t j = fresh_at[r];
      const uint32_t a = bm.id[topm + j];
      const float d = row_dist(query, data + (size_t)a * dim, dim);
      bm.dis[topm + j] = d;
      if (ring_id) {
        ring_id[(curr + r) % kSelectCand] = a;
        ring_dis[(curr + r) % kSelectCand] = d;
      }
    }
    curr += nfresh;
    __syncwarp();
    beam_update(bm, topm, K, fresh_at, nfresh, lane);
  }
  if (ring_count) *ring_count = curr;
  return bm.id[0];
}

// Sort by distance with the reference network, then mark adjacent repeats
// using the ids as they were before marking (:1345-1348).
__device__ __noinline__ void warp_sort_mark(uint32_t* cand, float* dis, uint32_t len, int lane) {
  warp_network(len, lane, [&](uint32_t u, uint32_t d) { return dis[u] > dis[d]; },
               [&](uint32_t u, uint32_t d) {
                 swap_(dis[u], dis[d]);
                 swap_(cand[u], cand[d]);
               });
  // Marks decided from the unmarked ids: chunks from the last to the first,
  // so a chunk's comparisons read only its own entries and the last entry of
  // the chunk before it, none of them marked yet.
  const uint32_t chunks = (len + 31) / 32;
  for (uint32_t c = chunks; c-- > 0;) {
    const uint32_t i = c * 32 + lane;
    const bool rep = i >= 1 && i < len && cand[i] == cand[i - 1];
    __syncwarp();
    if (rep) cand[i] = kInv;
  }
  __syncwarp();
}

// Position of the r-th (0-based) set bit of m; m has more than r set bits.
// Binary search on population counts: five steps whatever r is.
__device__ __forceinline__ uint32_t nth_bit(unsigned m, uint32_t r) {
  uint32_t pos = 0;
#pragma unroll
  for (int w = 16; w >= 1; w >>= 1) {
    const uint32_t c = (uint32_t)__popc(m & ((1u << w) - 1u));
    const bool skip = r >= c;
    r -= skip ? c : 0u;
    m = skip ? m >> w : m;
    pos += skip ? (uint32_t)w : 0u;
  }
  return pos;
}

// Filter stage, lazily evaluated (see file header). Returns the number of ids
// the reference stores: one less than its selection steps (:1462, :1623).
//
// The lanes work through the sorted list as a queue: each takes the next live
// candidate and tests it against the kept neighbours in order, one exact
// thread-serial distance per step, until a rule fires or it has passed them
// all. The earliest unresolved candidate that has passed is kept, in list
// order; a candidate further on that had passed must then also pass the new
// neighbour. Each candidate is thus tested against exactly the neighbours
// kept before it, as in the sequential filter.
__device__ uint32_t warp_filter(const uint32_t* cand, const float* cdis, uint32_t len,
                                uint32_t bid, uint32_t fd, int metric, float thre,
                                const __half* __restrict__ data, uint32_t dim, uint32_t* sel,
                                float* seld, int lane, uint32_t* scored = nullptr) {
  uint32_t first = kInv;
  for (uint32_t base = 0; base < len; base += 32) {
    const uint32_t i = base + lane;
    const bool ok = i < len && cand[i] != bid && cand[i] != kInv;
    const unsigned m = __ballot_sync(kFull, ok);
    if (m) {
      first = base + __ffs(m) - 1;
      break;
    }
  }
  if (first == kInv) return 0;
  if (lane == 0) {
    sel[0] = cand[first];
    seld[0] = cdis[first];
  }
  __syncwarp();
  uint32_t nsel = 1, last_pos = first, rows = 0;
  const unsigned below = (1u << lane) - 1u;
  // lane state: 0 idle, 1 testing against sel[s], 2 passed sel[0, nsel)
  int st = 0;
  uint32_t pos = kInv, c = kInv, s = 0;
  float dc = 0.0f;
  uint32_t next = first + 1;  // next list position to hand out
  while (nsel < fd) {
    unsigned idle = __ballot_sync(kFull, st == 0);
    while (idle && next < len) {
      const uint32_t p = next + lane;
      const unsigned live = __ballot_sync(kFull, p < len && cand[p] != kInv);
      const uint32_t nlive = __popc(live);
      const uint32_t take = min(nlive, (uint32_t)__popc(idle));
      if (st == 0) {
        const uint32_t r = __popc(idle & below);
        if (r < take) {
          pos = next + nth_bit(live, r);
          c = cand[pos];
          dc = cdis[pos];
          s = 0;
          st = 1;
        }
      }
      next = take == nlive ? min(len, next + 32) : next + nth_bit(live, take - 1) + 1;
      idle = __ballot_sync(kFull, st == 0);
    }
    if (!__any_sync(kFull, st != 0)) break;
    if (st == 1) {
      const uint32_t q = sel[s];
      if (q == c) {
        st = 0;  // a repeat of a kept neighbour (:1423-1427)
      } else {
        const float res = row_dist(data + (size_t)q * dim, data + (size_t)c * dim, dim);
        ++rows;
        if (pruned_by(metric, res, dc, seld[s], thre)) st = 0;
        else if (++s == nsel) st = 2;
      }
    }
    while (true) {
      const uint32_t key = st != 0 ? pos : kInv;
      const uint32_t mn = __reduce_min_sync(kFull, key);
      if (mn == kInv) break;
      const int o = __ffs(__ballot_sync(kFull, key == mn)) - 1;
      if (__shfl_sync(kFull, st, o) != 2) break;
      if (lane == o) {
        sel[nsel] = c;
        seld[nsel] = dc;
        st = 0;
      }
      __syncwarp();
      ++nsel;
      last_pos = mn;
      if (nsel == fd) break;
      if (st == 2) st = 1;  // s == nsel - 1: test the new neighbour
    }
  }
  __syncwarp();
  if (scored) *scored = __reduce_add_sync(kFull, rows);
  if (nsel == fd) return fd - 1;
  if (nsel >= 2 && last_pos == len - 1) return nsel - 1;
  return nsel;
}

// The same filter, warp-cooperative (where wide_filter picks it). A
// thread-serial distance over a wide row is a long chain of scattered 16-byte
// loads per lane; here the warp takes the candidates in list order and tests
// each against the kept neighbours G at a time with coalesced row reads,
// stopping at the first group in which a rule fires. A candidate is dropped
// when any of its tests fires, whichever fires first, so the kept set and the
// return value are those of warp_filter. G kept neighbours per step: 8 at 96 dims (warp_dist8_d96, a half-warp per
// distance), 4 otherwise (warp_dist4). DIM != 0 fixes the width at compile
// time. At 128 dims (one chunk per lane) the candidate's chunk is loaded once
// for all its tests; at 960 the eight chunks a lane would hold cost more in
// registers than their reloads (NSSG at 1M x 960: 0.80 s against 0.54 s).
template <int G, uint32_t DIM>
static __device__ __noinline__ uint32_t warp_filter_group(const uint32_t* cand, const float* cdis,
                                                          uint32_t len, uint32_t bid, uint32_t fd,
                                                          int metric, float thre,
                                                          const __half* __restrict__ data,
                                                          uint32_t dim, uint32_t* sel, float* seld,
                                                          int lane, uint32_t* scored) {
  uint32_t nsel = 0, last_pos = 0, rows = 0;
  for (uint32_t i = 0; i < len && nsel < fd; ++i) {
    const uint32_t c = cand[i];
    if (c == bid || c == kInv) continue;
    const float dc = cdis[i];
    const __half* crow = data + (size_t)c * dim;
    bool keep = true;
    constexpr bool kPreload = G == 4 && DIM != 0 && DIM <= 128;
    [[maybe_unused]] QRow<kPreload ? DIM : 4u> qr;
    if constexpr (kPreload)
      if (nsel > 0) load_qrow(crow, qr, lane);
    for (uint32_t s0 = 0; s0 < nsel && keep; s0 += G) {
      uint32_t ids[G];
      float o[G];
#pragma unroll
      for (int t = 0; t < G; ++t) {
        ids[t] = s0 + t < nsel ? sel[s0 + t] : kInv;
        if (ids[t] == c) keep = false;  // a repeat of a kept neighbour (:1423-1427)
      }
      if (!keep) break;
      if constexpr (G == 8)
        warp_dist8_d96(crow, data, ids, o, lane);
      else if constexpr (kPreload)
        warp_dist4_q<DIM>(qr, data, ids, o, lane);
      else
        warp_dist4<DIM>(crow, data, dim, ids, o, lane);
#pragma unroll
      for (int t = 0; t < G; ++t) {
        if (ids[t] == kInv) continue;
        ++rows;
        if (pruned_by(metric, o[t], dc, seld[s0 + t], thre)) keep = false;
      }
    }
    if (keep) {
      if (lane == 0) {
        sel[nsel] = c;
        seld[nsel] = dc;
      }
      __syncwarp();
      ++nsel;
      last_pos = i;
    }
  }
  __syncwarp();
  if (scored) *scored = rows;
  if (nsel == fd) return fd - 1;
  if (nsel >= 2 && last_pos == len - 1) return nsel - 1;
  return nsel;
}

// Which filter a prune runs. Measured at 1M-2M nodes: the cooperative filter
// wins wherever the thread-serial tree is not the 128-dim one (d = 96: the
// Vamana select 1,098 -> 466 ms; d = 960: NSSG 5.5 -> 0.51 s) and, at 128
// dims, where alpha > 1 keeps long lists that take many tests per candidate
// (Vamana 1.2: 262 -> 170 ms). At 128 dims with alpha 1 most candidates fall
// to their first tests, and 32 lanes each working through its own candidate
// keep more loads in flight (NSG select 203 ms against 226).
__device__ __forceinline__ bool wide_filter(uint32_t dim, int metric, float thre) {
  return dim != 128 || (metric == 0 && thre > 1.0f);
}

static __device__ __forceinline__ uint32_t warp_filter_wide(const uint32_t* cand, const float* cdis,
                                                            uint32_t len, uint32_t bid, uint32_t fd,
                                                            int metric, float thre,
                                                            const __half* __restrict__ data,
                                                            uint32_t dim, uint32_t* sel, float* seld,
                                                            int lane, uint32_t* scored) {
  if (dim == 96)
    return warp_filter_group<8, 96>(cand, cdis, len, bid, fd, metric, thre, data, dim, sel, seld,
                                    lane, scored);
  if (dim == 960)
    return warp_filter_group<4, 960>(cand, cdis, len, bid, fd, metric, thre, data, dim, sel, seld,
                                     lane, scored);
  if (dim == 128)
    return warp_filter_group<4, 128>(cand, cdis, len, bid, fd, metric, thre, data, dim, sel, seld,
                                     lane, scored);
  return warp_filter_group<4, 0>(cand, cdis, len, bid, fd, metric, thre, data, dim, sel, seld,
                                 lane, scored);
}

// Per-warp shared layout of the select kernels: the beam (path collect) and
// the candidate list share one region, since the list is filled only after
// the beam has finished (its ring of scored nodes lives in global memory).
struct SelLayout {
  uint32_t W, L, fd;
  __host__ __device__ size_t bytes() const {
    const size_t list = (size_t)L * 8 + (size_t)fd * 8;
    const size_t beam = W ? beam_bytes(W) : 0;
    return ((beam > list ? beam : list) + 64 + 15) & ~(size_t)15;
  }
};

// ---------------------------------------------------------------------------
// Processing order of the select kernels. A node's select reads only the kNN
// snapshot and writes only its own rows, so the order in which nodes are
// taken changes no result. Taking together nodes that share kNN
// neighbourhoods keeps the rows the warps in flight gather resident in L2
// (at d = 960 the base is 15x larger than L2). Labels: each node takes the
// smallest label among itself and its first kLabelHops neighbours, in place
// (labels only decrease, so concurrent updates are harmless), for
// kLabelRounds rounds; nodes of one cluster converge to a common label. The
// order is the nodes sorted by label.
constexpr uint32_t kLabelHops = 4, kLabelRounds = 16;

__global__ void k_label_init(uint32_t* __restrict__ lab, uint32_t* __restrict__ ids, uint32_t n) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    lab[u] = u;
    ids[u] = u;
  }
}

__global__ void k_label_min(const uint32_t* __restrict__ G, uint32_t K, uint32_t hops,
                            uint32_t* lab, uint32_t n) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    uint32_t m = lab[u];
    for (uint32_t j = 0; j < hops; ++j) m = min(m, lab[__ldg(G + (size_t)u * K + j)]);
    if (m < lab[u]) lab[u] = m;
  }
}

__global__ void k_validate(const uint32_t* __restrict__ g, size_t cnt, uint32_t n,
                           uint32_t* bad) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt;
       i += (size_t)gridDim.x * blockDim.x)
    if (g[i] >= n) atomicExch(bad, 1u);
}

// cal_ep_gpu (:1889-2058): one warp, 30 expansions from node 0 toward the centre.
__global__ void k_cal_ep(const uint32_t* __restrict__ G, const __half* __restrict__ data,
                         const __half* __restrict__ center, uint32_t dim, uint32_t K,
                         uint32_t topm, uint32_t* ep) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t W = topm + K;
  Beam bm = beam_carve(smem, W);
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  const uint32_t best = warp_beam(G, data, dim, K, center, 0, topm, 30, bm, nullptr, nullptr,
                                  nullptr, lane);
  if (lane == 0) *ep = best;
}

// select_path (:1498-1517) and select_2hop (:1520-1534) into scratch rows.
// path: collect_path + Filter_path(distance_filter); 2-hop: collect_2hop +
// Filter_path(angle_filter). The reference always uses these two filters.
// Node handed to this warp: one shared counter, taken a node at a time, keeps
// the SMs busy to the end whatever the per-node search length.
__device__ __forceinline__ uint32_t next_node(uint32_t* ctr, int lane) {
  uint32_t b = 0;
  if (lane == 0) b = atomicAdd(ctr, 1u);
  return __shfl_sync(kFull, b, 0);
}
// The node at position i of the processing order (identity without one).
__device__ __forceinline__ uint32_t node_at(const uint32_t* __restrict__ order, uint32_t i) {
  return order ? __ldg(order + i) : i;
}

// ring_ids / ring_dis: per-warp rings of kSelectCand scored nodes (path
// collect), indexed by the warp's global number.
template <bool kPath>
__global__ void __launch_bounds__(kWarps * 32, 6)
    k_select(const uint32_t* __restrict__ G, float* __restrict__ nd, const __half* __restrict__ data,
             uint32_t n, uint32_t dim, uint32_t K, const uint32_t* __restrict__ ep_dev,
             uint32_t* __restrict__ ctr, uint32_t topm, uint32_t fd, float thre,
             uint32_t* __restrict__ P_ids, float* __restrict__ P_dis, uint32_t* __restrict__ P_cnt,
             unsigned long long* __restrict__ work, uint32_t* __restrict__ ring_ids,
             float* __restrict__ ring_dis, const uint32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  SelLayout lay{kPath ? topm + K : 0u, kSelectCand + K, fd};
  unsigned char* mine = smem + (size_t)warp * lay.bytes();
  uint32_t* cand = reinterpret_cast<uint32_t*>(mine);
  float* cdis = reinterpret_cast<float*>(cand + lay.L);
  uint32_t* sel = reinterpret_cast<uint32_t*>(cdis + lay.L);
  float* seld = reinterpret_cast<float*>(sel + fd);
  Beam bm = beam_carve(mine, lay.W);  // same region as the list, used before it
  const size_t gw = (size_t)blockIdx.x * kWarps + warp;
  uint32_t* rid = kPath ? ring_ids + gw * kSelectCand : nullptr;
  float* rds = kPath ? ring_dis + gw * kSelectCand : nullptr;
  const uint32_t L = lay.L;
  const uint32_t ep = kPath ? *ep_dev : 0u;
  for (uint32_t pos = next_node(ctr, lane); pos < n; pos = next_node(ctr, lane)) {
    const uint32_t b = node_at(order, pos);
    const __half* q = data + (size_t)b * dim;
    uint32_t scored = kSelectCand;  // rows scored for this node (2-hop: the 480 collected)
    if (kPath) {
      uint32_t curr = 0;
      warp_beam(G, data, dim, K, q, ep, topm, 10, bm, rid, rds, &curr, lane);
      scored = curr;
      __syncwarp();  // the ring (global) and the beam's region are done
      for (uint32_t i = lane; i < kSelectCand; i += 32) {
        const bool in = i < curr;
        cand[K + i] = in ? rid[i] : kInv;
        cdis[K + i] = in ? rds[i] : kInfDis;
      }
    } else {
      for (uint32_t i = lane; i < kSelectCand; i += 32)
        cand[K + i] = __ldg(G + (size_t)__ldg(G + (size_t)b * K + i / K) * K + i % K);
      __syncwarp();
      // The two-hop rows are scored four at a time by the whole warp: each
      // lane reads its 8-byte chunks of four rows at once (coalesced across
      // the warp) and the four shuffle trees interleave. Same lane order as
      // the thread-serial distance, so the same values.
      auto score = [&](auto&& dist4) {
        for (uint32_t i = 0; i < kSelectCand; i += 4) {
          const uint32_t ids[4] = {cand[K + i], cand[K + i + 1], cand[K + i + 2], cand[K + i + 3]};
          float o[4];
          dist4(ids, o);
          if (lane < 4)
            cdis[K + i + lane] = lane == 0 ? o[0] : lane == 1 ? o[1] : lane == 2 ? o[2] : o[3];
        }
      };
      if (dim == 960) {
        score([&](const uint32_t* ids, float* o) { warp_dist4<960>(q, data, dim, ids, o, lane); });
      } else {
        score([&](const uint32_t* ids, float* o) { warp_dist4(q, data, dim, ids, o, lane); });
      }
    }
    for (uint32_t i = lane; i < K; i += 32) {
      cand[i] = __ldg(G + (size_t)b * K + i);
      cdis[i] = nd[(size_t)b * K + i];
    }
    __syncwarp();
    warp_sort_mark(cand, cdis, L, lane);
    uint32_t filtered = 0;
    const uint32_t stored =
        wide_filter(dim, kPath ? 0 : 1, thre)
            ? warp_filter_wide(cand, cdis, L, b, fd, kPath ? 0 : 1, thre, data, dim, sel, seld,
                               lane, &filtered)
            : warp_filter(cand, cdis, L, b, fd, kPath ? 0 : 1, thre, data, dim, sel, seld, lane,
                          &filtered);
    if (work && lane == 0) atomicAdd(work, (unsigned long long)(scored + filtered));
    for (uint32_t i = lane; i < stored; i += 32) {
      P_ids[(size_t)b * fd + i] = sel[i];
      P_dis[(size_t)b * fd + i] = seld[i];
      nd[(size_t)b * K + i] = seld[i];  // own row only: no other block reads it
    }
    if (lane == 0) P_cnt[b] = stored;
    __syncwarp();
  }
}

// filter_reverse (:1537-1657) plus the in-place row writes of the select
// kernels (:1462-1464, :1477): the stored row is the kNN row overwritten by
// the select result, then by this stage's result.
__global__ void __launch_bounds__(kWarps * 32)
    k_filter_reverse(uint32_t* __restrict__ graph, const float* __restrict__ nd,
                     const uint32_t* __restrict__ rg, const float* __restrict__ rd,
                     const uint32_t* __restrict__ rnum, const __half* __restrict__ data,
                     uint32_t n, uint32_t dim, uint32_t K, uint32_t fd, int metric, float thre,
                     const uint32_t* __restrict__ P_ids, const uint32_t* __restrict__ P_cnt,
                     const uint32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t cap = fd + K;  // cur_num <= fd - 1, rever_num <= K
  unsigned char* mine = smem + (size_t)warp * ((size_t)cap * 8 + (size_t)fd * 8 + 16);
  uint32_t* cand = reinterpret_cast<uint32_t*>(mine);
  float* cdis = reinterpret_cast<float*>(cand + cap);
  uint32_t* sel = reinterpret_cast<uint32_t*>(cdis + cap);
  float* seld = reinterpret_cast<float*>(sel + fd);
  for (uint32_t pos = blockIdx.x * kWarps + warp; pos < n; pos += gridDim.x * kWarps) {
    const uint32_t b = node_at(order, pos);
    const uint32_t cur_num = P_cnt[b];
    const uint32_t rn = min(K, rnum[b]);
    const uint32_t len = cur_num + rn;
    for (uint32_t i = lane; i < cur_num; i += 32) {
      cand[i] = P_ids[(size_t)b * fd + i];
      cdis[i] = nd[(size_t)b * K + i];
    }
    for (uint32_t i = lane; i < rn; i += 32) {
      cand[cur_num + i] = rg[(size_t)b * K + i];
      cdis[cur_num + i] = rd[(size_t)b * kReserve + i];
    }
    __syncwarp();
    uint32_t* row = graph + (size_t)b * K;
    uint32_t out_cnt;
    if (len > fd) {
      warp_sort_mark(cand, cdis, len, lane);
      out_cnt = wide_filter(dim, metric, thre)
                    ? warp_filter_wide(cand, cdis, len, b, fd, metric, thre, data, dim, sel, seld,
                                       lane, nullptr)
                    : warp_filter(cand, cdis, len, b, fd, metric, thre, data, dim, sel, seld, lane);
    } else {
      // Union in ascending reverse-slot order (:1632-1647).
      for (uint32_t i = lane; i < cur_num; i += 32) sel[i] = cand[i];
      uint32_t dup = 0;
      for (uint32_t i = 0; i < rn; ++i) {
        const uint32_t r = cand[cur_num + i];
        bool found = false;
        for (uint32_t j0 = 0; j0 < cur_num; j0 += 32) {
          const uint32_t j = j0 + lane;
          if (__any_sync(kFull, j < cur_num && cand[j] == r)) {
            found = true;
            break;
          }
        }
        // A stride-K row holds at most K-1 ids; with FINAL_DEGREE == K the
        // reference would spill its last union id into the next row.
        if (!found && cur_num + dup + 1 < K) {
          if (lane == 0) sel[cur_num + dup] = r;
          ++dup;
        }
      }
      out_cnt = cur_num + dup;
    }
    __syncwarp();
    const uint32_t top = max(out_cnt, cur_num);
    for (uint32_t i = lane; i < top; i += 32)
      row[i + 1] = (i < out_cnt) ? sel[i] : P_ids[(size_t)b * fd + i];
    if (lane == 0) row[0] = out_cnt;
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Rank-based prunes. collect_1hop + filter_cagra (:1660-1710): detour[m]
// counts the kept-earlier neighbours a whose own list holds n_m, over the
// pairs the reference visits (a in {i, K-1-i : i < K/2}, m > a).
__global__ void __launch_bounds__(kWarps * 32)
    k_select_cagra(const uint32_t* __restrict__ G, uint32_t n, uint32_t K, uint32_t d,
                   uint32_t* __restrict__ hybrid, uint32_t* __restrict__ E_tgt,
                   uint32_t* __restrict__ E_val, const uint32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr uint32_t H = 256;  // hash slots, K <= 128 keeps the load <= 1/2
  unsigned char* mine = smem + (size_t)warp * (H * 4 + (size_t)K * 8);
  uint32_t* hash = reinterpret_cast<uint32_t*>(mine);
  uint32_t* nei0 = hash + H;
  uint32_t* det = nei0 + K;
  for (uint32_t pos = blockIdx.x * kWarps + warp; pos < n; pos += gridDim.x * kWarps) {
    const uint32_t b = node_at(order, pos);
    for (uint32_t j = lane; j < K; j += 32) {
      nei0[j] = __ldg(G + (size_t)b * K + j);
      det[j] = 0;
    }
    __syncwarp();
    for (uint32_t i = 0; i < K / 2; ++i) {
      for (int side = 0; side < 2; ++side) {
        const uint32_t a = side ? (K - 1 - i) : i;
        if (a + 1 >= K) continue;
        for (uint32_t t = lane; t < H; t += 32) hash[t] = kInv;
        __syncwarp();
        const uint32_t* row = G + (size_t)nei0[a] * K;
        for (uint32_t j = lane; j < K; j += 32) {
          const uint32_t key = __ldg(row + j);
          uint32_t h = (key * 0x9E3779B1u) >> 24;
          while (true) {
            const uint32_t prev = atomicCAS(&hash[h], kInv, key);
            if (prev == kInv || prev == key) break;
            h = (h + 1) & (H - 1);
          }
        }
        __syncwarp();
        for (uint32_t m = a + 1 + lane; m < K; m += 32) {
          const uint32_t key = nei0[m];
          uint32_t h = (key * 0x9E3779B1u) >> 24;
          bool hit = false;
          while (true) {
            const uint32_t v = hash[h];
            if (v == key) {
              hit = true;
              break;
            }
            if (v == kInv) break;
            h = (h + 1) & (H - 1);
          }
          if (hit) det[m] += 1;  // m is owned by this lane
        }
        __syncwarp();
      }
    }
    warp_network(K, lane, [&](uint32_t u, uint32_t v) { return det[u] > det[v]; },
                 [&](uint32_t u, uint32_t v) {
                   swap_(det[u], det[v]);
                   swap_(nei0[u], nei0[v]);
                 });
    for (uint32_t i = lane; i < d; i += 32) {
      E_tgt[(size_t)b * d + i] = nei0[i];
      E_val[(size_t)b * d + i] = det[i];
      hybrid[(size_t)b * K + i] = nei0[i];
    }
    __syncwarp();
  }
}

// collect_1hop + filter_dpg (:1713-1785): detour[m] counts earlier a with
// d(n_a, n_m) < d(u, n_m), each warp using its own vector (see header note).
__global__ void __launch_bounds__(kWarps * 32)
    k_select_dpg(const uint32_t* __restrict__ G, const float* __restrict__ nd,
                 const __half* __restrict__ data, uint32_t n, uint32_t dim, uint32_t K, uint32_t d,
                 uint32_t* __restrict__ hybrid, uint32_t* __restrict__ E_tgt,
                 uint32_t* __restrict__ E_val, const uint32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned char* mine = smem + (size_t)warp * ((size_t)K * 12);
  uint32_t* nei0 = reinterpret_cast<uint32_t*>(mine);
  uint32_t* det = nei0 + K;
  float* nrow = reinterpret_cast<float*>(det + K);
  for (uint32_t pos = blockIdx.x * kWarps + warp; pos < n; pos += gridDim.x * kWarps) {
    const uint32_t b = node_at(order, pos);
    for (uint32_t j = lane; j < K; j += 32) {
      nei0[j] = __ldg(G + (size_t)b * K + j);
      det[j] = 0;
      nrow[j] = nd[(size_t)b * K + j];
    }
    __syncwarp();
    for (uint32_t i = 0; i < K / 2; ++i) {
      for (int side = 0; side < 2; ++side) {
        const uint32_t a = side ? (K - 1 - i) : i;
        const uint32_t m0 = side ? (K - i) : (i + 1);
        const __half* qa = data + (size_t)nei0[a] * dim;
        for (uint32_t m = m0; m < K; m += 4) {
          uint32_t ids[4];
          float r4[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) ids[t] = (m + t < K) ? nei0[m + t] : kInv;
          warp_dist4(qa, data, dim, ids, r4, lane);
          if (lane == 0) {
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if (m + t < K && r4[t] < nrow[m + t]) det[m + t] += 1;
          }
          __syncwarp();
        }
      }
    }
    warp_network(K, lane, [&](uint32_t u, uint32_t v) { return det[u] > det[v]; },
                 [&](uint32_t u, uint32_t v) {
                   swap_(det[u], det[v]);
                   swap_(nei0[u], nei0[v]);
                 });
    for (uint32_t i = lane; i < d; i += 32) {
      E_tgt[(size_t)b * d + i] = nei0[i];
      E_val[(size_t)b * d + i] = det[i];
      hybrid[(size_t)b * K + i] = nei0[i];
    }
    __syncwarp();
  }
}

// The same select for wide rows, one node per block. The node's K neighbour
// rows (123 KB at K = 64, d = 960) are read by all K(K-1)/2 pair distances;
// with one 1,024-thread block per SM they stay in that SM's L1 while its 32
// warps share the pairs. Work items are (a, m0): row a against the four rows
// m0..m0+3 (m > a), over the reference's pair set (a < K/2 from the front,
// a >= K - K/2 from the back, :1715-1717); detour counts are shared-memory
// integer atomics, so the order of the items changes no count.
constexpr int kDpgThreads = 1024;

__global__ void __launch_bounds__(kDpgThreads, 1)
    k_select_dpg_block(const uint32_t* __restrict__ G, const float* __restrict__ nd,
                       const __half* __restrict__ data, uint32_t n, uint32_t dim, uint32_t K,
                       uint32_t d, uint32_t* __restrict__ hybrid, uint32_t* __restrict__ E_tgt,
                       uint32_t* __restrict__ E_val, const uint32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kBlockWarps = kDpgThreads / 32;
  uint32_t* nei0 = reinterpret_cast<uint32_t*>(smem);
  uint32_t* det = nei0 + K;
  float* nrow = reinterpret_cast<float*>(det + K);
  uint16_t* items = reinterpret_cast<uint16_t*>(nrow + K);  // (a << 8) | m0
  __shared__ uint32_t n_items;
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t a = 0; a + 1 < K; ++a) {
      if (a >= K / 2 && a < K - K / 2) continue;  // the middle row of an odd K (:1715-1717)
      for (uint32_t m0 = a + 1; m0 < K; m0 += 4) items[t++] = (uint16_t)((a << 8) | m0);
    }
    n_items = t;
  }
  __syncthreads();
  const uint32_t T = n_items;
  for (uint32_t pos = blockIdx.x; pos < n; pos += gridDim.x) {
    const uint32_t b = node_at(order, pos);
    for (uint32_t j = threadIdx.x; j < K; j += kDpgThreads) {
      nei0[j] = __ldg(G + (size_t)b * K + j);
      det[j] = 0;
      nrow[j] = nd[(size_t)b * K + j];
    }
    __syncthreads();
    for (uint32_t t = warp; t < T; t += kBlockWarps) {
      const uint32_t a = items[t] >> 8, m0 = items[t] & 0xFFu;
      uint32_t ids[4];
      float r4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) ids[q] = (m0 + q < K) ? nei0[m0 + q] : kInv;
      if (dim == 960)
        warp_dist4<960>(data + (size_t)nei0[a] * dim, data, dim, ids, r4, lane);
      else
        warp_dist4(data + (size_t)nei0[a] * dim, data, dim, ids, r4, lane);
      if (lane < 4 && m0 + lane < K) {
        const float r = lane == 0 ? r4[0] : lane == 1 ? r4[1] : lane == 2 ? r4[2] : r4[3];
        if (r < nrow[m0 + lane]) atomicAdd(&det[m0 + lane], 1u);
      }
    }
    __syncthreads();
    if (warp == 0) {
      warp_network(K, lane, [&](uint32_t u, uint32_t v) { return det[u] > det[v]; },
                   [&](uint32_t u, uint32_t v) {
                     swap_(det[u], det[v]);
                     swap_(nei0[u], nei0[v]);
                   });
      for (uint32_t i = lane; i < d; i += 32) {
        E_tgt[(size_t)b * d + i] = nei0[i];
        E_val[(size_t)b * d + i] = det[i];
        hybrid[(size_t)b * K + i] = nei0[i];
      }
    }
    __syncthreads();
  }
}

// filter_reverse_1hop (:1812-1886): dense stride-d rows written over the
// graph buffer (no kernel of this stage reads it), first d/2 forward,
// then reverse ids by ascending detour that are not already forward, then the
// remaining forward ids.
__global__ void __launch_bounds__(kWarps * 32)
    k_filter_reverse_1hop(uint32_t* __restrict__ out, const uint32_t* __restrict__ rg,
                          const uint32_t* __restrict__ rnum, const uint32_t* __restrict__ hybrid,
                          uint32_t n, uint32_t K, uint32_t d) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned char* mine = smem + (size_t)warp * ((size_t)d * 16);
  uint32_t* rev = reinterpret_cast<uint32_t*>(mine);
  uint32_t* rdet = rev + d;
  uint32_t* nid = rdet + d;
  uint32_t* row = nid + d;
  for (uint32_t b = blockIdx.x * kWarps + warp; b < n; b += gridDim.x * kWarps) {
    const uint32_t rn = min(d, rnum[b]);
    for (uint32_t i = lane; i < rn; i += 32) {
      rev[i] = rg[(size_t)b * d * 2 + i * 2];
      rdet[i] = rg[(size_t)b * d * 2 + i * 2 + 1];
    }
    for (uint32_t i = lane; i < d; i += 32) nid[i] = hybrid[(size_t)b * K + i];
    __syncwarp();
    warp_network(rn, lane, [&](uint32_t u, uint32_t v) { return rev[u] > rev[v]; },
                 [&](uint32_t u, uint32_t v) {
                   swap_(rev[u], rev[v]);
                   swap_(rdet[u], rdet[v]);
                 });
    {
      unsigned marks[4];
      for (uint32_t c = 0; c * 32 < rn; ++c) {
        const uint32_t i = c * 32 + lane;
        marks[c] = __ballot_sync(kFull, i >= 1 && i < rn && rev[i] == rev[i - 1]);
      }
      __syncwarp();
      for (uint32_t c = 0; c * 32 < rn; ++c)
        if ((marks[c] >> lane) & 1u) rdet[c * 32 + lane] = kInv;
      __syncwarp();
    }
    for (uint32_t i = lane; i < d / 2; i += 32) row[i] = nid[i];
    warp_network(rn, lane, [&](uint32_t u, uint32_t v) { return rdet[u] > rdet[v]; },
                 [&](uint32_t u, uint32_t v) {
                   swap_(rdet[u], rdet[v]);
                   swap_(rev[u], rev[v]);
                 });
    uint32_t cnt = 0;
    const uint32_t span = (rn < d / 2) ? (d - rn) : (d / 2);
    for (uint32_t i = 0; i < rn; ++i) {
      if (rn >= d / 2 && cnt >= d / 2) break;
      const uint32_t r = rev[i];
      bool flag = false;
      for (uint32_t j0 = 0; j0 < span; j0 += 32) {
        const uint32_t j = j0 + lane;
        if (__any_sync(kFull, j < span && nid[j] == r)) {
          flag = true;
          break;
        }
      }
      if (!flag) {
        if (lane == 0) row[d / 2 + cnt] = r;
        ++cnt;
      }
    }
    __syncwarp();
    const uint32_t m = min(cnt, d / 2);
    for (uint32_t i = lane; i < d / 2 - m; i += 32) row[d / 2 + m + i] = nid[i + d / 2];
    __syncwarp();
    const uint32_t written = 2 * (d / 2);
    for (uint32_t i = lane; i < written; i += 32) out[(size_t)b * d + i] = row[i];
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Deterministic reverse-edge store. Edges e = src * stride + i are sorted by
// target with a stable radix sort, so each target's edges come in ascending
// (source, i). Slot s of a target then receives, in that order, the inserts
// whose running count c satisfies c == s (direct, c < cap) or c % mod == s
// (replacement, c >= cap), as in the sequential reading of :1465-1475 and
// :1697-1707.
__global__ void k_edge_keys(const uint32_t* __restrict__ E_tgt, const uint32_t* __restrict__ cnt,
                            uint32_t n, uint32_t stride, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, uint32_t* __restrict__ deg) {
  const size_t total = (size_t)n * stride;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint32_t src = (uint32_t)(e / stride), i = (uint32_t)(e % stride);
    const bool valid = cnt ? (i < cnt[src]) : true;
    const uint32_t t = valid ? E_tgt[e] : n;
    keys[e] = t;
    vals[e] = (uint32_t)e;
    if (valid) atomicAdd(&deg[t], 1u);
  }
}

// mode 0: (id, f32 dist) into rg[t*K+s], rd[t*128+s], replace when closer.
// mode 1: (id, u32 detour) pairs into rg[t*2d + 2s], replace when fewer detours.
template <int kMode>
__global__ void k_reverse_fill(const uint32_t* __restrict__ sorted_e,
                               const uint32_t* __restrict__ deg, const uint32_t* __restrict__ off,
                               const uint32_t* __restrict__ E_val, uint32_t n, uint32_t stride,
                               uint32_t cap, uint32_t mod, uint32_t K, uint32_t* __restrict__ rg,
                               float* __restrict__ rd, uint32_t* __restrict__ rnum) {
  const int lane = threadIdx.x & 31;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n;
       t += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t c0 = rnum[t], dg = deg[t], o = off[t];
    for (uint32_t s = lane; s < mod; s += 32) {
      uint32_t cur_id, cur_v;
      if (kMode == 0) {
        cur_id = rg[(size_t)t * K + s];
        cur_v = __float_as_uint(rd[(size_t)t * kReserve + s]);
      } else {
        cur_id = rg[(size_t)t * mod * 2 + 2 * s];
        cur_v = rg[(size_t)t * mod * 2 + 2 * s + 1];
      }
      bool touched = false;
      // smallest c >= c0 with c % mod == s
      uint32_t c = (c0 <= s) ? s : (s + ((c0 - s + mod - 1) / mod) * mod);
      for (; c < c0 + dg; c += mod) {
        const uint32_t e = sorted_e[o + (c - c0)];
        const uint32_t src = e / stride, v = E_val[e];
        bool take;
        if (c < cap) take = true;
        else if (kMode == 0) take = __uint_as_float(v) < __uint_as_float(cur_v);
        else take = cur_v > v;
        if (take) {
          cur_id = src;
          cur_v = v;
          touched = true;
        }
      }
      if (touched) {
        if (kMode == 0) {
          rg[(size_t)t * K + s] = cur_id;
          rd[(size_t)t * kReserve + s] = __uint_as_float(cur_v);
        } else {
          rg[(size_t)t * mod * 2 + 2 * s] = cur_id;
          rg[(size_t)t * mod * 2 + 2 * s + 1] = cur_v;
        }
      }
    }
    __syncwarp();
    if (lane == 0) rnum[t] = c0 + dg;
  }
}

int grid_for(uint32_t items_per_block, uint64_t items) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t need = (items + items_per_block - 1) / items_per_block;
  const uint64_t cap = (uint64_t)sms * 16;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(need, cap));
}

int reverse_store(const Dev& d, const uint32_t* E_tgt, const uint32_t* E_val, const uint32_t* cnt,
                  uint32_t stride, int mode, uint32_t cap, uint32_t mod, cudaStream_t s) {
  const size_t E = (size_t)d.n * stride;
  if (E >= 0xFFFFFFFFull) return fail(TAGORE_EINVAL, "too many reverse edges (%zu)", E);
  int end_bit = 1;
  while (end_bit < 32 && ((uint64_t)1 << end_bit) <= d.n) ++end_bit;
  size_t sort_tmp = 0, scan_tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (uint32_t*)nullptr, (uint32_t*)nullptr, (int)E, 0, end_bit, s);
  cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                (int)d.n, s);
  const size_t tmp = std::max(sort_tmp, scan_tmp);
  Scratch sc(s);
  const size_t bytes = E * 16 + (size_t)d.n * 8 + tmp + 256;
  TG_TRY(sc.alloc(bytes));
  uint32_t* keys = sc.as<uint32_t>();
  uint32_t* vals = keys + E;
  uint32_t* keys2 = vals + E;
  uint32_t* vals2 = keys2 + E;
  uint32_t* deg = vals2 + E;
  uint32_t* off = deg + d.n;
  void* tmp_p = reinterpret_cast<void*>(((uintptr_t)(off + d.n) + 255) & ~(uintptr_t)255);
  TG_CUDA(cudaMemsetAsync(deg, 0, (size_t)d.n * 4, s));
  k_edge_keys<<<grid_for(256, E), 256, 0, s>>>(E_tgt, cnt, d.n, stride, keys, vals, deg);
  TG_CUDA(cudaGetLastError());
  size_t t1 = tmp;
  TG_CUDA(cub::DeviceScan::ExclusiveSum(tmp_p, t1, deg, off, (int)d.n, s));
  t1 = tmp;
  TG_CUDA(cub::DeviceRadixSort::SortPairs(tmp_p, t1, keys, keys2, vals, vals2, (int)E, 0, end_bit,
                                          s));
  const int grid = grid_for(8, d.n);
  if (mode == 0)
    k_reverse_fill<0><<<grid, 256, 0, s>>>(vals2, deg, off, E_val, d.n, stride, cap, mod, d.k,
                                           d.rgraph, d.rd, d.rnum);
  else
    k_reverse_fill<1><<<grid, 256, 0, s>>>(vals2, deg, off, E_val, d.n, stride, cap, mod, d.k,
                                           d.rgraph, d.rd, d.rnum);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

int validate(const Dev& d, cudaStream_t s) {
  Scratch sc(s);
  TG_TRY(sc.alloc(4));
  TG_CUDA(cudaMemsetAsync(sc.p, 0, 4, s));
  const size_t cnt = (size_t)d.n * d.k;
  k_validate<<<grid_for(256, cnt), 256, 0, s>>>(d.graph, cnt, d.n, sc.as<uint32_t>());
  TG_CUDA(cudaGetLastError());
  uint32_t bad = 0;
  TG_CUDA(cudaMemcpyAsync(&bad, sc.p, 4, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  if (bad) return fail(TAGORE_EINVAL, "graph holds an id >= POINTS (%u)", d.n);
  return TAGORE_OK;
}

int check_shape(const Dev& d, uint32_t fd) {
  if (d.n == 0 || d.k == 0 || d.dim == 0) return fail(TAGORE_EINVAL, "empty graph");
  if (d.dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", d.dim);
  if (d.k > 128) return fail(TAGORE_EINVAL, "K must be <= 128 (got %u)", d.k);
  if (fd == 0 || fd > d.k) return fail(TAGORE_EINVAL, "FINAL_DEGREE must be in [1, K]");
  return TAGORE_OK;
}

// One wave of resident blocks (SMs x blocks per SM at this shared-memory
// size), fewer when the items do not fill it.
int resident_grid(const void* fn, int threads, size_t smem, uint32_t items_per_block,
                  uint64_t items, int* grid) {
  int dev = 0, sms = 0, per_sm = 0;
  TG_CUDA(cudaGetDevice(&dev));
  TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  TG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  if (per_sm < 1) return fail(TAGORE_EINVAL, "kernel does not fit on an SM (%zu B shared)", smem);
  const uint64_t need = (items + items_per_block - 1) / items_per_block;
  *grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)sms * per_sm));
  return TAGORE_OK;
}

int set_smem(const void* fn, size_t bytes) {
  if (bytes > 227 * 1024) return fail(TAGORE_EINVAL, "shared memory request too large (%zu)", bytes);
  TG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return TAGORE_OK;
}

// Select (path or 2-hop) + reverse store + filter_reverse.
// The select's processing order (see k_label_min), in scratch `sc`.
int locality_order(const Dev& d, Scratch& sc, const uint32_t** order, cudaStream_t s) {
  const uint32_t n = d.n, hops = std::min(kLabelHops, d.k);
  int end_bit = 1;
  while (end_bit < 32 && ((uint64_t)1 << end_bit) <= n) ++end_bit;
  size_t tmp = 0;
  TG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                          (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0,
                                          end_bit, s));
  TG_TRY(sc.alloc((size_t)n * 16 + tmp + 256));
  uint32_t* lab = sc.as<uint32_t>();
  uint32_t* ids = lab + n;
  uint32_t* lab2 = ids + n;
  uint32_t* out = lab2 + n;
  void* tmp_p = reinterpret_cast<char*>(out + n) + (256 - ((uintptr_t)(out + n) & 255)) % 256;
  const int g = grid_for(256, n);
  k_label_init<<<g, 256, 0, s>>>(lab, ids, n);
  count_launch();
  for (uint32_t r = 0; r < kLabelRounds; ++r) {
    k_label_min<<<g, 256, 0, s>>>(d.graph, d.k, hops, lab, n);
    count_launch();
  }
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cub::DeviceRadixSort::SortPairs(tmp_p, tmp, lab, lab2, ids, out, (int)n, 0, end_bit, s));
  *order = out;
  return TAGORE_OK;
}

int run_dist_prune(const Dev& d, const PruneArgs& a, bool path, int metric, uint32_t* ep_host,
                   cudaStream_t s) {
  const uint32_t fd = a.final_degree, K = d.k;
  if (!path && K * K < kSelectCand) return fail(TAGORE_EINVAL, "2-hop collect needs K*K >= 480");
  if (path && (a.topm == 0 || a.topm > 256)) return fail(TAGORE_EINVAL, "TOPM must be in [1, 256]");
  Scratch sc(s);
  TG_TRY(sc.alloc(16 + (size_t)d.n * fd * 8 + (size_t)d.n * 4));
  // [u64 rows scored][u32 entry point][u32 node counter] | select rows
  unsigned long long* work = sc.as<unsigned long long>();
  uint32_t* ep_dev = reinterpret_cast<uint32_t*>(work + 1);
  uint32_t* P_ids = ep_dev + 2;
  float* P_dis = reinterpret_cast<float*>(P_ids + (size_t)d.n * fd);
  uint32_t* P_cnt = reinterpret_cast<uint32_t*>(P_dis + (size_t)d.n * fd);
  if (path) {
    const uint32_t W = a.topm + K;
    const size_t sm = beam_bytes(W) + 64;
    TG_TRY(set_smem((const void*)k_cal_ep, sm));
    stage_begin("prune_cal_ep", s);
    k_cal_ep<<<1, 32, sm, s>>>(d.graph, d.data, d.center, d.dim, K, a.topm, ep_dev);
    count_launch();
    stage_end("prune_cal_ep", s);
    TG_CUDA(cudaGetLastError());
  }
  SelLayout lay{path ? a.topm + K : 0u, kSelectCand + K, fd};
  const size_t sm = lay.bytes() * kWarps;
  const void* fn = path ? (const void*)k_select<true> : (const void*)k_select<false>;
  TG_TRY(set_smem(fn, sm));
  int grid = 0;
  TG_TRY(resident_grid(fn, kWarps * 32, sm, kWarps, d.n, &grid));
  Scratch rings(s);
  if (path) TG_TRY(rings.alloc((size_t)grid * kWarps * kSelectCand * 8));
  uint32_t* ring_ids = path ? rings.as<uint32_t>() : nullptr;
  float* ring_dis =
      path ? reinterpret_cast<float*>(ring_ids + (size_t)grid * kWarps * kSelectCand) : nullptr;
  uint32_t* ctr = ep_dev + 1;
  TG_CUDA(cudaMemsetAsync(work, 0, 8, s));
  TG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t), s));
  Scratch ord(s);
  const uint32_t* order = nullptr;
  stage_begin("prune_order", s);
  TG_TRY(locality_order(d, ord, &order, s));
  stage_end("prune_order", s);
  const char* sel_name = path ? "prune_select_path" : "prune_select_2hop";
  stage_begin(sel_name, s);
  if (path)
    k_select<true><<<grid, kWarps * 32, sm, s>>>(d.graph, d.nd, d.data, d.n, d.dim, K, ep_dev, ctr,
                                                 a.topm, fd, a.thre, P_ids, P_dis, P_cnt, work,
                                                 ring_ids, ring_dis, order);
  else
    k_select<false><<<grid, kWarps * 32, sm, s>>>(d.graph, d.nd, d.data, d.n, d.dim, K, ep_dev,
                                                  ctr, a.topm, fd, a.thre, P_ids, P_dis, P_cnt,
                                                  work, nullptr, nullptr, order);
  count_launch();
  stage_end(sel_name, s);
  TG_CUDA(cudaGetLastError());
  stage_begin("prune_reverse_store", s);
  TG_TRY(reverse_store(d, P_ids, reinterpret_cast<const uint32_t*>(P_dis), P_cnt, fd, 0, K, K, s));
  stage_end("prune_reverse_store", s);
  const size_t sm2 = ((size_t)(fd + K) * 8 + (size_t)fd * 8 + 16) * kWarps;
  TG_TRY(set_smem((const void*)k_filter_reverse, sm2));
  stage_begin("prune_filter_reverse", s);
  k_filter_reverse<<<grid, kWarps * 32, sm2, s>>>(d.graph, d.nd, d.rgraph, d.rd, d.rnum, d.data,
                                                  d.n, d.dim, K, fd, metric, a.thre, P_ids, P_cnt,
                                                  order);
  count_launch();
  stage_end("prune_filter_reverse", s);
  TG_CUDA(cudaGetLastError());
  if (path && ep_host) {
    TG_CUDA(cudaMemcpyAsync(ep_host, ep_dev, 4, cudaMemcpyDeviceToHost, s));
  }
  unsigned long long rows = 0;
  if (profiling()) TG_CUDA(cudaMemcpyAsync(&rows, work, 8, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  // select traffic: every scored row (2d bytes), the kNN row and distances
  // read (8 B per slot), the selected ids and distances written (8 B each)
  if (profiling())
    stage_add(sel_name, rows * 2ull * d.dim + (uint64_t)d.n * (8ull * K + 8ull * fd + 4), d.n);
  return TAGORE_OK;
}

int run_rank_prune(const Dev& d, const PruneArgs& a, bool dpg, cudaStream_t s) {
  const uint32_t K = d.k, dd = a.final_degree;
  if (2 * dd > kReserve) return fail(TAGORE_EINVAL, "degree must be <= 64 for rank prunes");
  uint32_t cap = dd;
  if (dpg) {
    if (K < dd + 1 || K - dd - 1 > dd)
      return fail(TAGORE_EINVAL,
                  "DPG needs degree+1 <= K <= 2*degree+1 (the reference's reverse rows overflow)");
    cap = K - dd - 1;
  }
  Scratch sc(s);
  TG_TRY(sc.alloc((size_t)d.n * dd * 8 + 16));
  uint32_t* E_tgt = sc.as<uint32_t>();
  uint32_t* E_val = E_tgt + (size_t)d.n * dd;
  const int grid = grid_for(kWarps, d.n);
  Scratch ord(s);
  const uint32_t* order = nullptr;
  stage_begin("prune_order", s);
  TG_TRY(locality_order(d, ord, &order, s));
  stage_end("prune_order", s);
  const char* sel_name = dpg ? "prune_select_dpg" : "prune_select_cagra";
  stage_begin(sel_name, s);
  if (!dpg) {
    const size_t sm = (256 * 4 + (size_t)K * 8) * kWarps;
    TG_TRY(set_smem((const void*)k_select_cagra, sm));
    k_select_cagra<<<grid, kWarps * 32, sm, s>>>(d.graph, d.n, K, dd, d.hybrid, E_tgt, E_val,
                                                 order);
  } else if (d.dim > 128 && K <= 128) {
    // the three K-arrays, then the (a, m0) items: fewer than (K/2 + 1)(K/4 + 2) * 2
    const size_t sm = (size_t)K * 12 + (size_t)(K / 2 + 1) * ((K + 3) / 4 + 1) * 2 * 2 + 16;
    TG_TRY(set_smem((const void*)k_select_dpg_block, sm));
    int dev = 0, sms = 148;
    TG_CUDA(cudaGetDevice(&dev));
    TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int g = (int)std::min<uint64_t>(d.n, (uint64_t)sms);
    k_select_dpg_block<<<g, kDpgThreads, sm, s>>>(d.graph, d.nd, d.data, d.n, d.dim, K, dd,
                                                  d.hybrid, E_tgt, E_val, order);
  } else {
    const size_t sm = ((size_t)K * 12) * kWarps;
    TG_TRY(set_smem((const void*)k_select_dpg, sm));
    k_select_dpg<<<grid, kWarps * 32, sm, s>>>(d.graph, d.nd, d.data, d.n, d.dim, K, dd, d.hybrid,
                                               E_tgt, E_val, order);
  }
  count_launch();
  TG_CUDA(cudaGetLastError());
  stage_end(sel_name, s);
  stage_begin("prune_reverse_store", s);
  TG_TRY(reverse_store(d, E_tgt, E_val, nullptr, dd, 1, cap, dd, s));
  stage_end("prune_reverse_store", s);
  stage_begin("prune_filter_reverse_1hop", s);
  const size_t sm2 = ((size_t)dd * 16) * kWarps;
  TG_TRY(set_smem((const void*)k_filter_reverse_1hop, sm2));
  k_filter_reverse_1hop<<<grid, kWarps * 32, sm2, s>>>(d.graph, d.rgraph, d.rnum, d.hybrid, d.n,
                                                       K, dd);
  count_launch();
  TG_CUDA(cudaGetLastError());
  stage_end("prune_filter_reverse_1hop", s);
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

}  // namespace

int stage_cal_ep(const Dev& d, uint32_t topm, uint32_t* ep_host, cudaStream_t s) {
  TG_TRY(check_shape(d, 1));
  TG_TRY(validate(d, s));
  Scratch sc(s);
  TG_TRY(sc.alloc(4));
  const uint32_t W = topm + d.k;
  const size_t sm = beam_bytes(W) + 64;
  TG_TRY(set_smem((const void*)k_cal_ep, sm));
  k_cal_ep<<<1, 32, sm, s>>>(d.graph, d.data, d.center, d.dim, d.k, topm, sc.as<uint32_t>());
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cudaMemcpyAsync(ep_host, sc.p, 4, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

int prune_index(const Dev& d, const PruneArgs& a, const std::string& type, uint32_t* ep_host,
                cudaStream_t s) {
  TG_TRY(check_shape(d, a.final_degree));
  TG_TRY(validate(d, s));
  if (type == "NSG" || type == "Vamana") {
    PruneArgs b = a;
    if (type == "NSG") b.thre = 1.0f;  // pybind.cu:181,183 pass 1.0
    return run_dist_prune(d, b, true, 0, ep_host, s);
  }
  if (type == "NSSG") return run_dist_prune(d, a, false, 1, ep_host, s);
  if (type == "CAGRA") return run_rank_prune(d, a, false, s);
  if (type == "DPG") return run_rank_prune(d, a, true, s);
  return fail(TAGORE_EINVAL, "unknown index_type '%s' (NSG, Vamana, NSSG, CAGRA, DPG)",
              type.c_str());
}

// ---------------------------------------------------------------------------
// Pruning_with_CFS for path|2-hop with dist|angle without allocating: every
// temporary of run_dist_prune and reverse_store (the validation flag, the
// select rows, the reverse-edge keys, CUB's temporary storage) is carved
// from one file-scope device array. The array is per device and shared by all
// calls on it, so calls whose GPU work overlaps would race on it; the C entry
// point serialises its calls under a lock and returns only after the work has
// finished.
namespace {
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct Carve {
  unsigned char* base;
  size_t used = 0;
  void* take(size_t bytes) {
    void* p = base ? base + used : nullptr;
    used += (bytes + 255) & ~(size_t)255;
    return p;
  }
};
}  // namespace

int prune_cfs_static(const Dev& d, const PruneArgs& a, const std::string& mode,
                     const std::string& metric, uint32_t* ep_host, cudaStream_t s) {
  TG_TRY(check_shape(d, a.final_degree));
  const bool path = mode == "path";
  if ((!path && mode != "2-hop") || (metric != "dist" && metric != "angle"))
    return fail(TAGORE_EINVAL,
                "without allocation only path|2-hop with dist|angle are offered (mode='%s' "
                "metric='%s')",
                mode.c_str(), metric.c_str());
  const int m = metric == "angle" ? 1 : 0;
  const uint32_t fd = a.final_degree, K = d.k;
  if (!path && K * K < kSelectCand) return fail(TAGORE_EINVAL, "2-hop collect needs K*K >= 480");
  if (path && (a.topm == 0 || a.topm > 256)) return fail(TAGORE_EINVAL, "TOPM must be in [1, 256]");
  const size_t E = (size_t)d.n * fd;
  if (E >= 0xFFFFFFFFull) return fail(TAGORE_EINVAL, "too many reverse edges (%zu)", E);
  int end_bit = 1;
  while (end_bit < 32 && ((uint64_t)1 << end_bit) <= d.n) ++end_bit;
  size_t sort_tmp = 0, scan_tmp = 0;
  TG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (uint32_t*)nullptr,
                                          (uint32_t*)nullptr, (uint32_t*)nullptr,
                                          (uint32_t*)nullptr, (int)E, 0, end_bit, s));
  TG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                        (int)d.n, s));
  const size_t tmp = std::max(sort_tmp, scan_tmp);
  // The select kernel's grid is capped here so that its per-warp rings of
  // scored nodes (path collect) stay small: 64 blocks, under 1 MB.
  SelLayout lay{path ? a.topm + K : 0u, kSelectCand + K, fd};
  const size_t sm = lay.bytes() * kWarps;
  const void* fn = path ? (const void*)k_select<true> : (const void*)k_select<false>;
  TG_TRY(set_smem(fn, sm));
  int grid = 0;
  TG_TRY(resident_grid(fn, kWarps * 32, sm, kWarps, d.n, &grid));
  grid = std::min(grid, 64);
  const size_t ring_n = path ? (size_t)grid * kWarps * kSelectCand : 0;
  // Layout: flags | select rows | reverse-edge keys | CUB temporary | rings.
  uint32_t* ring_ids = nullptr;
  float* ring_dis = nullptr;
  auto layout = [&](Carve& c, uint32_t** flags, uint32_t** P_ids, float** P_dis, uint32_t** P_cnt,
                    uint32_t** keys, uint32_t** vals, uint32_t** keys2, uint32_t** vals2,
                    uint32_t** deg, uint32_t** off, void** tmp_p) {
    *flags = (uint32_t*)c.take(16);  // [0] bad id, [1] entry point, [2] node counter
    *P_ids = (uint32_t*)c.take(E * 4);
    *P_dis = (float*)c.take(E * 4);
    *P_cnt = (uint32_t*)c.take((size_t)d.n * 4);
    *keys = (uint32_t*)c.take(E * 4);
    *vals = (uint32_t*)c.take(E * 4);
    *keys2 = (uint32_t*)c.take(E * 4);
    *vals2 = (uint32_t*)c.take(E * 4);
    *deg = (uint32_t*)c.take((size_t)d.n * 4);
    *off = (uint32_t*)c.take((size_t)d.n * 4);
    *tmp_p = c.take(tmp);
    ring_ids = (uint32_t*)c.take(ring_n * 4);
    ring_dis = (float*)c.take(ring_n * 4);
  };
  uint32_t *flags, *P_ids, *P_cnt, *keys, *vals, *keys2, *vals2, *deg, *off;
  float* P_dis;
  void* tmp_p;
  Carve sizing{nullptr};
  layout(sizing, &flags, &P_ids, &P_dis, &P_cnt, &keys, &vals, &keys2, &vals2, &deg, &off, &tmp_p);
  if (sizing.used > kStaticScratchBytes)
    return fail(TAGORE_EINVAL,
                "POINTS=%u FINAL_DEGREE=%u needs %zu bytes of scratch; the static scratch holds "
                "%zu",
                d.n, fd, sizing.used, kStaticScratchBytes);
  void* base = nullptr;
  TG_CUDA(cudaGetSymbolAddress(&base, g_static_scratch));
  Carve c{static_cast<unsigned char*>(base)};
  layout(c, &flags, &P_ids, &P_dis, &P_cnt, &keys, &vals, &keys2, &vals2, &deg, &off, &tmp_p);

  // From the first queued operation on, every return waits for the stream,
  // so the caller's lock is released only when no work on the shared array
  // is still in flight, error paths included.
  struct DrainOnExit {
    cudaStream_t s;
    ~DrainOnExit() { cudaStreamSynchronize(s); }
  } drain{s};

  // validate (as validate())
  TG_CUDA(cudaMemsetAsync(flags, 0, 16, s));
  const size_t cnt = (size_t)d.n * d.k;
  k_validate<<<grid_for(256, cnt), 256, 0, s>>>(d.graph, cnt, d.n, flags);
  count_launch();
  TG_CUDA(cudaGetLastError());
  uint32_t bad = 0;
  TG_CUDA(cudaMemcpyAsync(&bad, flags, 4, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  if (bad) return fail(TAGORE_EINVAL, "graph holds an id >= POINTS (%u)", d.n);

  // select (as run_dist_prune)
  uint32_t* ep_dev = flags + 1;
  uint32_t* ctr = flags + 2;
  if (path) {
    const size_t sm = beam_bytes(a.topm + K) + 64;
    TG_TRY(set_smem((const void*)k_cal_ep, sm));
    k_cal_ep<<<1, 32, sm, s>>>(d.graph, d.data, d.center, d.dim, K, a.topm, ep_dev);
    count_launch();
    TG_CUDA(cudaGetLastError());
  }
  if (path)
    k_select<true><<<grid, kWarps * 32, sm, s>>>(d.graph, d.nd, d.data, d.n, d.dim, K, ep_dev, ctr,
                                                 a.topm, fd, a.thre, P_ids, P_dis, P_cnt, nullptr,
                                                 ring_ids, ring_dis, nullptr);
  else
    k_select<false><<<grid, kWarps * 32, sm, s>>>(d.graph, d.nd, d.data, d.n, d.dim, K, ep_dev,
                                                  ctr, a.topm, fd, a.thre, P_ids, P_dis, P_cnt,
                                                  nullptr, nullptr, nullptr, nullptr);
  count_launch();
  TG_CUDA(cudaGetLastError());

  // reverse store (as reverse_store with mode 0, cap = mod = K)
  TG_CUDA(cudaMemsetAsync(deg, 0, (size_t)d.n * 4, s));
  k_edge_keys<<<grid_for(256, E), 256, 0, s>>>(P_ids, P_cnt, d.n, fd, keys, vals, deg);
  count_launch();
  TG_CUDA(cudaGetLastError());
  size_t t1 = tmp;
  TG_CUDA(cub::DeviceScan::ExclusiveSum(tmp_p, t1, deg, off, (int)d.n, s));
  t1 = tmp;
  TG_CUDA(cub::DeviceRadixSort::SortPairs(tmp_p, t1, keys, keys2, vals, vals2, (int)E, 0, end_bit,
                                          s));
  k_reverse_fill<0><<<grid_for(8, d.n), 256, 0, s>>>(vals2, deg, off,
                                                     reinterpret_cast<const uint32_t*>(P_dis),
                                                     d.n, fd, K, K, d.k, d.rgraph, d.rd, d.rnum);
  count_launch();
  TG_CUDA(cudaGetLastError());

  // filter_reverse
  const size_t sm2 = ((size_t)(fd + K) * 8 + (size_t)fd * 8 + 16) * kWarps;
  TG_TRY(set_smem((const void*)k_filter_reverse, sm2));
  k_filter_reverse<<<grid, kWarps * 32, sm2, s>>>(d.graph, d.nd, d.rgraph, d.rd, d.rnum, d.data,
                                                  d.n, d.dim, K, fd, m, a.thre, P_ids, P_cnt,
                                                  nullptr);
  count_launch();
  TG_CUDA(cudaGetLastError());
  if (path && ep_host) TG_CUDA(cudaMemcpyAsync(ep_host, ep_dev, 4, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

int prune_cfs(const Dev& d, const PruneArgs& a, const std::string& mode, const std::string& metric,
              uint32_t* ep_host, cudaStream_t s) {
  TG_TRY(check_shape(d, a.final_degree));
  TG_TRY(validate(d, s));
  const bool dist_like = metric == "dist" || metric == "angle";
  const int m = metric == "angle" ? 1 : 0;
  if (mode == "path" && dist_like) return run_dist_prune(d, a, true, m, ep_host, s);
  if (mode == "2-hop" && dist_like) return run_dist_prune(d, a, false, m, ep_host, s);
  if (mode == "1-hop" && metric == "rank") return run_rank_prune(d, a, false, s);
  return fail(TAGORE_EINVAL,
              "unsupported CFS combination mode='%s' metric='%s' (path|2-hop with dist|angle, "
              "1-hop with rank)",
              mode.c_str(), metric.c_str());
}

}  // namespace tagore
