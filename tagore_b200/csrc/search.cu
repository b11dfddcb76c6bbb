// search.cu -- batched greedy graph search: the recall evaluator for built
// indexes. It is NSG's search (src/common.cu:65-127): a sorted pool of L
// candidates, each expanded once in pool order, its unseen neighbours scored
// and merged; the pool starts from the entry point's neighbours, topped up to
// L with seeded random nodes (seed != 0) or preceded by the entry point itself
// (seed == 0).
//
// Layout: one warp per query, queries strided over a resident grid. The
// query, the pool and its merge buffer sit in shared memory; the visited set
// is an open-addressing table in global memory per warp whose keys carry the
// query number in their high half, so a table is cleared once per call, not
// per query.
//
// The visiting order is the sequential one, done 32 ids at a time: a batch of
// neighbours (in adjacency order) is deduplicated with __match_any_sync, the
// unseen ones are scored by one lane each, and the batch is merged into the
// pool as if the ids had been inserted one by one -- a pool entry goes before
// a new one at equal distance, earlier new ones before later ones. Distances
// are summed per lane in dimension order with round-to-nearest adds and
// multiplies (no contraction), the same arithmetic as a plain C loop, so the
// result equals the sequential search id for id.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "internal.h"

namespace tagore {
namespace {

constexpr uint32_t kOpen = 0x80000000u;  // pool entry not yet expanded
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint64_t kGold = 0x9E3779B97F4A7C15ull;
constexpr uint32_t kMaxWarps = 8;

struct Entry {
  float d;
  uint32_t id;  // | kOpen while unexpanded
};

struct SearchArgs {
  const float* base;
  uint32_t n, dim;
  const uint64_t* offs;
  const uint32_t* adj;
  uint64_t edges;
  uint32_t ep;
  const float* queries;
  uint32_t nq;
  uint32_t L, k;
  uint64_t seed;
  uint32_t cap_log2;
  unsigned long long* table;
  uint32_t* out;
  uint32_t* err;
};

// splitmix64's output function (Steele, Lea and Flood, OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Visited set of one query: linear probing over 2^cap_log2 slots, filled to
// half at most. Only the owning warp touches it; reads go to L2 (ld.cg) so a
// slot claimed by another lane's atomicCAS is never read stale from L1.
struct Visited {
  unsigned long long* tab;
  uint32_t mask, shift;
  uint32_t tag;  // query number + 1

  __device__ __forceinline__ uint32_t slot(uint32_t id) const {
    return (id * 0x9E3779B1u) >> shift;
  }
  __device__ bool contains(uint32_t id) const {
    for (uint32_t h = slot(id);; h = (h + 1) & mask) {
      const unsigned long long v = __ldcg(tab + h);
      if ((uint32_t)(v >> 32) != tag) return false;
      if ((uint32_t)v == id) return true;
    }
  }
  __device__ void insert(uint32_t id) const {
    const unsigned long long key = ((unsigned long long)tag << 32) | id;
    for (uint32_t h = slot(id);;) {
      const unsigned long long v = __ldcg(tab + h);
      if ((uint32_t)(v >> 32) != tag) {
        if (atomicCAS(tab + h, v, key) == v) return;
        continue;  // another lane took the slot: read it again
      }
      if (v == key) return;
      h = (h + 1) & mask;
    }
  }
};

template <bool kVec>
__device__ __forceinline__ float sq_dist(const float* __restrict__ q, const float* __restrict__ y,
                                         uint32_t dim) {
  float acc = 0.0f;
  if (kVec) {
    const float4* y4 = reinterpret_cast<const float4*>(y);
    const float4* q4 = reinterpret_cast<const float4*>(q);
#pragma unroll 4
    for (uint32_t j = 0; j < dim / 4; ++j) {
      const float4 v = __ldg(y4 + j);
      const float4 w = q4[j];
      float t = __fsub_rn(w.x, v.x);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
      t = __fsub_rn(w.y, v.y);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
      t = __fsub_rn(w.z, v.z);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
      t = __fsub_rn(w.w, v.w);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
  } else {
    for (uint32_t j = 0; j < dim; ++j) {
      const float t = __fsub_rn(q[j], __ldg(y + j));
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
  }
  return acc;
}

template <bool kVec>
struct WarpSearch {
  const SearchArgs& a;
  uint32_t lane;
  float* qv;       // query, dim floats
  Entry* P;        // pool, `size` entries sorted by (d, arrival)
  Entry* Q;        // merge target
  float* fresh_d;  // the batch's new distances in sorted order
  Visited vis;
  uint32_t size, touched, limit;
  bool over;

  // Visits the ids of the active lanes in lane order; at most `need` unseen
  // ones are taken (the rest stay unvisited).
  __device__ void batch(uint32_t id, bool active, uint32_t need) {
    const bool valid = active && id < a.n;
    const uint32_t same = __match_any_sync(~0u, valid ? id : kNone);
    const bool first = valid && (uint32_t)(__ffs(same) - 1) == lane;
    const bool unseen = first && !vis.contains(id);
    const uint32_t ub = __ballot_sync(~0u, unseen);
    const bool take = unseen && (uint32_t)__popc(ub & ((1u << lane) - 1u)) < need;
    const uint32_t tb = __ballot_sync(~0u, take);
    const uint32_t m = __popc(tb);
    if (m == 0) return;
    if (touched + m > limit) {
      over = true;
      return;
    }
    touched += m;
    float d = 0.0f;
    if (take) {
      vis.insert(id);
      d = sq_dist<kVec>(qv, a.base + (size_t)id * a.dim, a.dim);
    }
    // Rank among the batch's new entries: earlier lanes first on ties.
    uint32_t within = 0;
    for (uint32_t b = tb; b; b &= b - 1) {
      const uint32_t j = __ffs(b) - 1;
      const float dj = __shfl_sync(~0u, d, j);
      within += (dj < d) || (dj == d && j < lane);
    }
    if (take) fresh_d[within] = d;
    __syncwarp();
    const uint32_t L = a.L;
    for (uint32_t p = lane; p < size; p += 32) {
      const Entry e = P[p];
      uint32_t lo = 0, hi = m;  // new entries strictly closer than e
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (fresh_d[mid] < e.d) lo = mid + 1;
        else hi = mid;
      }
      if (p + lo < L) Q[p + lo] = e;
    }
    if (take) {
      uint32_t lo = 0, hi = size;  // pool entries at most as far as d
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (P[mid].d <= d) lo = mid + 1;
        else hi = mid;
      }
      if (lo + within < L) Q[lo + within] = Entry{d, id | kOpen};
    }
    __syncwarp();
    size = min(L, size + m);
    Entry* t = P;
    P = Q;
    Q = t;
  }

  __device__ void neighbours(uint32_t u) {
    if (u >= a.n) return;
    const uint64_t lo = a.offs[u];
    const uint64_t hi = min(a.offs[u + 1], a.edges);
    for (uint64_t e = lo; e < hi && !over; e += 32) {
      const bool act = e + lane < hi;
      batch(act ? a.adj[e + lane] : kNone, act, kNone);
    }
  }

  __device__ void run(uint32_t q) {
    size = 0;
    touched = 0;
    over = false;
    vis.tag = q + 1;
    for (uint32_t j = lane; j < a.dim; j += 32) qv[j] = a.queries[(size_t)q * a.dim + j];
    __syncwarp();
    if (a.seed == 0) batch(a.ep, lane == 0, kNone);
    neighbours(a.ep);
    if (a.seed != 0) {
      // splitmix64's stream: z advances by the golden gamma per draw, lane i
      // takes draw i of the batch, and a batch that fills the pool ends it.
      uint64_t z = a.seed ^ (kGold * (uint64_t)(q + 1));
      const uint32_t want = min(a.L, a.n);
      while (touched < want && !over) {
        const uint64_t x = mix64(z + kGold * (uint64_t)(lane + 1));
        batch((uint32_t)(x % (uint64_t)a.n), true, want - touched);
        z += kGold * 32ull;
      }
    }
    // Expand the first open entry until none is left. Every expansion closes
    // an entry that was opened by a first visit, so the loop ends.
    while (!over) {
      int idx = -1;
      for (uint32_t c = 0; c < size; c += 32) {
        const bool open = c + lane < size && (P[c + lane].id & kOpen);
        const uint32_t b = __ballot_sync(~0u, open);
        if (b) {
          idx = (int)(c + __ffs(b) - 1);
          break;
        }
      }
      if (idx < 0) break;
      const uint32_t u = P[idx].id & ~kOpen;
      __syncwarp();
      if (lane == 0) P[idx].id = u;
      __syncwarp();
      neighbours(u);
    }
    for (uint32_t j = lane; j < a.k; j += 32)
      a.out[(size_t)q * a.k + j] = (over || j >= size) ? kNone : (P[j].id & ~kOpen);
    if (over && lane == 0) atomicOr(a.err, 1u);
    __syncwarp();
  }
};

template <bool kVec>
__global__ void __launch_bounds__(kMaxWarps * 32) k_search(const __grid_constant__ SearchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t nw = blockDim.x >> 5;
  const uint32_t dpad = (a.dim + 3) & ~3u;
  const size_t per_warp = (size_t)dpad * 4 + 2ull * a.L * sizeof(Entry) + 32 * 4;
  unsigned char* mine = smem + wib * per_warp;
  const uint32_t gwarp = blockIdx.x * nw + wib;
  const uint32_t nwarps = gridDim.x * nw;
  WarpSearch<kVec> w{a, lane};
  w.qv = reinterpret_cast<float*>(mine);
  w.P = reinterpret_cast<Entry*>(mine + (size_t)dpad * 4);
  w.Q = w.P + a.L;
  w.fresh_d = reinterpret_cast<float*>(w.Q + a.L);
  w.vis = Visited{a.table + ((size_t)gwarp << a.cap_log2), (1u << a.cap_log2) - 1u,
                  32u - a.cap_log2, 0u};
  w.limit = 1u << (a.cap_log2 - 1);
  for (uint32_t q = gwarp; q < a.nq; q += nwarps) w.run(q);
}

uint32_t ceil_log2(uint64_t v) {
  uint32_t r = 0;
  while ((1ull << r) < v) ++r;
  return r;
}

}  // namespace

int search_check(const TagoreSearchParams& p, const float* base, uint64_t n, uint32_t dim,
                 const uint64_t* offs, const uint32_t* adj, uint64_t edges, uint32_t ep,
                 const float* queries, uint32_t nq, const uint32_t* out) {
  if (n == 0 || n >= kOpen || dim == 0 || p.L == 0 || p.k == 0)
    return fail(TAGORE_EINVAL, "search: need 0 < n < 2^31 and dim, L, k > 0");
  if (ep >= n) return fail(TAGORE_EINVAL, "search: entry point %u outside %llu nodes", ep,
                           (unsigned long long)n);
  if (p.visit_cap > (1u << 28)) return fail(TAGORE_EINVAL, "search: visit_cap above 2^28");
  if (nq == 0) return TAGORE_OK;
  if (!base || !offs || (!adj && edges) || !queries || !out)
    return fail(TAGORE_EINVAL, "search: null pointer");
  return TAGORE_OK;
}

int greedy_search(const TagoreSearchParams& p, const float* base, uint64_t n, uint32_t dim,
                  const uint64_t* offs, const uint32_t* adj, uint64_t edges, uint32_t ep,
                  const float* queries, uint32_t nq, uint32_t* out, cudaStream_t s) {
  TG_TRY(search_check(p, base, n, dim, offs, adj, edges, ep, queries, nq, out));
  if (nq == 0) return TAGORE_OK;
  uint32_t cap_log2 = p.visit_cap ? ceil_log2(p.visit_cap) : ceil_log2(64ull * p.L);
  if (cap_log2 < 14) cap_log2 = 14;

  const uint32_t dpad = (dim + 3) & ~3u;
  const size_t per_warp = (size_t)dpad * 4 + 2ull * p.L * sizeof(Entry) + 32 * 4;
  int dev = 0, sms = 0, smem_max = 0;
  TG_CUDA(cudaGetDevice(&dev));
  TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  TG_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const uint32_t nw = (uint32_t)std::min<size_t>(kMaxWarps, (size_t)smem_max / per_warp);
  if (nw == 0) return fail(TAGORE_EINVAL, "search: dim %u with L %u needs %zu B of shared memory per warp",
                           dim, p.L, per_warp);
  const bool vec = dim % 4 == 0 && ((uintptr_t)base & 15) == 0;
  const void* fn = vec ? (const void*)k_search<true> : (const void*)k_search<false>;
  const size_t smem = per_warp * nw;
  TG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  TG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nw * 32, smem));
  per_sm = std::max(1, std::min(per_sm, 2));
  const uint64_t want = (nq + nw - 1) / nw;
  const uint32_t grid = (uint32_t)std::min<uint64_t>(want, (uint64_t)sms * per_sm);

  Scratch tab(s);
  const size_t tab_bytes = ((size_t)grid * nw << cap_log2) * sizeof(unsigned long long);
  TG_TRY(tab.alloc(tab_bytes + 16));
  TG_CUDA(cudaMemsetAsync(tab.p, 0, tab_bytes + 16, s));
  SearchArgs a{base, (uint32_t)n, dim, offs, adj, edges, ep, queries, nq, p.L, p.k, p.seed, cap_log2,
               tab.as<unsigned long long>(), out,
               reinterpret_cast<uint32_t*>(tab.as<unsigned char>() + tab_bytes)};
  stage_begin("search", s);
  if (vec) k_search<true><<<grid, nw * 32, smem, s>>>(a);
  else k_search<false><<<grid, nw * 32, smem, s>>>(a);
  TG_CUDA(cudaGetLastError());
  count_launch();
  stage_end("search", s, 0, nq);
  uint32_t err = 0;
  TG_CUDA(cudaMemcpyAsync(&err, a.err, 4, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  if (err) return fail(TAGORE_EINVAL, "search: a query visited more than %u nodes; raise visit_cap",
                       1u << (cap_log2 - 1));
  return TAGORE_OK;
}

}  // namespace tagore
