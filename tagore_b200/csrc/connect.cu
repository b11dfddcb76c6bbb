// connect.cu -- opt-in connectivity fix of a pruned graph (sm_100a).
//
// No counterpart in the reference: its Pruning stores the pruned rows as they
// are (pybind.cu:177-187), and on data made of separated clusters part of the
// graph is not reachable from the entry point. This pass, in the manner of
// NSG's tree growing, makes every node reachable from `ep` by adding edges;
// rows keep their [deg, ids...] layout with stride K, so added edges use the
// row's unused slots. It changes the edge lists, hence opt-in.
//
//   1. reach: level-synchronous BFS from ep over the rows;
//   2. attach: for up to kBatch unreachable nodes u (lowest ids first), a warp
//      walks greedily from ep toward u (exact reference-order distances; all
//      walks finish before any row changes), then u is appended to the row of
//      the walk's end node v, which is reachable; when v's row is full the
//      walk's previous nodes, then hashed reachable nodes, are tried;
//   3. BFS again from the attached nodes; repeat until all are reachable.
#include "common.cuh"
#include "internal.h"

namespace tagore {
namespace {

constexpr uint32_t kBatch = 256;  // unreachable nodes attached per round
constexpr uint32_t kWalk = 256;   // greedy steps per walk
constexpr int kEnds = 8;          // walk nodes kept as attach points, end first
constexpr int kProbe = 64;        // hashed reachable nodes tried after them

// One BFS level: every frontier node marks its unmarked out-neighbours and
// appends them to the next frontier. Warp per frontier node.
__global__ void k_bfs(const uint32_t* __restrict__ rows, uint32_t K, uint32_t n,
                      const uint32_t* __restrict__ front, uint32_t nfront,
                      uint32_t* __restrict__ reach, uint32_t* __restrict__ next,
                      uint32_t* __restrict__ nnext) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; f < nfront;
       f += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t u = front[f];
    const uint32_t* row = rows + (size_t)u * K;
    const uint32_t deg = min(row[0], K - 1);
    for (uint32_t j = lane; j < deg; j += 32) {
      const uint32_t v = row[1 + j];
      if (v < n && atomicExch(&reach[v], 1u) == 0u) next[atomicAdd(nnext, 1u)] = v;
    }
  }
}

// Unreachable nodes in ascending id order, at most `cap` of them; *total
// counts them all.
__global__ void k_unreached(const uint32_t* __restrict__ reach, uint32_t n, uint32_t cap,
                            uint32_t* __restrict__ out, uint32_t* __restrict__ total) {
  // one block scans in order so that the list is the lowest ids
  __shared__ uint32_t base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (uint32_t i0 = 0; i0 < n; i0 += blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    const bool un = i < n && reach[i] == 0u;
    const unsigned m = __ballot_sync(kFull, un);
    __shared__ uint32_t warp_off[32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    if (lane == 0) warp_off[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t acc = base;
      for (uint32_t q = 0; q < blockDim.x / 32; ++q) {
        const uint32_t c = warp_off[q];
        warp_off[q] = acc;
        acc += c;
      }
      base = acc;
    }
    __syncthreads();
    if (un) {
      const uint32_t pos = warp_off[w] + __popc(m & ((1u << lane) - 1u));
      if (pos < cap) out[pos] = i;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = base;
}

// For each listed node u: a greedy walk from ep toward u over the rows (the
// closest out-neighbour while it is closer), recording the walk's last kEnds
// nodes, end first. All of them are reachable from ep. Reads rows only.
__global__ void k_walk(const uint32_t* __restrict__ rows, uint32_t K, uint32_t n,
                       const __half* __restrict__ data, uint32_t dim, uint32_t ep,
                       const uint32_t* __restrict__ todo, uint32_t ntodo,
                       uint32_t* __restrict__ ends) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntodo;
       t += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t u = todo[t];
    const __half* q = data + (size_t)u * dim;
    uint32_t path[kEnds];
#pragma unroll
    for (int h = 0; h < kEnds; ++h) path[h] = ep;
    uint32_t cur = ep;
    float cd = warp_dist(q, data + (size_t)ep * dim, dim, lane);
    for (uint32_t step = 0; step < kWalk; ++step) {
      const uint32_t* row = rows + (size_t)cur * K;
      const uint32_t deg = min(row[0], K - 1);
      float best = cd;
      uint32_t bid = cur;
      for (uint32_t j0 = 0; j0 < deg; j0 += 32) {
        const uint32_t j = j0 + lane;
        float d = INFINITY;
        uint32_t v = kInv;
        if (j < deg) {
          v = row[1 + j];
          if (v < n) d = row_dist(q, data + (size_t)v * dim, dim);
        }
        // warp minimum (distance, then id) of this chunk
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float od = __shfl_xor_sync(kFull, d, o);
          const uint32_t ov = __shfl_xor_sync(kFull, v, o);
          if (od < d || (od == d && ov < v)) {
            d = od;
            v = ov;
          }
        }
        if (d < best) {
          best = d;
          bid = v;
        }
      }
      if (bid == cur) break;  // local minimum
#pragma unroll
      for (int h = kEnds - 1; h > 0; --h) path[h] = path[h - 1];
      path[0] = bid;
      cur = bid;
      cd = best;
    }
#pragma unroll
    for (int h = 0; h < kEnds; ++h)
      if (lane == (uint32_t)h) ends[(size_t)t * kEnds + h] = path[h];
  }
}

// Appends each listed node u to the first row among its walk's ends that has
// a free slot; when all of them are full (walks that cannot leave the
// reachable part all end at the same few nodes), to a reachable node with a
// free slot found by hashed probing. Attached nodes start the next BFS.
__global__ void k_append(uint32_t* __restrict__ rows, uint32_t K, uint32_t n,
                         const uint32_t* __restrict__ todo, uint32_t ntodo,
                         const uint32_t* __restrict__ ends, uint32_t* __restrict__ reach,
                         uint32_t* __restrict__ front, uint32_t* __restrict__ nfront,
                         unsigned long long* __restrict__ added) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntodo) return;
  const uint32_t u = todo[t];
  auto try_row = [&](uint32_t v) -> bool {
    if (v == u || v >= n) return false;
    uint32_t* row = rows + (size_t)v * K;
    const uint32_t slot = atomicAdd(&row[0], 1u);
    if (slot + 1 < K) {
      row[1 + slot] = u;
      return true;
    }
    atomicSub(&row[0], 1u);
    return false;
  };
  bool done = false;
  for (int h = 0; h < kEnds && !done; ++h) done = try_row(ends[(size_t)t * kEnds + h]);
  uint64_t x = 0x9E3779B97F4A7C15ull * (uint64_t)(u + 1);
  for (int p = 0; p < kProbe && !done; ++p) {
    x ^= x >> 29;
    x *= 0xBF58476D1CE4E5B9ull;
    const uint32_t v = (uint32_t)(x % n);
    if (reach[v] == 1u && v != u) done = try_row(v);
  }
  if (done) {
    atomicAdd(added, 1ull);
    if (atomicExch(&reach[u], 1u) == 0u) front[atomicAdd(nfront, 1u)] = u;
  }
}

}  // namespace

int connect_graph(const Dev& d, uint32_t ep, uint64_t* added_out, cudaStream_t s) {
  if (ep >= d.n) return fail(TAGORE_EINVAL, "entry point %u >= POINTS %u", ep, d.n);
  if (d.k < 2) return fail(TAGORE_EINVAL, "K must be >= 2");
  Scratch sc(s);
  const size_t n = d.n;
  TG_TRY(sc.alloc(16 + n * 4 * 3 + (size_t)kBatch * kEnds * 4));
  unsigned long long* added = sc.as<unsigned long long>();
  uint32_t* ctr = reinterpret_cast<uint32_t*>(added + 1);  // [0] frontier size, [1] unreachable
  uint32_t* reach = ctr + 2;
  uint32_t* fa = reach + n;
  uint32_t* fb = fa + n;
  uint32_t* ends = fb + n;  // [kBatch][kEnds] walk ends
  TG_CUDA(cudaMemsetAsync(added, 0, 16 + n * 4, s));  // counters and reach
  const uint32_t one = 1;
  TG_CUDA(cudaMemcpyAsync(reach + ep, &one, 4, cudaMemcpyHostToDevice, s));
  TG_CUDA(cudaMemcpyAsync(fa, &ep, 4, cudaMemcpyHostToDevice, s));
  uint32_t nfront = 1;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto bfs = [&]() -> int {
    while (nfront) {
      TG_CUDA(cudaMemsetAsync(ctr, 0, 4, s));
      const uint32_t blocks = std::min<uint32_t>((nfront + 7) / 8, (uint32_t)sms * 32);
      k_bfs<<<blocks, 256, 0, s>>>(d.graph, d.k, d.n, fa, nfront, reach, fb, ctr);
      count_launch();
      TG_CUDA(cudaGetLastError());
      TG_CUDA(cudaMemcpyAsync(&nfront, ctr, 4, cudaMemcpyDeviceToHost, s));
      TG_CUDA(cudaStreamSynchronize(s));
      std::swap(fa, fb);
    }
    return TAGORE_OK;
  };
  TG_TRY(bfs());
  uint32_t prev_unreached = 0xFFFFFFFFu;
  for (int round = 0; round < 1 << 20; ++round) {
    k_unreached<<<1, 1024, 0, s>>>(reach, d.n, kBatch, fb, ctr + 1);
    count_launch();
    TG_CUDA(cudaGetLastError());
    uint32_t unreached = 0;
    TG_CUDA(cudaMemcpyAsync(&unreached, ctr + 1, 4, cudaMemcpyDeviceToHost, s));
    TG_CUDA(cudaStreamSynchronize(s));
    if (unreached == 0) break;
    if (unreached >= prev_unreached)
      return fail(TAGORE_EINVAL, "connectivity fix made no progress (%u nodes unreachable)",
                  unreached);
    prev_unreached = unreached;
    const uint32_t todo = std::min(unreached, kBatch);
    TG_CUDA(cudaMemsetAsync(ctr, 0, 4, s));
    // the nodes to attach are listed in fb; attached nodes start the next BFS in fa
    k_walk<<<std::min<uint32_t>((todo + 7) / 8, (uint32_t)sms * 16), 256, 0, s>>>(
        d.graph, d.k, d.n, d.data, d.dim, ep, fb, todo, ends);
    k_append<<<(todo + 255) / 256, 256, 0, s>>>(d.graph, d.k, d.n, fb, todo, ends, reach, fa,
                                                ctr, added);
    count_launch(2);
    TG_CUDA(cudaGetLastError());
    TG_CUDA(cudaMemcpyAsync(&nfront, ctr, 4, cudaMemcpyDeviceToHost, s));
    TG_CUDA(cudaStreamSynchronize(s));
    TG_TRY(bfs());
  }
  unsigned long long h = 0;
  TG_CUDA(cudaMemcpyAsync(&h, added, 8, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  if (added_out) *added_out = h;
  return TAGORE_OK;
}

}  // namespace tagore
