// knn_tc.cu -- local join on tcgen05 tensor cores (sm_100a).
//
// Persistent blocks (three per SM, so their three 128-column TMEM
// accumulators always fit in the SM's 512) walk the nodes. For each node's
// join list (<= 128 FP16 rows):
//   1. TMA tile::gather4 copies the rows into a K-major 128-byte-swizzled tile
//      X in shared memory (box 64 halves x 1 row, four rows per copy);
//   2. one thread issues D/16 tcgen05.mma.kind::f16 (M = N = 128, K = 16), X as
//      both operands, so TMEM holds the Gram tile X X^T in FP32;
//   3. each thread owns one row: it reads its TMEM lane, forms the screened
//      distance n_r + n_c - 2 g_rc from exact FP32 norms, and keeps its
//      `per_row` closest partners that could beat the row's k-th entry
//      (screened value below k-th + 2^-12 (n_r + n_c); the Gram entry's FP32
//      accumulation error is below 2^-16 (n_r + n_c));
//   4. the kept pairs of all rows are pooled and re-ranked exactly
//      (reference-order FP32 from the same shared tile) by all threads; a pair
//      is proposed only when the exact value beats the k-th entry. No stored
//      distance comes from a tensor core.
// A producer warp fills two tile stages: while node i is screened and
// re-ranked, node i+1's rows are in flight, and its MMA goes into the single
// accumulator as soon as the screen of node i has read it.
// Every wait is bounded by %globaltimer; on expiry the block records an error,
// waits (bounded) for its own copies and MMAs, frees its TMEM and returns.
#include <cuda.h>

#include <algorithm>

#include "knn_shared.cuh"

namespace tagore {
namespace knn {
namespace {

constexpr int kConsumers = 128;             // warps 0-3: one thread per tile row
constexpr int kThreads = kConsumers + 32;    // warp 4: the producer
constexpr int kStages = 2;                   // row tiles in flight
constexpr uint32_t kTmemCols = 128;          // one 128-column accumulator
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s per wait
constexpr uint32_t kDone = 0xFFFFFFFFu;      // stage node: the producer has finished
constexpr float kOneMinusEps = 1.0f - 0.000244140625f;  // 1 - 2^-12, the screen's margin

struct __align__(1024) Tile {
  uint8_t x[2][kMaxList][128];  // [64-half column block][row][128 B], SW128
};

struct __align__(1024) TcSmem {
  Tile tile[kStages];
  uint32_t ids[kStages][kMaxList];
  float hnrm[kStages][kMaxList];  // (1 - 2^-12) x exact squared norm
  float kth[kStages][kMaxList];
  uint32_t pairs[kConsumers * 4];  // kept (row << 16 | column) pairs of the node
  uint32_t warp_pairs[kConsumers / 32];
  unsigned long long full_bar[kStages];   // rows landed and stage filled
  unsigned long long empty_bar[kStages];  // consumers done with the stage
  unsigned long long mma_bar[2];          // accumulator written
  uint32_t taddr;
  uint32_t node[kStages], nn[kStages], total[kStages];
  uint32_t filled, consumed;  // producer fills with rows; fills the consumers saw land
  int flag;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait by one thread; true when the phase completed in time.
__device__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = now_ns();
  while (!mbar_try(bar, parity))
    if (now_ns() - t0 > kWaitNs) return false;
  return true;
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  // K-major, 128-byte swizzle: LBO 16 B (encoded 1), SBO 1024 B between
  // 8-row groups (encoded 64), descriptor version 1, layout type 2.
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// kind::f16 instruction descriptor: F16 x F16 -> F32, both K-major, M = N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (0u << 7) | (0u << 10) | ((128u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// (v0, v1) = (-2 g0 + h0, -2 g1 + h1) as one packed FP32 pair FMA (each half
// rounded once, as fmaf).
__device__ __forceinline__ void fma2_m2(float g0, float g1, float h0, float h1, float& v0,
                                        float& v1) {
  asm("{.reg .b64 a, b, c;\n\t"
      "mov.b64 a, {%2, %3};\n\t"
      "mov.b64 b, {%6, %6};\n\t"
      "mov.b64 c, {%4, %5};\n\t"
      "fma.rn.f32x2 c, a, b, c;\n\t"
      "mov.b64 {%0, %1}, c;}"
      : "=f"(v0), "=f"(v1)
      : "f"(g0), "f"(g1), "f"(h0), "f"(h1), "f"(-2.0f));
}

// Chunk j (4 halves) of row r inside a swizzled tile.
__device__ __forceinline__ uint2 tile_chunk(const Tile& t, uint32_t r, uint32_t j) {
  const uint32_t blk = j >> 4, unit = ((j & 15u) >> 1) ^ (r & 7u), half8 = j & 1u;
  return *reinterpret_cast<const uint2*>(&t.x[blk][r][unit * 16 + half8 * 8]);
}

// Chunks 2p and 2p+1 of row r (one 16-byte unit of the swizzled tile).
__device__ __forceinline__ uint4 tile_pair(const Tile& t, uint32_t r, uint32_t p) {
  return *reinterpret_cast<const uint4*>(&t.x[p >> 3][r][((p & 7u) ^ (r & 7u)) * 16]);
}

// Exact reference-order FP32 distance of two tile rows, by one thread.
template <int D>
__device__ __forceinline__ float tile_dist(const Tile& t, uint32_t ra, uint32_t rb, uint32_t dim) {
  if constexpr (D == 128) {
    return dist128_pairs([&](int p, int w) { return tile_pair(t, w ? rb : ra, (uint32_t)p); });
  } else if constexpr (D > 0) {
    return serial_dist<D>([&](int j, int w) { return tile_chunk(t, w ? rb : ra, (uint32_t)j); });
  } else {
    float x[32], y[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) {
      x[l] = 0.0f;
      y[l] = 0.0f;
    }
    for (uint32_t j = 0; j < dim / 4; ++j)
      chunk_acc(tile_chunk(t, ra, j), tile_chunk(t, rb, j), x[j & 31], y[j & 31]);
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

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void consumers_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory");
}

// Barrier of the consumer warps that also tells whether any of them passed
// `v` true.
__device__ __forceinline__ bool consumers_any(bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"(v ? 1u : 0u), "n"(kConsumers)
      : "memory");
  return out != 0;
}

// Producer warp: walks this block's nodes (blockIdx.x, +gridDim.x, ...),
// skips those without a join, and fills stage j % kStages with node j: ids,
// norms and k-th distances (one packed record per row) by the lanes, rows by TMA tile::gather4. Runs
// kStages nodes ahead of the consumers; ends by publishing kDone.
template <int D>
__device__ void join_producer(TcSmem& s, const CUtensorMap& tmap, const float2* __restrict__ meta,
                              const uint32_t* __restrict__ lists,
                              const uint32_t* __restrict__ lcnt, uint32_t n, uint32_t dim,
                              uint32_t K, unsigned long long* n_rows,
                              const uint32_t* __restrict__ order) {
  const uint32_t lane = threadIdx.x & 31u, blocks = (dim + 63) / 64;
  uint32_t next = blockIdx.x;
  uint32_t ph_empty[kStages] = {};
  for (uint32_t j = 0;; ++j) {
    const int st = (int)(j % kStages);
    if (j >= (uint32_t)kStages) {
      bool ok = true;
      if (lane == 0) {
        ok = mbar_wait_bounded(smem_u32(&s.empty_bar[st]), ph_empty[st]);
        if (!ok) s.flag = 0;
      }
      ph_empty[st] ^= 1u;
      if (!__shfl_sync(kFull, ok ? 1 : 0, 0)) return;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    // next node with a join: 32 positions of the order per step, one per lane
    uint32_t u = kDone, nn = 0, tot = 0;
    while (next < n) {
      const uint32_t c = next + lane * gridDim.x;
      const uint32_t node = c < n ? (order ? __ldg(order + c) : c) : 0u;
      uint2 cnt = make_uint2(0, 0);
      if (c < n) cnt = *reinterpret_cast<const uint2*>(lcnt + 2 * (size_t)node);
      const unsigned ok = __ballot_sync(kFull, c < n && cnt.x > 0 && cnt.y >= 2);
      if (ok) {
        const int w = __ffs(ok) - 1;
        u = __shfl_sync(kFull, node, w);
        nn = __shfl_sync(kFull, cnt.x, w);
        tot = __shfl_sync(kFull, cnt.y, w);
        next += ((uint32_t)w + 1u) * gridDim.x;
        break;
      }
      next += 32u * gridDim.x;
    }
    if (lane == 0) {
      s.node[st] = u;
      s.nn[st] = nn;
      s.total[st] = tot;
    }
    if (u == kDone) {
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&s.full_bar[st]));
      return;
    }
    for (uint32_t t = lane; t < tot; t += 32) {
      const uint32_t id = lists[(size_t)u * kMaxList + t];
      s.ids[st][t] = id;
      const float2 m = __ldg(meta + id);
      s.hnrm[st][t] = kOneMinusEps * m.x;
      s.kth[st][t] = m.y;
    }
    __syncwarp();
    const uint32_t groups = (tot + 3) / 4, bar = smem_u32(&s.full_bar[st]);
    if (lane == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                   "r"(groups * 4 * 128 * blocks)
                   : "memory");
      *n_rows += tot;
      s.filled = j + 1;
    }
    __syncwarp();
    for (uint32_t g = lane; g < groups; g += 32) {
      uint32_t r[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) r[t] = s.ids[st][min(4 * g + t, tot - 1)];
      for (uint32_t b = 0; b < blocks; ++b) {
        const uint32_t dst = smem_u32(&s.tile[st].x[b][4 * g][0]);
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::"
            "bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
            "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(b * 64), "r"(r[0]), "r"(r[1]), "r"(r[2]),
            "r"(r[3]), "r"(bar)
            : "memory");
      }
    }
  }
}

// Warp-specialised persistent join. The producer warp (join_producer) keeps
// kStages nodes in flight; the four consumer warps take node i from stage
// i % kStages: thread 0 has issued its Gram tile X X^T (tcgen05, M = N = 128,
// K = 16 steps) into the block's accumulator right after the screen of node
// i - 1; every thread owns one tile row, screens it from TMEM and re-ranks the
// kept pairs exactly. Three blocks per SM (12 consumer warps) with one
// 128-column accumulator each hide more latency than two blocks with two
// accumulators each (240 against 312 ms for the 1M x 128 build's ten joins).
template <int D>
__global__ void __launch_bounds__(kThreads, 3)
    k_join_tc(const __grid_constant__ CUtensorMap tmap, const float2* __restrict__ meta,
              const uint32_t* __restrict__ lists,
              const uint32_t* __restrict__ lcnt, uint32_t n, uint32_t dim, uint32_t K, uint32_t T,
              uint32_t P, unsigned long long* __restrict__ pool,
              unsigned long long* __restrict__ stats, int* __restrict__ err,
              const uint32_t* __restrict__ order) {
  extern __shared__ unsigned char smem_raw[];
  TcSmem& s = *reinterpret_cast<TcSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ksteps = dim / 16;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s.taddr)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int st = 0; st < kStages; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.full_bar[st])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&s.empty_bar[st])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mma_bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mma_bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;");
    asm volatile("fence.proxy.async.shared::cta;");
    s.flag = 1;
    s.filled = 0;
    s.consumed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s.taddr;
  unsigned long long n_pairs = 0, n_props = 0, n_rows = 0;

  if (warp == kConsumers / 32) {
    join_producer<D>(s, tmap, meta, lists, lcnt, n, dim, K, &n_rows, order);
  } else {
    uint32_t ph_full[kStages] = {}, ph_mma[2] = {0, 0};
    bool pending[2] = {false, false};  // thread 0: committed MMAs not yet waited for
    // Thread 0: waits for stage st's rows (phase ph) and issues their Gram
    // tile into accumulator acc. No MMA for a kDone stage or on timeout.
    auto issue = [&](int st, uint32_t ph, uint32_t acc) {
      if (!mbar_wait_bounded(smem_u32(&s.full_bar[st]), ph)) {
        s.flag = 0;
        return;
      }
      if (s.node[st] == kDone) return;
      asm volatile("tcgen05.fence::after_thread_sync;");
      for (uint32_t k = 0; k < ksteps; ++k) {
        const uint64_t desc = sw128_desc(smem_u32(&s.tile[st].x[k >> 2][0][0]) + (k & 3u) * 32);
        const uint32_t accum = k > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + acc * 128),
            "l"(desc), "l"(desc), "r"(kIdesc), "r"(accum));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&s.mma_bar[acc])));
      pending[acc] = true;
    };
    if (tid == 0) issue(0, 0, 0);
    const uint32_t r = tid, lane = tid & 31u;
    uint32_t got_full = 0;  // nodes whose rows this thread has seen land
    for (uint32_t i = 0;; ++i) {
      const int st = (int)(i % kStages);
      const uint32_t acc = 0u;  // one accumulator, refilled once the screen has read it
      const bool got = mbar_wait_bounded(smem_u32(&s.full_bar[st]), ph_full[st]);
      ph_full[st] ^= 1u;
      got_full += got ? 1u : 0u;
      const bool done = got && s.node[st] == kDone;
      bool ok = got;
      if (got && !done) {
        ok = mbar_wait_bounded(smem_u32(&s.mma_bar[acc]), ph_mma[acc]);
        ph_mma[acc] ^= 1u;
        pending[acc] = false;
      }
      // every consumer leaves together: on any thread's timeout, or at kDone
      if (consumers_any(!ok)) {
        if (tid == 0) s.flag = 0;
        break;
      }
      if (done) break;
      const uint32_t nn = s.nn[st], total = s.total[st];
      asm volatile("tcgen05.fence::after_thread_sync;");
      // ---- screen: each thread owns one row ----
      // Pair (r, c) may beat row r's k-th entry only if its screened distance
      // nr + nc - 2g is below thr + eps (nr + nc), i.e. hc - 2g < thr - (1-eps) nr
      // with hc = (1-eps) nc (eps = 2^-12). Candidates are ranked by hc - 2g.
      const bool live = r < total;
      const float lim = live ? s.kth[st][r] - s.hnrm[st][r] : -INFINITY;
      float bd[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
      uint32_t bc[4] = {kInv, kInv, kInv, kInv};
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if ((uint32_t)t >= T) bd[t] = -INFINITY;  // unused slots never accept
      // columns a row may pair with: all others if r is new, new ones if old;
      // the warp reads only the column blocks one of its rows needs
      const uint32_t cmax = live ? ((r < nn) ? total : nn) : 0u;
      const uint32_t wmax = __reduce_max_sync(kFull, cmax);
      // cut = min(lim, the row's current T-th kept value), refreshed only when
      // a pair is kept; a column takes the insertion branch only below it
      float cut = fminf(lim, T == 1 ? bd[0] : (T == 2 ? bd[1] : (T == 3 ? bd[2] : bd[3])));
#pragma unroll 1
      for (uint32_t q = 0; q * 32 < wmax; ++q) {
        float g[32];
        tmem_ld32(tmem + acc * 128 + ((warp * 32u) << 16) + q * 32u, g);
        if (q * 32 >= cmax) continue;  // no column of this block pairs with row r
        const float4* h4 = reinterpret_cast<const float4*>(&s.hnrm[st][q * 32]);
#pragma unroll
        for (int k4 = 0; k4 < 8; ++k4) {
          const float4 h = h4[k4];
          float v4[4];
          fma2_m2(g[4 * k4], g[4 * k4 + 1], h.x, h.y, v4[0], v4[1]);
          fma2_m2(g[4 * k4 + 2], g[4 * k4 + 3], h.z, h.w, v4[2], v4[3]);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t c = q * 32 + 4 * k4 + j;
            if (v4[j] < cut && c < cmax && c != r) {
              float v = v4[j];
              uint32_t vc = c;
#pragma unroll
              for (int t = 0; t < 4; ++t)
                if (v < bd[t]) {
                  swap_(v, bd[t]);
                  swap_(vc, bc[t]);
                }
              cut = fminf(lim, T == 1 ? bd[0] : (T == 2 ? bd[1] : (T == 3 ? bd[2] : bd[3])));
            }
          }
        }
      }
      // kept pairs go to one list so that the exact re-rank is shared evenly
      uint32_t kept = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t) kept += bc[t] != kInv ? 1u : 0u;
      uint32_t incl = kept;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kFull, incl, o);
        if (lane >= (uint32_t)o) incl += v;
      }
      if (lane == 31) s.warp_pairs[warp] = incl;
      // every consumer has read the accumulator: node i + 1's tile may go in
      asm volatile("tcgen05.fence::before_thread_sync;");
      consumers_sync();
      if (tid == 0) {
        const int st1 = (int)((i + 1) % kStages);
        issue(st1, ph_full[st1], 0u);  // the phase node i + 1 completes
      }
      uint32_t off = incl - kept, npairs = 0;
#pragma unroll
      for (int w = 0; w < kConsumers / 32; ++w) {
        const uint32_t c = s.warp_pairs[w];
        if ((uint32_t)w < warp) off += c;
        npairs += c;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (bc[t] != kInv) s.pairs[off++] = (r << 16) | bc[t];
      consumers_sync();
      // ---- exact re-rank of the kept pairs ----
      for (uint32_t q = tid; q < npairs; q += kConsumers) {
        const uint32_t pr = s.pairs[q], row = pr >> 16, col = pr & 0xFFFFu;
        const float d = tile_dist<D>(s.tile[st], row, col, dim);
        ++n_pairs;
        if (d < s.kth[st][row]) {
          propose(pool, s.ids[st][row], P, s.ids[st][col], d);
          ++n_props;
        }
      }
      __syncwarp();
      if ((tid & 31u) == 0) mbar_arrive(smem_u32(&s.empty_bar[st]));
    }
    if (tid == 0) {
      // MMAs committed but not consumed (only after a timeout) land first
      for (int a = 0; a < 2; ++a)
        if (pending[a]) mbar_wait_bounded(smem_u32(&s.mma_bar[a]), ph_mma[a]);
      s.consumed = got_full;
    }
  }
  __syncthreads();
  if (tid == 0 && !s.flag) {
    // after a timeout, row copies the consumers never waited for land before
    // the block's shared memory is released (at most kStages of them)
    for (uint32_t j = s.consumed; j < s.filled; ++j)
      mbar_wait_bounded(smem_u32(&s.full_bar[j % kStages]), (j / kStages) & 1u);
  }
  __syncthreads();
  if (!s.flag && tid == 0) atomicExch(err, 1);
  if (n_props) atomicAdd(&stats[0], n_props);
  if (n_pairs) atomicAdd(&stats[1], n_pairs);
  if (n_rows) atomicAdd(&stats[3], n_rows);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
}

// ---------------------------------------------------------------------------
// Wide rows (128 < d <= 1024). A 128-row FP16 tile no longer fits in shared
// memory, so the Gram tile accumulates over K as a GEMM's K loop does: the
// producer warp gathers one 64-half column block of the node's rows at a time
// into a ring of stages, a dedicated MMA warp adds each block's four K = 16
// steps into one of two TMEM accumulators and frees the stage when its MMAs
// complete, and the four consumer warps screen the finished tile exactly as
// k_join_tc does. The kept pairs are re-ranked from the base rows in global
// memory (the tile's rows have left the ring by then). TMA fills past d with
// zeros, which leave the Gram sums unchanged. The FP32 accumulation error of a
// Gram entry over d <= 1024 terms stays below 1024 * 2^-24 * (n_r + n_c) / 2 =
// 2^-15 (n_r + n_c), inside the screen's 2^-12 (n_r + n_c) margin.
constexpr int kWideRing = 6;                       // column blocks in flight
constexpr int kWideNodes = 2;                      // node metadata slots
constexpr int kWideThreads = kConsumers + 64;      // consumers, producer (warp 4), MMA (warp 5)
constexpr uint32_t kWideTmemCols = 256;            // two 128-column accumulators

struct __align__(1024) WideSmem {
  uint8_t ring[kWideRing][kMaxList][128];  // one column block: [row][128 B], SW128
  uint32_t ids[kWideNodes][kMaxList];
  float hnrm[kWideNodes][kMaxList];  // (1 - 2^-12) x exact squared norm
  float kth[kWideNodes][kMaxList];
  uint32_t pairs[kConsumers * 4];
  uint32_t warp_pairs[kConsumers / 32];
  unsigned long long ring_full[kWideRing], ring_empty[kWideRing];
  unsigned long long node_full[kWideNodes], node_empty[kWideNodes];
  unsigned long long acc_full[2], acc_empty[2], drain;
  uint32_t taddr;
  uint32_t node[kWideNodes], nn[kWideNodes], total[kWideNodes];
  uint32_t filled, taken;  // column blocks the producer issued / the MMA warp waited for
  int flag;
};

// Producer warp of the wide join: node metadata into slot j % 2, then the
// node's column blocks, each into the next ring stage once the MMAs that read
// it before have completed.
__device__ void wide_producer(WideSmem& s, const CUtensorMap& tmap, const float2* __restrict__ meta,
                              const uint32_t* __restrict__ lists,
                              const uint32_t* __restrict__ lcnt, uint32_t n, uint32_t dim,
                              uint32_t K, unsigned long long* n_rows,
                              const uint32_t* __restrict__ order) {
  const uint32_t lane = threadIdx.x & 31u, blocks = (dim + 63) / 64;
  uint32_t next = blockIdx.x, fill = 0;
  uint32_t ph_node[kWideNodes] = {};
  for (uint32_t j = 0;; ++j) {
    const int ns = (int)(j % kWideNodes);
    if (j >= (uint32_t)kWideNodes) {
      bool ok = true;
      if (lane == 0) {
        ok = mbar_wait_bounded(smem_u32(&s.node_empty[ns]), ph_node[ns]);
        if (!ok) s.flag = 0;
      }
      ph_node[ns] ^= 1u;
      if (!__shfl_sync(kFull, ok ? 1 : 0, 0)) return;
    }
    uint32_t u = kDone, nn = 0, tot = 0;
    while (next < n) {
      const uint32_t c = next + lane * gridDim.x;
      const uint32_t node = c < n ? (order ? __ldg(order + c) : c) : 0u;
      uint2 cnt = make_uint2(0, 0);
      if (c < n) cnt = *reinterpret_cast<const uint2*>(lcnt + 2 * (size_t)node);
      const unsigned ok = __ballot_sync(kFull, c < n && cnt.x > 0 && cnt.y >= 2);
      if (ok) {
        const int w = __ffs(ok) - 1;
        u = __shfl_sync(kFull, node, w);
        nn = __shfl_sync(kFull, cnt.x, w);
        tot = __shfl_sync(kFull, cnt.y, w);
        next += ((uint32_t)w + 1u) * gridDim.x;
        break;
      }
      next += 32u * gridDim.x;
    }
    for (uint32_t t = lane; t < tot; t += 32) {
      const uint32_t id = lists[(size_t)u * kMaxList + t];
      s.ids[ns][t] = id;
      const float2 m = __ldg(meta + id);
      s.hnrm[ns][t] = kOneMinusEps * m.x;
      s.kth[ns][t] = m.y;
    }
    if (lane == 0) {
      s.node[ns] = u;
      s.nn[ns] = nn;
      s.total[ns] = tot;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&s.node_full[ns]));
    if (u == kDone) return;
    if (lane == 0) *n_rows += tot;
    const uint32_t groups = (tot + 3) / 4;
    for (uint32_t b = 0; b < blocks; ++b, ++fill) {
      const int slot = (int)(fill % kWideRing);
      const uint32_t bar = smem_u32(&s.ring_full[slot]);
      bool ok = true;
      if (lane == 0) {
        if (fill >= (uint32_t)kWideRing)
          ok = mbar_wait_bounded(smem_u32(&s.ring_empty[slot]), ((fill / kWideRing) - 1) & 1u);
        if (!ok) {
          s.flag = 0;
        } else {
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                       "r"(groups * 4 * 128)
                       : "memory");
          s.filled = fill + 1;
        }
      }
      if (!__shfl_sync(kFull, ok ? 1 : 0, 0)) return;
      for (uint32_t g = lane; g < groups; g += 32) {
        uint32_t r[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) r[t] = s.ids[ns][min(4 * g + t, tot - 1)];
        const uint32_t dst = smem_u32(&s.ring[slot][4 * g][0]);
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::"
            "bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
            "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(b * 64), "r"(r[0]), "r"(r[1]), "r"(r[2]),
            "r"(r[3]), "r"(bar)
            : "memory");
      }
    }
  }
}

// MMA thread of the wide join: node j's Gram tile into accumulator j % 2,
// one column block (four K = 16 steps) at a time.
__device__ void wide_mma(WideSmem& s, uint32_t tmem, uint32_t dim) {
  const uint32_t blocks = (dim + 63) / 64;
  uint32_t ph_node[kWideNodes] = {}, ph_acc[2] = {}, take = 0;
  for (uint32_t j = 0;; ++j) {
    const int ns = (int)(j % kWideNodes), acc = (int)(j % 2);
    if (!mbar_wait_bounded(smem_u32(&s.node_full[ns]), ph_node[ns])) {
      s.flag = 0;
      break;
    }
    ph_node[ns] ^= 1u;
    if (s.node[ns] == kDone) {
      mbar_arrive(smem_u32(&s.acc_full[acc]));  // wakes the consumers, who see kDone
      break;
    }
    if (j >= 2) {
      if (!mbar_wait_bounded(smem_u32(&s.acc_empty[acc]), ph_acc[acc])) {
        s.flag = 0;
        break;
      }
      ph_acc[acc] ^= 1u;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    bool ok = true;
    for (uint32_t b = 0; b < blocks && ok; ++b, ++take) {
      const int slot = (int)(take % kWideRing);
      ok = mbar_wait_bounded(smem_u32(&s.ring_full[slot]), (take / kWideRing) & 1u);
      if (!ok) break;
      s.taken = take + 1;
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) {
        const uint64_t desc = sw128_desc(smem_u32(&s.ring[slot][0][0]) + k * 32);
        const uint32_t accum = (b | k) != 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + acc * 128),
            "l"(desc), "l"(desc), "r"(kIdesc), "r"(accum));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&s.ring_empty[slot])));
    }
    if (!ok) {
      s.flag = 0;
      break;
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(&s.acc_full[acc])));
  }
  // every MMA this thread issued has completed before TMEM is released
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
      smem_u32(&s.drain)));
  if (!mbar_wait_bounded(smem_u32(&s.drain), 0)) s.flag = 0;
}

__global__ void __launch_bounds__(kWideThreads, 2)
    k_join_tc_wide(const __grid_constant__ CUtensorMap tmap, const __half* __restrict__ data,
                   const float2* __restrict__ meta, const uint32_t* __restrict__ lists, const uint32_t* __restrict__ lcnt,
                   uint32_t n, uint32_t dim, uint32_t K, uint32_t T, uint32_t P,
                   unsigned long long* __restrict__ pool, unsigned long long* __restrict__ stats,
                   int* __restrict__ err, const uint32_t* __restrict__ order) {
  extern __shared__ unsigned char smem_raw[];
  WideSmem& s = *reinterpret_cast<WideSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s.taddr)),
                 "r"(kWideTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < kWideRing; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.ring_full[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.ring_empty[i])));
    }
    for (int i = 0; i < kWideNodes; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.node_full[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&s.node_empty[i])));
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.acc_full[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&s.acc_empty[i])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.drain)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    asm volatile("fence.proxy.async.shared::cta;");
    s.flag = 1;
    s.filled = 0;
    s.taken = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s.taddr;
  unsigned long long n_pairs = 0, n_props = 0, n_rows = 0;

  if (warp == 4) {
    wide_producer(s, tmap, meta, lists, lcnt, n, dim, K, &n_rows, order);
  } else if (warp == 5) {
    if ((tid & 31u) == 0) wide_mma(s, tmem, dim);
    __syncwarp();
  } else {
    uint32_t ph_node[kWideNodes] = {}, ph_acc[2] = {};
    const uint32_t r = tid, lane = tid & 31u;
    for (uint32_t i = 0;; ++i) {
      const int ns = (int)(i % kWideNodes), acc = (int)(i % 2);
      bool ok = mbar_wait_bounded(smem_u32(&s.node_full[ns]), ph_node[ns]);
      ph_node[ns] ^= 1u;
      if (ok) ok = mbar_wait_bounded(smem_u32(&s.acc_full[acc]), ph_acc[acc]);
      ph_acc[acc] ^= 1u;
      // every consumer leaves together: on any thread's timeout, or at kDone
      if (consumers_any(!ok)) {
        if (tid == 0) s.flag = 0;
        break;
      }
      if (s.node[ns] == kDone) break;
      const uint32_t nn = s.nn[ns], total = s.total[ns];
      asm volatile("tcgen05.fence::after_thread_sync;");
      // ---- screen: the same rule and order as k_join_tc ----
      const bool live = r < total;
      const float lim = live ? s.kth[ns][r] - s.hnrm[ns][r] : -INFINITY;
      float bd[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
      uint32_t bc[4] = {kInv, kInv, kInv, kInv};
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if ((uint32_t)t >= T) bd[t] = -INFINITY;
      const uint32_t cmax = live ? ((r < nn) ? total : nn) : 0u;
      const uint32_t wmax = __reduce_max_sync(kFull, cmax);
      float cut = fminf(lim, T == 1 ? bd[0] : (T == 2 ? bd[1] : (T == 3 ? bd[2] : bd[3])));
#pragma unroll 1
      for (uint32_t q = 0; q * 32 < wmax; ++q) {
        float g[32];
        tmem_ld32(tmem + acc * 128 + ((warp * 32u) << 16) + q * 32u, g);
        if (q * 32 >= cmax) continue;
        const float4* h4 = reinterpret_cast<const float4*>(&s.hnrm[ns][q * 32]);
#pragma unroll
        for (int k4 = 0; k4 < 8; ++k4) {
          const float4 h = h4[k4];
          float v4[4];
          fma2_m2(g[4 * k4], g[4 * k4 + 1], h.x, h.y, v4[0], v4[1]);
          fma2_m2(g[4 * k4 + 2], g[4 * k4 + 3], h.z, h.w, v4[2], v4[3]);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t c = q * 32 + 4 * k4 + j;
            if (v4[j] < cut && c < cmax && c != r) {
              float v = v4[j];
              uint32_t vc = c;
#pragma unroll
              for (int t = 0; t < 4; ++t)
                if (v < bd[t]) {
                  swap_(v, bd[t]);
                  swap_(vc, bc[t]);
                }
              cut = fminf(lim, T == 1 ? bd[0] : (T == 2 ? bd[1] : (T == 3 ? bd[2] : bd[3])));
            }
          }
        }
      }
      // the accumulator is read: the MMA warp may refill it with node i + 2
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&s.acc_empty[acc]));
      uint32_t kept = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t) kept += bc[t] != kInv ? 1u : 0u;
      uint32_t incl = kept;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kFull, incl, o);
        if (lane >= (uint32_t)o) incl += v;
      }
      if (lane == 31) s.warp_pairs[warp] = incl;
      consumers_sync();
      uint32_t off = incl - kept, npairs = 0;
#pragma unroll
      for (int w = 0; w < kConsumers / 32; ++w) {
        const uint32_t c = s.warp_pairs[w];
        if ((uint32_t)w < warp) off += c;
        npairs += c;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (bc[t] != kInv) s.pairs[off++] = (r << 16) | bc[t];
      consumers_sync();
      // ---- exact re-rank of the kept pairs from the base rows ----
      // Four lanes per pair, one level-2 quarter p of the reference tree each
      // (dist_pairs_rounds), combined in that function's order: p += p + 2,
      // then p0 += p1, then x + y. Each lane walks a quarter of the loads.
      const uint32_t sub = lane & 3u;
      for (uint32_t base = 0; base < npairs; base += kConsumers / 4) {
        const uint32_t q = base + (tid >> 2);
        const bool have = q < npairs;
        float x[2] = {0.0f, 0.0f}, y[2] = {0.0f, 0.0f};
        uint32_t row = 0, a = 0, c = 0;
        if (have) {
          const uint32_t pr = s.pairs[q];
          row = pr >> 16;
          a = s.ids[ns][row];
          c = s.ids[ns][pr & 0xFFFFu];
          const uint4* A4 = reinterpret_cast<const uint4*>(data + (size_t)a * dim);
          const uint4* B4 = reinterpret_cast<const uint4*>(data + (size_t)c * dim);
          auto load = [&](uint32_t u, int w) { return __ldg((w ? B4 : A4) + u); };
          // the 960-dim width at compile time, so that the quarter's loads
          // are issued ahead of its sums
          if (dim == 960)
            level2_pair_fixed<120>(load, (int)sub, x, y);
          else
            level2_pair_rounds(load, (int)sub, dim >> 3, x, y);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float ox = __shfl_xor_sync(kFull, x[h], 2), oy = __shfl_xor_sync(kFull, y[h], 2);
          if (sub < 2) add2(x[h], y[h], ox, oy);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float ox = __shfl_xor_sync(kFull, x[h], 1), oy = __shfl_xor_sync(kFull, y[h], 1);
          if (sub == 0) add2(x[h], y[h], ox, oy);
        }
        if (have && sub == 0) {
          add2(x[0], y[0], x[1], y[1]);
          const float d = __fadd_rn(x[0], y[0]);
          ++n_pairs;
          if (d < s.kth[ns][row]) {
            propose(pool, a, P, c, d);
            ++n_props;
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&s.node_empty[ns]));
    }
  }
  __syncthreads();
  if (tid == 0 && !s.flag) {
    // after a timeout, column blocks the MMA thread never waited for land
    // before the block's shared memory is released
    for (uint32_t f = s.taken; f < s.filled; ++f)
      mbar_wait_bounded(smem_u32(&s.ring_full[f % kWideRing]), (f / kWideRing) & 1u);
  }
  __syncthreads();
  if (!s.flag && tid == 0) atomicExch(err, 1);
  if (n_props) atomicAdd(&stats[0], n_props);
  if (n_pairs) atomicAdd(&stats[1], n_pairs);
  if (n_rows) atomicAdd(&stats[3], n_rows);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kWideTmemCols));
}

// One block that waits, bounded, on an mbarrier nothing arrives on, holding
// TMEM as the join kernels do: the wait runs out after kWaitNs, the block
// records it, frees its TMEM and returns.
__global__ void k_wait_selftest(int* __restrict__ timed_out) {
  __shared__ __align__(8) unsigned long long bar;
  __shared__ uint32_t taddr;
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(&taddr)),
               "r"(32u));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  __syncwarp();
  if (threadIdx.x == 0 && !mbar_wait_bounded(smem_u32(&bar), 0)) *timed_out = 1;
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncwarp();
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(32u));
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_row_map(CUtensorMap* map, const __half* base, uint32_t n, uint32_t dim) {
  // looked up once; a function-local static is initialised once across threads
  static const EncodeTiled fn = []() -> EncodeTiled {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        !p || q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  if (!fn) return fail(TAGORE_ECUDA, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t gdim[2] = {dim, n};
  const cuuint64_t gstride[1] = {(cuuint64_t)dim * 2};
  const cuuint32_t box[2] = {64, 1};
  const cuuint32_t estride[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, (void*)base, gdim, gstride, box,
                        estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TAGORE_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TAGORE_OK;
}

template <int D>
int launch(const Work& w, const CUtensorMap& map, cudaStream_t s) {
  // More than a quarter of an SM's shared memory per block keeps residency at
  // three blocks per SM, so their 3 x 128 TMEM columns always fit.
  const size_t sm = std::max<size_t>(sizeof(TcSmem) + 1024, 60 * 1024);
  TG_CUDA(cudaFuncSetAttribute((const void*)k_join_tc<D>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int* err = reinterpret_cast<int*>(w.stats + 4);
  k_join_tc<D><<<sms * 3, kThreads, sm, s>>>(map, w.meta, w.lists, w.lcnt, w.n, w.dim,
                                             w.K, w.T, w.P, w.pool, w.stats, err, w.order);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

int launch_wide(const Work& w, const CUtensorMap& map, cudaStream_t s) {
  const size_t sm = sizeof(WideSmem) + 1024;
  TG_CUDA(cudaFuncSetAttribute((const void*)k_join_tc_wide,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int* err = reinterpret_cast<int*>(w.stats + 4);
  k_join_tc_wide<<<sms * 2, kWideThreads, sm, s>>>(map, w.data, w.meta, w.lists, w.lcnt,
                                                    w.n, w.dim, w.K, w.T, w.P, w.pool, w.stats, err,
                                                    w.order);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

}  // namespace

int wait_selftest(int* timed_out, cudaStream_t s) {
  Scratch flag(s);
  TG_TRY(flag.alloc(sizeof(int)));
  TG_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  k_wait_selftest<<<1, 32, 0, s>>>(flag.as<int>());
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cudaMemcpyAsync(timed_out, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

int join_tc_wide(const Work& w, cudaStream_t s) {
  if (!tc_wide_supported(w.dim))
    return fail(TAGORE_EINVAL, "wide tensor-core join needs 128 < DIM <= 1024, DIM %% 8 == 0 (got %u)",
                w.dim);
  if (w.T > 4) return fail(TAGORE_EINVAL, "tensor-core join keeps at most 4 partners per row");
  CUtensorMap map;
  TG_TRY(make_row_map(&map, w.data, w.n, w.dim));
  return launch_wide(w, map, s);
}

int join_tc(const Work& w, cudaStream_t s) {
  if (w.dim > 128 || w.dim % 16)
    return fail(TAGORE_EINVAL, "tensor-core join needs DIM in {16,32,..,128} (got %u)", w.dim);
  if (w.T > 4) return fail(TAGORE_EINVAL, "tensor-core join keeps at most 4 partners per row");
  CUtensorMap map;
  TG_TRY(make_row_map(&map, w.data, w.n, w.dim));
  switch (w.dim) {
    case 96: return launch<96>(w, map, s);
    case 128: return launch<128>(w, map, s);
    default: return launch<0>(w, map, s);
  }
}

}  // namespace knn
}  // namespace tagore
