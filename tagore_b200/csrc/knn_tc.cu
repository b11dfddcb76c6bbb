// knn_tc.cu -- local join on tcgen05 tensor cores (sm_100a).
//
// Persistent blocks (at most three per SM, so their three 128-column TMEM
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
//   4. each thread re-ranks its kept pairs exactly (reference-order FP32 from
//      the same shared tile) and proposes a pair only when the exact value beats
//      the k-th entry. No stored distance comes from a tensor core.
// Two tile stages pipeline the loop: while node i is screened and re-ranked,
// node i+1's rows are in flight and its MMA runs as soon as TMEM is free.
// Every wait is bounded by %globaltimer; on expiry the block records an error,
// waits (bounded) for its own copies and MMAs, frees its TMEM and returns.
#include <cuda.h>

#include <algorithm>

#include "knn_shared.cuh"

namespace tagore {
namespace knn {
namespace {

constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s per wait

struct __align__(1024) Tile {
  uint8_t x[2][kMaxList][128];  // [64-half column block][row][128 B], SW128
};

struct __align__(1024) TcSmem {
  Tile tile[2];
  uint32_t ids[2][kMaxList];
  float nrm[2][kMaxList];
  float kth[2][kMaxList];
  unsigned long long tma_bar[2];
  unsigned long long mma_bar;
  uint32_t taddr;
  uint32_t node[2], nn[2], total[2];
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
  }
  if constexpr (D > 0) {
    return serial_dist<D>([&](int j, int w) { return tile_chunk(t, w ? rb : ra, (uint32_t)j); });
  }
  float x[32], y[32];
#pragma unroll
  for (int l = 0; l < 32; ++l) {
    x[l] = 0.0f;
    y[l] = 0.0f;
  }
  if constexpr (D > 0) {
#pragma unroll
    for (int j = 0; j < D / 4; ++j) chunk_acc(tile_chunk(t, ra, j), tile_chunk(t, rb, j), x[j & 31], y[j & 31]);
  } else {
    for (uint32_t j = 0; j < dim / 4; ++j)
      chunk_acc(tile_chunk(t, ra, j), tile_chunk(t, rb, j), x[j & 31], y[j & 31]);
  }
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

template <int D>
__global__ void __launch_bounds__(kThreads, 1)
    k_join_tc(const __grid_constant__ CUtensorMap tmap, const uint64_t* __restrict__ nb,
              const float* __restrict__ norms, const uint32_t* __restrict__ lists,
              const uint32_t* __restrict__ lcnt, uint32_t n, uint32_t dim, uint32_t K, uint32_t T,
              uint32_t P, unsigned long long* __restrict__ pool,
              unsigned long long* __restrict__ stats, int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  TcSmem& s = *reinterpret_cast<TcSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t mma_bar = smem_u32(&s.mma_bar);
  const uint32_t ksteps = dim / 16, blocks = (dim + 63) / 64;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s.taddr)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.tma_bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.tma_bar[1])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_bar));
    asm volatile("fence.mbarrier_init.release.cluster;");
    asm volatile("fence.proxy.async.shared::cta;");
    s.flag = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s.taddr;
  uint32_t ph_tma[2] = {0, 0}, ph_mma = 0;
  unsigned long long n_pairs = 0, n_props = 0, n_rows = 0;

  // Finds this block's next joinable node at or after u into stage st, loads
  // its ids, starts its row copies and loads its norms and k-th distances.
  // Returns false at the end of the block's share.
  auto fetch = [&](uint32_t u, int st) -> bool {
    if (tid == 0) {
      uint32_t nn = 0, tot = 0;
      while (u < n) {
        nn = lcnt[2 * u];
        tot = lcnt[2 * u + 1];
        if (nn > 0 && tot >= 2) break;
        u += gridDim.x;
      }
      s.node[st] = u;
      s.nn[st] = nn;
      s.total[st] = tot;
    }
    __syncthreads();
    const uint32_t u2 = s.node[st], tot = s.total[st];
    if (u2 >= n) return false;
    if (tid < tot) s.ids[st][tid] = lists[(size_t)u2 * kMaxList + tid];
    __syncthreads();
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const uint32_t groups = (tot + 3) / 4, bar = smem_u32(&s.tma_bar[st]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                   "r"(groups * 4 * 128 * blocks)
                   : "memory");
      for (uint32_t g = 0; g < groups; ++g) {
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
      n_rows += tot;
    }
    if (tid < tot) {
      const uint32_t id = s.ids[st][tid];
      s.nrm[st][tid] = norms[id];
      s.kth[st][tid] = kth_of(nb[(size_t)id * K + K - 1]);
    }
    return true;
  };

  // Waits for stage st's rows (thread 0, bounded) and issues its MMAs.
  auto mma = [&](int st) {
    if (tid == 0) {
      if (!mbar_wait_bounded(smem_u32(&s.tma_bar[st]), ph_tma[st])) {
        s.flag = 0;
        return;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      for (uint32_t k = 0; k < ksteps; ++k) {
        const uint64_t desc = sw128_desc(smem_u32(&s.tile[st].x[k >> 2][0][0]) + (k & 3u) * 32);
        const uint32_t acc = k > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(desc), "l"(desc), "r"(kIdesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          mma_bar));
    }
  };

  int cur = 0;
  bool have = fetch(blockIdx.x, 0);
  __syncthreads();
  if (have) mma(0);
  __syncthreads();
  bool failed = s.flag == 0;
  while (have && !failed) {
    const int nxt = cur ^ 1;
    const uint32_t u = s.node[cur], nn = s.nn[cur], total = s.total[cur];
    // next node's rows go in flight while this one is finished
    const bool have_next = fetch(u + gridDim.x, nxt);
    // ---- Gram tile of the current node ----
    if (tid == 0 && s.flag) s.flag = mbar_wait_bounded(mma_bar, ph_mma) ? 1 : 0;
    __syncthreads();
    if (!s.flag) {
      failed = true;
      break;
    }
    mbar_try(mma_bar, ph_mma);
    mbar_try(smem_u32(&s.tma_bar[cur]), ph_tma[cur]);
    asm volatile("tcgen05.fence::after_thread_sync;");
    ph_mma ^= 1u;
    ph_tma[cur] ^= 1u;
    // ---- screen: each thread owns one row ----
    // Pair (r, c) may beat row r's k-th entry only if its screened distance
    // nr + nc - 2g is below thr + eps (nr + nc), i.e. hc - 2g < thr - (1-eps) nr
    // with hc = (1-eps) nc (eps = 2^-12). Candidates are ranked by hc - 2g.
    const uint32_t r = tid;
    const bool live = r < total;
    const float one_m = 1.0f - 0.000244140625f;
    const float lim = live ? s.kth[cur][r] - one_m * s.nrm[cur][r] : -INFINITY;
    float bd[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    uint32_t bc[4] = {kInv, kInv, kInv, kInv};
#pragma unroll
    for (int t = 0; t < 4; ++t)
      if ((uint32_t)t >= T) bd[t] = -INFINITY;  // unused slots never accept
    // columns a row may pair with: all others if r is new, new ones if old
    const uint32_t cmax = (r < nn) ? total : nn;
#pragma unroll 1
    for (uint32_t q = 0; q < 4; ++q) {
      float g[32];
      tmem_ld32(tmem + ((warp * 32u) << 16) + q * 32u, g);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const uint32_t c = q * 32 + i;
        const float v0 = fmaf(-2.0f, g[i], one_m * s.nrm[cur][c]);
        const float worst = T == 1 ? bd[0] : (T == 2 ? bd[1] : (T == 3 ? bd[2] : bd[3]));
        if (v0 < lim && v0 < worst && c < cmax && c != r) {
          float v = v0;
          uint32_t vc = c;
#pragma unroll
          for (int t = 0; t < 4; ++t)
            if (v < bd[t]) {
              swap_(v, bd[t]);
              swap_(vc, bc[t]);
            }
        }
      }
    }
    // TMEM is free: start the next node's MMA (its rows are likely in already)
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (have_next) mma(nxt);
    // ---- exact re-rank of the kept pairs, thread per row ----
    if (live) {
      const uint32_t a = s.ids[cur][r];
      const float thr = s.kth[cur][r];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (bc[t] == kInv) continue;  // unused and empty slots
        const float d = tile_dist<D>(s.tile[cur], r, bc[t], dim);
        ++n_pairs;
        if (d < thr) {
          propose(pool, a, P, s.ids[cur][bc[t]], d);
          ++n_props;
        }
      }
    }
    __syncthreads();
    have = have_next;
    cur = nxt;
    failed = s.flag == 0;
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, 1);
      // let this block's own copies and MMAs land before TMEM is released
      mbar_wait_bounded(smem_u32(&s.tma_bar[0]), ph_tma[0]);
      mbar_wait_bounded(smem_u32(&s.tma_bar[1]), ph_tma[1]);
      mbar_wait_bounded(mma_bar, ph_mma);
    }
    __syncthreads();
  }
  if (n_props) atomicAdd(&stats[0], n_props);
  if (n_pairs) atomicAdd(&stats[1], n_pairs);
  if (tid == 0) atomicAdd(&stats[3], n_rows);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_row_map(CUtensorMap* map, const __half* base, uint32_t n, uint32_t dim) {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    TG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      return fail(TAGORE_ECUDA, "cuTensorMapEncodeTiled is unavailable");
    fn = reinterpret_cast<EncodeTiled>(p);
  }
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
  // At least 72 KB of shared memory per block caps residency at three blocks
  // per SM, so their 3 x 128 TMEM columns always fit.
  const size_t sm = std::max<size_t>(sizeof(TcSmem) + 1024, 72 * 1024);
  TG_CUDA(cudaFuncSetAttribute((const void*)k_join_tc<D>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int* err = reinterpret_cast<int*>(w.stats + 4);
  k_join_tc<D><<<sms * 3, kThreads, sm, s>>>(map, w.nb, w.norms, w.lists, w.lcnt, w.n, w.dim,
                                             w.K, w.T, w.P, w.pool, w.stats, err);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

}  // namespace

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
