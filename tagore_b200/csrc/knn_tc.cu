// knn_tc.cu -- local join on tcgen05 tensor cores (sm_100a).
//
// One block joins one node's list at a time (persistent blocks, at most three
// per SM so three 128-column TMEM accumulators always fit in the SM's 512):
//   1. TMA tile::gather4 copies the list's FP16 rows (<= 128) into a K-major
//      128-byte-swizzled tile X in shared memory (box 64 halves x 1 row);
//   2. one thread issues D/16 tcgen05.mma.kind::f16 (M = N = 128, K = 16),
//      X as both operands, so TMEM holds the Gram tile X X^T in FP32;
//   3. each thread owns one row: it reads its TMEM lane, forms the screened
//      distance n_r + n_c - 2 g_rc from exact FP32 norms, and keeps its
//      `per_row` closest partners that could beat the row's k-th entry
//      (screened value below k-th + margin, margin = 2^-12 (n_r + n_c), far
//      above the FP32 rounding of the Gram entry and of the norms);
//   4. the kept pairs are re-ranked exactly (reference-order FP32 from the
//      same shared tile, one warp per pair) and proposed only when the exact
//      value beats the k-th entry. No stored distance comes from a tensor core.
// Every wait is bounded by %globaltimer; on expiry the block records an error,
// waits (bounded) for its own copies, frees its TMEM and returns.
#include <cuda.h>

#include <algorithm>

#include "knn_shared.cuh"

namespace tagore {
namespace knn {
namespace {

constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s per wait

struct __align__(1024) TcSmem {
  uint8_t x[2][kMaxList][128];  // [64-half column block][row][128 B], SW128
  uint32_t ids[kMaxList];
  float nrm[kMaxList];
  float kth[kMaxList];
  unsigned long long tma_bar;
  unsigned long long mma_bar;
  uint32_t taddr;
  uint32_t nn, total;
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

// Chunk j (4 halves) of row r inside the swizzled tile.
__device__ __forceinline__ uint2 tile_chunk(const TcSmem& s, uint32_t r, uint32_t j) {
  const uint32_t blk = j >> 4, unit = ((j & 15u) >> 1) ^ (r & 7u), half8 = j & 1u;
  return *reinterpret_cast<const uint2*>(&s.x[blk][r][unit * 16 + half8 * 8]);
}

__global__ void __launch_bounds__(kThreads, 1)
    k_join_tc(const __grid_constant__ CUtensorMap tmap, const uint64_t* __restrict__ nb,
              const float* __restrict__ norms, const uint32_t* __restrict__ lists,
              const uint32_t* __restrict__ lcnt, uint32_t n, uint32_t dim, uint32_t K, uint32_t T,
              uint32_t P, unsigned long long* __restrict__ pool,
              unsigned long long* __restrict__ stats, int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  TcSmem& s = *reinterpret_cast<TcSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t tma_bar = smem_u32(&s.tma_bar), mma_bar = smem_u32(&s.mma_bar);
  const uint32_t ksteps = dim / 16, blocks = (dim + 63) / 64;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s.taddr)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tma_bar));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_bar));
    asm volatile("fence.mbarrier_init.release.cluster;");
    asm volatile("fence.proxy.async.shared::cta;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s.taddr;
  uint32_t phase = 0;
  unsigned long long n_pairs = 0, n_props = 0, n_rows = 0;
  bool failed = false;

  for (uint32_t u = blockIdx.x; u < n && !failed; u += gridDim.x) {
    if (tid == 0) {
      s.nn = lcnt[2 * u];
      s.total = lcnt[2 * u + 1];
    }
    __syncthreads();
    const uint32_t nn = s.nn, total = s.total;
    if (nn == 0 || total < 2) {
      __syncthreads();
      continue;
    }
    if (tid == 0) n_rows += total;
    if (tid < total) {
      const uint32_t id = lists[(size_t)u * kMaxList + tid];
      s.ids[tid] = id;
      s.nrm[tid] = norms[id];
      s.kth[tid] = kth_of(nb[(size_t)id * K + K - 1]);
    }
    __syncthreads();
    // ---- 1. gather rows (one thread issues every copy) ----
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const uint32_t groups = (total + 3) / 4;
      const uint32_t bytes = groups * 4 * 128 * blocks;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_bar),
                   "r"(bytes)
                   : "memory");
      for (uint32_t g = 0; g < groups; ++g) {
        uint32_t r[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) r[t] = s.ids[min(4 * g + t, total - 1)];
        for (uint32_t b = 0; b < blocks; ++b) {
          const uint32_t dst = smem_u32(&s.x[b][4 * g][0]);
          asm volatile(
              "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::"
              "bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
              "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(b * 64), "r"(r[0]), "r"(r[1]), "r"(r[2]),
              "r"(r[3]), "r"(tma_bar)
              : "memory");
        }
      }
      s.flag = mbar_wait_bounded(tma_bar, phase) ? 1 : 0;
    }
    __syncthreads();
    if (!s.flag) {
      failed = true;
      break;
    }
    mbar_try(tma_bar, phase);  // completed: gives every thread the acquire
    // ---- 2. Gram tile on the tensor cores ----
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      for (uint32_t k = 0; k < ksteps; ++k) {
        const uint32_t a = smem_u32(&s.x[k >> 2][0][0]) + (k & 3u) * 32;
        const uint64_t desc = sw128_desc(a);
        const uint32_t acc = k > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(desc), "l"(desc), "r"(kIdesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          mma_bar));
      s.flag = mbar_wait_bounded(mma_bar, phase) ? 1 : 0;
    }
    __syncthreads();
    if (!s.flag) {
      failed = true;
      break;
    }
    mbar_try(mma_bar, phase);
    asm volatile("tcgen05.fence::after_thread_sync;");
    phase ^= 1u;
    // ---- 3. screen: each thread owns one row ----
    const uint32_t r = tid;
    const bool live = r < total;
    const float nr = live ? s.nrm[r] : 0.0f;
    const float thr = live ? s.kth[r] : 0.0f;
    float bd[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    uint32_t bc[4] = {kInv, kInv, kInv, kInv};
#pragma unroll 1
    for (uint32_t q = 0; q < 4; ++q) {
      float g[32];
      tmem_ld32(tmem + ((warp * 32u) << 16) + q * 32u, g);
      if (live) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const uint32_t c = q * 32 + i;
          const float nc = s.nrm[c & (kMaxList - 1)];
          const bool ok = c < total && c != r && (r < nn || c < nn);
          const float dt = nr + nc - 2.0f * g[i];
          const float lim = thr + 0.000244140625f * (nr + nc);
          if (ok && dt < lim && dt < bd[T - 1]) {
            float v = dt;
            uint32_t vc = c;
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if ((uint32_t)t < T && v < bd[t]) {
                swap_(v, bd[t]);
                swap_(vc, bc[t]);
              }
          }
        }
      }
    }
    // ---- 4. exact re-rank, one warp per kept pair ----
#pragma unroll 1
    for (uint32_t t = 0; t < T; ++t) {
      unsigned m = __ballot_sync(kFull, live && bc[t] != kInv);
      while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t ra = warp * 32 + src;
        const uint32_t rb = __shfl_sync(kFull, bc[t], src);
        float x = 0.f, y = 0.f;
        for (uint32_t j = lane; j < dim / 4; j += 32) chunk_acc(tile_chunk(s, ra, j), tile_chunk(s, rb, j), x, y);
        const float d = warp_tree(x, y);
        if (lane == 0) {
          ++n_pairs;
          if (d < s.kth[ra]) {
            propose(pool, s.ids[ra], P, s.ids[rb], d);
            ++n_props;
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, 1);
      // let this block's own copies and MMAs land before TMEM is released
      mbar_wait_bounded(tma_bar, phase);
      mbar_wait_bounded(mma_bar, phase);
    }
    __syncthreads();
  }
  if (lane == 0) {
    atomicAdd(&stats[0], n_props);
    atomicAdd(&stats[1], n_pairs);
  }
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

}  // namespace

int join_tc(const Work& w, cudaStream_t s) {
  if (w.dim > 128 || w.dim % 16) return fail(TAGORE_EINVAL, "tensor-core join needs DIM in {16,32,..,128} (got %u)", w.dim);
  if (w.T > 4) return fail(TAGORE_EINVAL, "tensor-core join keeps at most 4 partners per row");
  CUtensorMap map;
  TG_TRY(make_row_map(&map, w.data, w.n, w.dim));
  // At least 57 KB of shared memory per block caps residency at three blocks
  // per SM, so their 3 x 128 TMEM columns always fit.
  const size_t sm = std::max<size_t>(sizeof(TcSmem) + 1024, 57 * 1024);
  TG_CUDA(cudaFuncSetAttribute((const void*)k_join_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sm));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int* err = reinterpret_cast<int*>(w.stats + 4);
  k_join_tc<<<sms * 3, kThreads, sm, s>>>(map, w.nb, w.norms, w.lists, w.lcnt, w.n, w.dim, w.K,
                                          w.T, w.P, w.pool, w.stats, err);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

}  // namespace knn
}  // namespace tagore
