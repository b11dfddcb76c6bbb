// prep.cu -- FP32 input to the reference's FP16 base on the device.
//
// GNN_descent prepares its base on the host (pybind.cu:24-61): a power-of-ten
// factor from vector 0, the centroid as a sequential float sum, and an FP16
// copy of base * factor. The factor and centroid stay on the host here (they
// need vector 0 and a fixed summation order; host_center() runs on host
// threads while the device builds the graph); the bulk conversion and the
// squared norms run on the device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <thread>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace tagore {
namespace {

// One warp per row: base * factor rounded to FP16 (as __float2half), and the
// exact squared norm of the FP16 row in FP32.
__global__ void k_to_half(const float* __restrict__ raw, uint32_t n, uint32_t dim, float factor,
                          __half* __restrict__ out, float* __restrict__ norms) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const float* src = raw + (size_t)r * dim;
    __half* dst = out + (size_t)r * dim;
    float acc = 0.0f;
    for (uint32_t j = lane * 4; j < dim; j += 128) {
      const float4 v = *reinterpret_cast<const float4*>(src + j);
      const __half2 lo = __halves2half2(__float2half_rn(__fmul_rn(v.x, factor)),
                                        __float2half_rn(__fmul_rn(v.y, factor)));
      const __half2 hi = __halves2half2(__float2half_rn(__fmul_rn(v.z, factor)),
                                        __float2half_rn(__fmul_rn(v.w, factor)));
      *reinterpret_cast<__half2*>(dst + j) = lo;
      *reinterpret_cast<__half2*>(dst + j + 2) = hi;
      const float2 a = __half22float2(lo), b = __half22float2(hi);
      acc = fmaf(a.x, a.x, acc);
      acc = fmaf(a.y, a.y, acc);
      acc = fmaf(b.x, b.x, acc);
      acc = fmaf(b.y, b.y, acc);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off);
    if (lane == 0 && norms) norms[r] = acc;
  }
}

// fvecs records [int32 d][d floats] to dense rows. One warp per record; a
// record whose count is not `dim` is reported as (index + 1) in *bad (the
// smallest such index wins) and its row is left unwritten.
__global__ void k_unpack_fvecs(const uint32_t* __restrict__ rec, uint32_t cnt, uint32_t dim,
                               uint64_t row0, float* __restrict__ out,
                               unsigned long long* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < cnt; r += warps) {
    const uint32_t* src = rec + (size_t)r * (dim + 1);
    if (src[0] != dim) {
      if (lane == 0) atomicMin(bad, (unsigned long long)(row0 + r + 1));
      continue;
    }
    float* dst = out + (size_t)(row0 + r) * dim;
    for (uint32_t j = lane; j < dim; j += 32) dst[j] = __uint_as_float(src[1 + j]);
  }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
}

constexpr uint32_t kCenterRows = 256;  // rows per shared-memory tile
constexpr uint32_t kCenterThreads = 256;

// Centroid of pybind.cu:39-51 on the device: lane j of warp 0 adds column
// c0 + j over the rows in order, one float add at a time -- the reference's
// sequential sum, so the result is the same float. The other warps only help
// to stage tiles of kCenterRows x 32 columns through shared memory with
// cp.async, one tile ahead of the sum.
__global__ void __launch_bounds__(kCenterThreads) k_center_seq(const float* __restrict__ raw,
                                                               uint32_t n, uint32_t dim,
                                                               float factor,
                                                               __half* __restrict__ center) {
  extern __shared__ __align__(16) float tile[];  // [2][kCenterRows][32]
  const uint32_t c0 = blockIdx.x * 32;
  const uint32_t width = min(32u, dim - c0);     // a multiple of 4 (dim % 4 == 0)
  const uint32_t chunks = width / 4;              // 16-byte pieces per row
  const uint32_t tiles = (n + kCenterRows - 1) / kCenterRows;
  auto issue = [&](uint32_t t) {
    float* buf = tile + (t & 1) * kCenterRows * 32;
    const uint32_t r0 = t * kCenterRows;
    const uint32_t rows = min(kCenterRows, n - r0);
    for (uint32_t i = threadIdx.x; i < rows * chunks; i += kCenterThreads) {
      const uint32_t r = i / chunks, c = i % chunks;
      cp_async16(buf + r * 32 + c * 4, raw + (size_t)(r0 + r) * dim + c0 + c * 4);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  float acc = 0.0f;
  issue(0);
  for (uint32_t t = 0; t < tiles; ++t) {
    if (t + 1 < tiles) {
      issue(t + 1);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const float* buf = tile + (t & 1) * kCenterRows * 32 + threadIdx.x;
      const uint32_t rows = min(kCenterRows, n - t * kCenterRows);
      if (threadIdx.x < width) {
#pragma unroll 8
        for (uint32_t r = 0; r < rows; ++r) acc = __fadd_rn(acc, buf[r * 32]);
      }
    }
    __syncthreads();  // the buffer is refilled by the issue of tile t + 2
  }
  if (threadIdx.x < width) {
    const float c = __fdiv_rn(acc, (float)n);
    center[c0 + threadIdx.x] = __float2half_rn(__fmul_rn(c, factor));
  }
}

}  // namespace

int device_center(const float* raw, uint32_t n, uint32_t dim, float factor, __half* center,
                  cudaStream_t s) {
  if (dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", dim);
  const size_t smem = 2ull * kCenterRows * 32 * sizeof(float);
  TG_CUDA(cudaFuncSetAttribute(k_center_seq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_center_seq<<<(dim + 31) / 32, kCenterThreads, smem, s>>>(raw, n, dim, factor, center);
  TG_CUDA(cudaGetLastError());
  count_launch();
  return TAGORE_OK;
}

// Streams an fvecs file to the device: records are read into two pinned
// chunks in turn, each copied while the next is read, and unpacked on the
// device into raw (n x dim FP32). *factor gets the power-of-ten factor of
// vector 0 (host_factor).
int ingest_fvecs(const char* path, uint32_t n, uint32_t dim, bool rescale, float* raw,
                 float* factor, cudaStream_t s) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(TAGORE_EIO, "cannot open '%s'", path);
  struct Closer {
    FILE* f;
    ~Closer() { std::fclose(f); }
  } closer{f};
  const size_t rec = 4ull * (dim + 1);
  const uint32_t per_chunk = (uint32_t)std::max<size_t>(1, ((size_t)32 << 20) / rec);
  const size_t chunk_bytes = rec * per_chunk;
  void* pinned[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  Scratch stage(s);
  struct Release {
    void** p;
    cudaEvent_t* e;
    ~Release() {
      for (int i = 0; i < 2; ++i) {
        if (e[i]) {
          cudaEventSynchronize(e[i]);
          cudaEventDestroy(e[i]);
        }
        if (p[i]) cudaFreeHost(p[i]);
      }
    }
  } release{pinned, ev};
  for (int i = 0; i < 2; ++i) {
    count_allocation();
    TG_CUDA(cudaMallocHost(&pinned[i], chunk_bytes));
    TG_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  }
  TG_TRY(stage.alloc(2 * chunk_bytes + 16));
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(stage.as<char>() + 2 * chunk_bytes);
  TG_CUDA(cudaMemsetAsync(bad, 0xFF, 8, s));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint32_t done = 0;
  for (uint32_t c = 0; done < n; ++c) {
    const int b = c & 1;
    const uint32_t cnt = std::min(per_chunk, n - done);
    TG_CUDA(cudaEventSynchronize(ev[b]));  // the copy out of this chunk (two reads ago) is done
    if (std::fread(pinned[b], 1, rec * cnt, f) != rec * cnt)
      return fail(TAGORE_EIO, "'%s': truncated at vector %u", path, done);
    if (c == 0) *factor = host_factor(static_cast<const float*>(pinned[0]) + 1, dim, rescale);
    char* dst = stage.as<char>() + b * chunk_bytes;
    TG_CUDA(cudaMemcpyAsync(dst, pinned[b], rec * cnt, cudaMemcpyHostToDevice, s));
    const uint32_t blocks = std::min<uint32_t>((cnt + 7) / 8, (uint32_t)sms * 8);
    k_unpack_fvecs<<<blocks, 256, 0, s>>>(reinterpret_cast<const uint32_t*>(dst), cnt, dim, done,
                                          raw, bad);
    TG_CUDA(cudaGetLastError());
    count_launch();
    TG_CUDA(cudaEventRecord(ev[b], s));
    done += cnt;
  }
  unsigned long long first_bad = 0;
  TG_CUDA(cudaMemcpyAsync(&first_bad, bad, 8, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  if (first_bad != ~0ull)
    return fail(TAGORE_EIO, "'%s': vector %llu does not have dim %u", path, first_bad - 1, dim);
  return TAGORE_OK;
}

int prep_base(const float* raw, uint32_t n, uint32_t dim, float factor, __half* data,
              float* norms, cudaStream_t s) {
  if (dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", dim);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_to_half<<<sms * 8, 256, 0, s>>>(raw, n, dim, factor, data, norms);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

// Power-of-ten factor of pybind.cu:24-36: vector 0's mean |x| brought into
// [0.5, 5]. An all-zero vector 0 (which would loop forever there) keeps 1.
float host_factor(const float* x, uint32_t dim, bool rescale) {
  float norm = 1.0f;
  if (!rescale) return norm;
  float ave = 0.0f;
  for (uint32_t i = 0; i < dim; ++i) ave += std::fabs(x[i]);
  ave /= (float)dim;
  if (ave > 0.0f && std::isfinite(ave)) {
    while (ave < 0.5f) {
      ave *= 10;
      norm *= 10;
    }
    while (ave > 5) {
      ave /= 10;
      norm /= 10;
    }
  }
  return norm;
}

// Centroid of pybind.cu:39-51: a sequential float sum per dimension (split
// over host threads by dimension, which keeps each sum's order), divided by
// n, times the factor, rounded to FP16.
void host_center(const float* x, uint32_t n, uint32_t dim, float factor, uint16_t* center_half) {
  std::vector<float> c(dim, 0.0f);
  const uint32_t hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  const uint32_t per = std::max<uint32_t>(16, (dim + hw - 1) / hw);
  std::vector<std::thread> th;
  for (uint32_t j0 = 0; j0 < dim; j0 += per) {
    const uint32_t j1 = std::min(dim, j0 + per);
    th.emplace_back([&, j0, j1]() {
      std::vector<float> acc(j1 - j0, 0.0f);
      for (uint32_t i = 0; i < n; ++i) {
        const float* row = x + (size_t)i * dim;
        for (uint32_t j = j0; j < j1; ++j) acc[j - j0] += row[j];
      }
      for (uint32_t j = j0; j < j1; ++j) c[j] = acc[j - j0];
    });
  }
  for (auto& t : th) t.join();
  for (uint32_t j = 0; j < dim; ++j) {
    c[j] /= (float)n;
    const __half h = __float2half_rn(c[j] * factor);
    center_half[j] = *reinterpret_cast<const uint16_t*>(&h);
  }
}

}  // namespace tagore
