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

}  // namespace

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
