// mlp.cu -- the learned candidate screen of the chosen kNN path (sm_100a).
//
// No counterpart in the reference. A small MLP z = W2^T relu(W1^T x + b1) + b2
// (d -> 128 -> 32) maps each FP16 base row to 32 numbers. It is trained on the
// GPU, with the kernels below, on triplets (a, p, m) taken from the kNN rows
// the first GNN-Descent iterations built: exact FP32 distances there order
// d(a, p) < d(a, m), and the loss softplus(log Dp - log Dm) on the projected
// squared distances asks the projection to keep that order. The join then
// screens candidate pairs by projected distance and re-ranks the kept ones
// exactly; no stored distance comes from the projection.
//
// Training runs in FP32 on master weights with Adam; the projection of the
// whole base uses BF16 copies of the weights with FP32 accumulation.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "mlp.cuh"

namespace tagore {
namespace mlp {
namespace {

constexpr int kRowsPerBlock = 16;

// Forward pass over rows[0, nrows): pre-activations (nrows x 128) and outputs
// (nrows x 32), FP32. One block per 16 rows; thread j owns hidden unit j.
__global__ void __launch_bounds__(kHidden)
    k_forward(const uint32_t* __restrict__ rows, uint32_t nrows, const __half* __restrict__ data,
              uint32_t dim, const float* __restrict__ mean, const float* __restrict__ w1,
              const float* __restrict__ b1, const float* __restrict__ w2,
              const float* __restrict__ b2, float* __restrict__ pre, float* __restrict__ z) {
  extern __shared__ float xs[];  // [16][dim], then h [16][128]
  float* hs = xs + kRowsPerBlock * dim;
  const uint32_t j = threadIdx.x, r0 = blockIdx.x * kRowsPerBlock;
  const uint32_t nr = min((uint32_t)kRowsPerBlock, nrows - r0);
  for (uint32_t i = j; i < nr * dim; i += kHidden) {
    const uint32_t r = i / dim, k = i % dim;
    xs[r * dim + k] = __half2float(data[(size_t)rows[r0 + r] * dim + k]) - mean[k];
  }
  __syncthreads();
  float acc[kRowsPerBlock];
#pragma unroll
  for (int r = 0; r < kRowsPerBlock; ++r) acc[r] = b1[j];
  for (uint32_t k = 0; k < dim; ++k) {
    const float w = w1[(size_t)k * kHidden + j];
#pragma unroll
    for (int r = 0; r < kRowsPerBlock; ++r) acc[r] = fmaf(xs[r * dim + k], w, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < kRowsPerBlock; ++r) {
    if ((uint32_t)r < nr) pre[(size_t)(r0 + r) * kHidden + j] = acc[r];
    hs[r * kHidden + j] = fmaxf(acc[r], 0.0f);
  }
  __syncthreads();
  for (uint32_t o = j; o < nr * kOut; o += kHidden) {
    const uint32_t r = o / kOut, c = o % kOut;
    float s = b2[c];
    for (uint32_t h = 0; h < kHidden; ++h) s = fmaf(hs[r * kHidden + h], w2[h * kOut + c], s);
    z[(size_t)(r0 + r) * kOut + c] = s;
  }
}

// Loss of each triplet (rows 3t, 3t+1, 3t+2 of the batch) and dL/dz, scaled
// by 1/B so that the gradients are those of the batch mean.
__global__ void k_loss(uint32_t B, const float* __restrict__ z, float* __restrict__ dz,
                       double* __restrict__ loss) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B) return;
  const float* za = z + (size_t)(3 * t) * kOut;
  const float* zp = za + kOut;
  const float* zm = zp + kOut;
  float dp = 0.0f, dm = 0.0f;
#pragma unroll
  for (int c = 0; c < kOut; ++c) {
    const float ep = za[c] - zp[c], em = za[c] - zm[c];
    dp = fmaf(ep, ep, dp);
    dm = fmaf(em, em, dm);
  }
  const float u = logf(dp + kEps) - logf(dm + kEps);
  const float l = u > 20.0f ? u : log1pf(expf(u));
  const float s = 1.0f / (1.0f + expf(-u)) / (float)B;
  const float gdp = s / (dp + kEps), gdm = -s / (dm + kEps);
  float* ga = dz + (size_t)(3 * t) * kOut;
  float* gp = ga + kOut;
  float* gm = gp + kOut;
#pragma unroll
  for (int c = 0; c < kOut; ++c) {
    const float ep = za[c] - zp[c], em = za[c] - zm[c];
    ga[c] = 2.0f * gdp * ep + 2.0f * gdm * em;
    gp[c] = -2.0f * gdp * ep;
    gm[c] = -2.0f * gdm * em;
  }
  atomicAdd(loss, (double)l / (double)B);
}

// dL/dpre = (dz W2^T) * [pre > 0], in place over `pre`; thread per (row, unit).
__global__ void k_back_hidden(uint32_t nrows, const float* __restrict__ dz,
                              const float* __restrict__ w2, float* __restrict__ pre) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nrows * kHidden) return;
  const uint32_t r = (uint32_t)(i / kHidden), j = (uint32_t)(i % kHidden);
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < kOut; ++c) s = fmaf(dz[(size_t)r * kOut + c], w2[j * kOut + c], s);
  pre[i] = pre[i] > 0.0f ? s : 0.0f;
}

// Gradients of W2 and b2: gw2[j][c] = sum_r relu(pre)[r][j] dz[r][c]. Needs
// the forward pre-activations, so it runs before k_back_hidden overwrites them.
__global__ void k_grad_out(uint32_t nrows, const float* __restrict__ pre,
                           const float* __restrict__ dz, float* __restrict__ gw2,
                           float* __restrict__ gb2) {
  const uint32_t j = blockIdx.x, c = threadIdx.x;  // 128 blocks (+1 for b2) x 32 threads
  float s = 0.0f;
  if (j < kHidden) {
    for (uint32_t r = 0; r < nrows; ++r)
      s = fmaf(fmaxf(pre[(size_t)r * kHidden + j], 0.0f), dz[(size_t)r * kOut + c], s);
    gw2[j * kOut + c] += s;
  } else {
    for (uint32_t r = 0; r < nrows; ++r) s += dz[(size_t)r * kOut + c];
    gb2[c] += s;
  }
}

// Gradients of W1 and b1: gw1[k][j] = sum_r x[r][k] dpre[r][j]. Blocks split
// the input dims (32 per block) and the rows (kSplit parts, added atomically).
constexpr uint32_t kKTile = 32, kRChunk = 32, kSplit = 16;
__global__ void __launch_bounds__(kHidden)
    k_grad_in(const uint32_t* __restrict__ rows, uint32_t nrows, const __half* __restrict__ data,
              uint32_t dim, const float* __restrict__ mean, const float* __restrict__ dpre,
              float* __restrict__ gw1, float* __restrict__ gb1) {
  __shared__ float xs[kRChunk][kKTile];
  const uint32_t j = threadIdx.x, k0 = blockIdx.x * kKTile;
  const uint32_t per = (nrows + kSplit - 1) / kSplit;
  const uint32_t rb = blockIdx.y * per, re = min(nrows, rb + per);
  float acc[kKTile];
#pragma unroll
  for (int k = 0; k < (int)kKTile; ++k) acc[k] = 0.0f;
  float bacc = 0.0f;
  for (uint32_t r0 = rb; r0 < re; r0 += kRChunk) {
    const uint32_t nr = min(kRChunk, re - r0);
    __syncthreads();
    for (uint32_t i = j; i < kRChunk * kKTile; i += kHidden) {
      const uint32_t r = i / kKTile, k = i % kKTile;
      xs[r][k] = (r < nr && k0 + k < dim)
                     ? __half2float(data[(size_t)rows[r0 + r] * dim + k0 + k]) - mean[k0 + k]
                     : 0.0f;
    }
    __syncthreads();
    for (uint32_t r = 0; r < nr; ++r) {
      const float g = dpre[(size_t)(r0 + r) * kHidden + j];
      bacc += g;
#pragma unroll
      for (int k = 0; k < (int)kKTile; ++k) acc[k] = fmaf(xs[r][k], g, acc[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < (int)kKTile; ++k)
    if (k0 + k < dim) atomicAdd(&gw1[(size_t)(k0 + k) * kHidden + j], acc[k]);
  if (blockIdx.x == 0) atomicAdd(&gb1[j], bacc);
}

// Adam step over all parameters (lr, beta1 0.9, beta2 0.999, eps 1e-8);
// clears the gradients.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t count, float lr, float c1, float c2) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = 0.9f * m[i] + 0.1f * gi;
  const float vi = 0.999f * v[i] + 0.001f * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
  g[i] = 0.0f;
}

// Triplets from the kNN rows (packed keys, ascending distance): anchor a,
// a near entry j1 < 8 and a farther entry j2 > j1 of a's row, whose exact
// distances order d(a, p) <= d(a, m). Counter-based, so a batch depends only
// on (seed, step).
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void k_triplets(const uint64_t* __restrict__ nb, uint32_t n, uint32_t K, uint32_t B,
                           uint64_t seed, uint32_t* __restrict__ rows) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B) return;
  uint64_t h = mix64(seed ^ ((uint64_t)t << 20));
  uint32_t a = 0, p = 0, m = 0;
  for (int tries = 0; tries < 8; ++tries) {
    a = (uint32_t)(h % n);
    h = mix64(h);
    const uint32_t near = min(8u, K - 1);
    const uint32_t j1 = (uint32_t)(h % near);
    h = mix64(h);
    const uint32_t j2 = j1 + 1 + (uint32_t)(h % (K - 1 - j1));
    h = mix64(h);
    const uint64_t k1 = nb[(size_t)a * K + j1], k2 = nb[(size_t)a * K + j2];
    if (k1 == knn_empty() || k2 == knn_empty()) continue;
    p = (uint32_t)(k1 >> 1) & 0x7FFFFFFFu;
    m = (uint32_t)(k2 >> 1) & 0x7FFFFFFFu;
    if ((k1 >> 32) < (k2 >> 32)) break;  // strictly ordered pair
    p = m = a;
  }
  rows[3 * t] = a;
  rows[3 * t + 1] = p;
  rows[3 * t + 2] = m;
}

// Projection of all rows with BF16 weights and FP32 accumulation: z (FP16,
// n x 32). One block per 16 rows; thread j owns hidden unit j.
__global__ void __launch_bounds__(kHidden)
    k_project(uint32_t n, const __half* __restrict__ data, uint32_t dim,
              const float* __restrict__ mean, const __nv_bfloat16* __restrict__ w1,
              const float* __restrict__ b1,
              const __nv_bfloat16* __restrict__ w2, const float* __restrict__ b2,
              __half* __restrict__ z) {
  extern __shared__ float xs[];
  float* hs = xs + kRowsPerBlock * dim;
  const uint32_t j = threadIdx.x;
  for (uint32_t r0 = blockIdx.x * kRowsPerBlock; r0 < n; r0 += gridDim.x * kRowsPerBlock) {
    const uint32_t nr = min((uint32_t)kRowsPerBlock, n - r0);
    __syncthreads();
    for (uint32_t i = j; i < nr * dim; i += kHidden)
      xs[i] = __half2float(data[(size_t)r0 * dim + i]) - mean[i % dim];
    __syncthreads();
    float acc[kRowsPerBlock];
#pragma unroll
    for (int r = 0; r < kRowsPerBlock; ++r) acc[r] = b1[j];
    for (uint32_t k = 0; k < dim; ++k) {
      const float w = __bfloat162float(w1[(size_t)k * kHidden + j]);
#pragma unroll
      for (int r = 0; r < kRowsPerBlock; ++r) acc[r] = fmaf(xs[r * dim + k], w, acc[r]);
    }
#pragma unroll
    for (int r = 0; r < kRowsPerBlock; ++r) hs[r * kHidden + j] = fmaxf(acc[r], 0.0f);
    __syncthreads();
    for (uint32_t o = j; o < nr * kOut; o += kHidden) {
      const uint32_t r = o / kOut, c = o % kOut;
      float s = b2[c];
      for (uint32_t h = 0; h < kHidden; ++h)
        s = fmaf(hs[r * kHidden + h], __bfloat162float(w2[h * kOut + c]), s);
      z[(size_t)(r0 + r) * kOut + c] = __float2half_rn(s);
    }
  }
}

// Mean of every input dim over `rows` evenly spaced base rows (the inputs are
// centred with it); thread per dim.
__global__ void k_col_mean(const __half* __restrict__ data, uint32_t n, uint32_t dim,
                           uint32_t rows, float* __restrict__ mean) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= dim) return;
  const uint64_t stride = n / rows;
  float s = 0.0f;
  for (uint32_t i = 0; i < rows; ++i) s += __half2float(data[(size_t)(i * stride) * dim + k]);
  mean[k] = s / (float)rows;
}

__global__ void k_to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst,
                          size_t count) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < count) dst[i] = __float2bfloat16_rn(src[i]);
}

// Deterministic N(0, 1) samples (splitmix64 + Box-Muller) for the start weights.
double host_normal(uint64_t& s) {
  auto u01 = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t x = s;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  const double a = u01(), b = u01();
  return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
}

}  // namespace

size_t Net::count(uint32_t dim) { return (size_t)dim * kHidden + kHidden + kHidden * kOut + kOut; }

int Net::init(uint32_t d, uint64_t seed, cudaStream_t s) {
  release(stream);
  dim = d;
  stream = s;
  const size_t c = count(d);
  TG_TRY(pool_alloc((void**)&buf, c * 4 * sizeof(float) + d * sizeof(float) +
                                      c * sizeof(__nv_bfloat16) + 256,
                     s));
  params = buf;
  grads = buf + c;
  mom = buf + 2 * c;
  vel = buf + 3 * c;
  mean = buf + 4 * c;
  half_w = reinterpret_cast<__nv_bfloat16*>(mean + d);
  std::vector<float> h(c, 0.0f);
  uint64_t st = seed;
  const double s1 = std::sqrt(2.0 / d), s2 = std::sqrt(1.0 / kHidden);
  for (size_t i = 0; i < (size_t)d * kHidden; ++i) h[i] = (float)(s1 * host_normal(st));
  float* w2 = h.data() + (size_t)d * kHidden + kHidden;
  for (size_t i = 0; i < (size_t)kHidden * kOut; ++i) w2[i] = (float)(s2 * host_normal(st));
  TG_CUDA(cudaMemcpyAsync(params, h.data(), c * 4, cudaMemcpyHostToDevice, s));
  TG_CUDA(cudaMemsetAsync(grads, 0, c * 3 * sizeof(float), s));
  TG_CUDA(cudaMemsetAsync(mean, 0, d * sizeof(float), s));
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

int Net::center(const __half* data, uint32_t n, cudaStream_t s) {
  const uint32_t rows = std::min<uint32_t>(n, 8192);
  k_col_mean<<<(dim + 127) / 128, 128, 0, s>>>(data, n, dim, rows, mean);
  count_launch();
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

void Net::release(cudaStream_t s) {
  if (buf) pool_free(buf, s);
  buf = nullptr;
}

int Net::set_params(const float* host, cudaStream_t s) {
  TG_CUDA(cudaMemcpyAsync(params, host, count(dim) * 4, cudaMemcpyHostToDevice, s));
  return TAGORE_OK;
}

int Net::get(float* host_params, float* host_grads, cudaStream_t s) const {
  if (host_params)
    TG_CUDA(cudaMemcpyAsync(host_params, params, count(dim) * 4, cudaMemcpyDeviceToHost, s));
  if (host_grads)
    TG_CUDA(cudaMemcpyAsync(host_grads, grads, count(dim) * 4, cudaMemcpyDeviceToHost, s));
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

// Forward, loss and backward of one batch; gradients are added to `grads`.
int Net::loss_grad(const uint32_t* rows_dev, uint32_t B, const __half* data, Scratch& work,
                   double* loss_host, cudaStream_t s) {
  const uint32_t nrows = 3 * B;
  const size_t need = (size_t)nrows * (kHidden + 2 * kOut) * 4 + 64;
  if (!work.p) TG_TRY(work.alloc(need));
  float* pre = work.as<float>();
  float* z = pre + (size_t)nrows * kHidden;
  float* dz = z + (size_t)nrows * kOut;
  double* loss = reinterpret_cast<double*>(dz + (size_t)nrows * kOut);
  const float* w1 = params;
  const float* b1 = w1 + (size_t)dim * kHidden;
  const float* w2 = b1 + kHidden;
  const float* b2 = w2 + kHidden * kOut;
  float* gw1 = grads;
  float* gb1 = gw1 + (size_t)dim * kHidden;
  float* gw2 = gb1 + kHidden;
  float* gb2 = gw2 + kHidden * kOut;
  const size_t fsm = ((size_t)kRowsPerBlock * dim + kRowsPerBlock * kHidden) * 4;
  if (fsm > 227 * 1024) return fail(TAGORE_EINVAL, "screen MLP: DIM %u too large", dim);
  TG_CUDA(cudaFuncSetAttribute((const void*)k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fsm));
  TG_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), s));
  k_forward<<<(nrows + kRowsPerBlock - 1) / kRowsPerBlock, kHidden, fsm, s>>>(
      rows_dev, nrows, data, dim, mean, w1, b1, w2, b2, pre, z);
  k_loss<<<(B + 127) / 128, 128, 0, s>>>(B, z, dz, loss);
  k_grad_out<<<kHidden + 1, kOut, 0, s>>>(nrows, pre, dz, gw2, gb2);
  k_back_hidden<<<(unsigned)(((size_t)nrows * kHidden + 255) / 256), 256, 0, s>>>(nrows, dz, w2,
                                                                                  pre);
  k_grad_in<<<dim3((dim + kKTile - 1) / kKTile, kSplit), kHidden, 0, s>>>(
      rows_dev, nrows, data, dim, mean, pre, gw1, gb1);
  count_launch(5);
  TG_CUDA(cudaGetLastError());
  if (loss_host) {
    TG_CUDA(cudaMemcpyAsync(loss_host, loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    TG_CUDA(cudaStreamSynchronize(s));
  }
  return TAGORE_OK;
}

int Net::adam(float lr, uint32_t t, cudaStream_t s) {
  const size_t c = count(dim);
  const float c1 = 1.0f - std::pow(0.9f, (float)t), c2 = 1.0f - std::pow(0.999f, (float)t);
  k_adam<<<(unsigned)((c + 255) / 256), 256, 0, s>>>(params, grads, mom, vel, c, lr, c1, c2);
  count_launch();
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

int Net::train(const uint64_t* nb, uint32_t n, uint32_t K, const __half* data, uint32_t steps,
               uint32_t batch, uint64_t seed, float* loss_first, float* loss_last,
               cudaStream_t s) {
  Scratch rows(s), work(s);
  TG_TRY(rows.alloc((size_t)batch * 3 * 4));
  double l = 0.0;
  for (uint32_t t = 0; t < steps; ++t) {
    k_triplets<<<(batch + 127) / 128, 128, 0, s>>>(nb, n, K, batch, seed + 0x1000193ull * t,
                                                   rows.as<uint32_t>());
    count_launch();
    const bool probe = t == 0 || t + 1 == steps;
    TG_TRY(loss_grad(rows.as<uint32_t>(), batch, data, work, probe ? &l : nullptr, s));
    if (t == 0 && loss_first) *loss_first = (float)l;
    if (t + 1 == steps && loss_last) *loss_last = (float)l;
    TG_TRY(adam(2e-3f, t + 1, s));
  }
  return TAGORE_OK;
}

int Net::project(const __half* data, uint32_t n, __half* z, cudaStream_t s) {
  const size_t c = count(dim);
  k_to_bf16<<<(unsigned)((c + 255) / 256), 256, 0, s>>>(params, half_w, c);
  const __nv_bfloat16* w1 = half_w;
  const float* b1 = params + (size_t)dim * kHidden;
  const __nv_bfloat16* w2 = half_w + (size_t)dim * kHidden + kHidden;
  const float* b2 = params + (size_t)dim * kHidden + kHidden + kHidden * kOut;
  const size_t sm = ((size_t)kRowsPerBlock * dim + kRowsPerBlock * kHidden) * 4;
  if (sm > 227 * 1024) return fail(TAGORE_EINVAL, "screen MLP: DIM %u too large", dim);
  TG_CUDA(cudaFuncSetAttribute((const void*)k_project, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sm));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t blocks = std::min<uint32_t>((n + kRowsPerBlock - 1) / kRowsPerBlock, sms * 16);
  k_project<<<blocks, kHidden, sm, s>>>(n, data, dim, mean, w1, b1, w2, b2, z);
  count_launch(2);
  TG_CUDA(cudaGetLastError());
  return TAGORE_OK;
}

}  // namespace mlp
}  // namespace tagore
