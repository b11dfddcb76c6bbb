// mlp.cuh -- the learned candidate screen (mlp.cu): a d -> 128 -> 32 MLP
// trained on the GPU and used to screen local-join pairs before their exact
// distance is computed.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "internal.h"

namespace tagore {
namespace mlp {

constexpr int kHidden = 128;
constexpr int kOut = 32;
constexpr float kEps = 1e-6f;  // added to projected squared distances in the loss
__host__ __device__ constexpr uint64_t knn_empty() { return ~0ull; }  // an empty kNN slot

// Parameters, gradients and Adam moments in one device block, FP32, each laid
// out [W1 (d x 128, row k = input dim) | b1 | W2 (128 x 32) | b2]; BF16 copies
// of the weights for the projection.
struct Net {
  uint32_t dim = 0;
  cudaStream_t stream = nullptr;  // stream the parameter block was allocated on
  float* buf = nullptr;
  float *params = nullptr, *grads = nullptr, *mom = nullptr, *vel = nullptr;
  float* mean = nullptr;  // input centre (dim), subtracted before the first layer
  __nv_bfloat16* half_w = nullptr;

  static size_t count(uint32_t dim);
  // He-scaled normal start weights from `seed` (deterministic), zero biases.
  int init(uint32_t dim, uint64_t seed, cudaStream_t s);
  void release(cudaStream_t s);
  ~Net() { release(stream); }
  int set_params(const float* host, cudaStream_t s);
  // Centres the inputs: the mean of 8192 evenly spaced base rows.
  int center(const __half* data, uint32_t n, cudaStream_t s);
  int get(float* host_params, float* host_grads, cudaStream_t s) const;
  // Forward + loss + backward of B triplets (rows_dev: 3B base-row ids, a p m
  // per triplet); gradients are added to `grads`. `work` holds the
  // activations (allocated on first use).
  int loss_grad(const uint32_t* rows_dev, uint32_t B, const __half* data, Scratch& work,
                double* loss_host, cudaStream_t s);
  int adam(float lr, uint32_t t, cudaStream_t s);
  // `steps` Adam steps on batches of `batch` triplets drawn from the kNN rows.
  int train(const uint64_t* nb, uint32_t n, uint32_t K, const __half* data, uint32_t steps,
            uint32_t batch, uint64_t seed, float* loss_first, float* loss_last, cudaStream_t s);
  // z[n x 32] (FP16) of every base row, with BF16 weights.
  int project(const __half* data, uint32_t n, __half* z, cudaStream_t s);
};

}  // namespace mlp
}  // namespace tagore
