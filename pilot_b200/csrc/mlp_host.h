// mlp_host.h — host-side declarations shared by the learned form's files.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "beams_params.h"
#include "mlp_common.cuh"

namespace beams {

// Activations and gradient scratch of one training batch.
struct TrainWS {
  __nv_bfloat16* H[4];  // rows x 64, the four hidden layers
  float* dA;            // rows x 112 gradient scratch
  float* dB;            // rows x 64 gradient scratch
  float* dz;            // rows
  float* T;             // rows
  float* loss;          // 1
  unsigned* err;        // tensor-core wait timeouts; null: the forward runs on the CUDA cores
};

cudaError_t mlp_gen_data(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                         const float4* lights, int nlights, unsigned seed, float focus, float4* samples,
                         float* target, int n, cudaStream_t st);
cudaError_t mlp_features(const float4* samples, const float4* lfeat, const mlp::Encoding& enc, __nv_bfloat16* X,
                         int n, cudaStream_t st);
cudaError_t mlp_fwd_bwd(const float* P, float* G, const __nv_bfloat16* X, const float* target, int n,
                        const TrainWS& w, cudaStream_t st);
// Forward pass on the tcgen05 tensor cores (k_mlp_tc.cu) of n rows of
// features (16-byte aligned): T per row.
cudaError_t mlp_forward_tc_features(const __nv_bfloat16* X, int n, const float* P, float* T, unsigned* err,
                                    cudaStream_t st);
// One training step on the tcgen05 tensor cores (k_mlp_tc.cu): forward, loss
// (sum of squared errors added to *loss when target is given), and with G
// non-null the backward, adding scale-weighted gradients to G; T per row when
// non-null.
cudaError_t mlp_train_step_tc(const float* P, float* G, const __nv_bfloat16* X, const float* target, int n,
                              float scale, float* T, float* loss, unsigned* err, cudaStream_t st);
cudaError_t mlp_adam(float* P, float* G, float* m, float* v, float lr, int t, cudaStream_t st);

}  // namespace beams
