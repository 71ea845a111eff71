// kernels.h — launch wrappers shared between the kernel files and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "beams_params.h"

namespace beams {

cudaError_t launch_light_march_f32(const ExactGeo& g, const float* field, const float4* tf,
                                   float* map, Counters* cnt, cudaStream_t st);
cudaError_t launch_view_march_f32(const ExactGeo& g, const float* field, const float4* tf,
                                  const float* map, float4* out, Counters* cnt, cudaStream_t st);

cudaError_t launch_generate_blobs(float* out, const int n[3], const float* d_params, int nblobs,
                                  cudaStream_t st);
cudaError_t launch_generate_noise(float* out, const int n[3], const unsigned char* d_perm, int octaves,
                                  float base_freq, float lacunarity, float gain, cudaStream_t st);
cudaError_t launch_normalise01(float* data, int64_t count, unsigned* d_minmax, cudaStream_t st);

}  // namespace beams
