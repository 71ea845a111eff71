// k_scene.cu — synthetic scalar fields on the device (inputs for tests and
// benchmarks; not part of the render path).
//
//  * blobs: sum of isotropic Gaussians amp * exp(-|p-c|^2 / (2 sigma^2)) over the
//    unit cube, p = (i/(nx-1), j/(ny-1), k/(nz-1)).
//  * noise: gradient noise after Perlin's "Improving Noise" (SIGGRAPH 2002):
//    quintic fade, 12 edge gradients picked by the low 4 hash bits, a 256-entry
//    permutation table; octaves summed as fBm (frequency *= lacunarity,
//    amplitude *= gain).
// Both can be remapped to [0,1] by the field's min and max.
#include <cuda_runtime.h>

#include "kernels.h"

namespace beams {

__global__ void k_blobs(float* __restrict__ out, int nx, int ny, int nz, const float* __restrict__ prm,
                        int nb) {
  const int64_t total = (int64_t)nx * ny * nz;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total;
       id += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = id / ((int64_t)nx * ny);
    const int64_t r = id - k * (int64_t)nx * ny;
    const int j = (int)(r / nx), i = (int)(r - (int64_t)j * nx);
    const float x = (float)i / (float)(nx - 1);
    const float y = (float)j / (float)(ny - 1);
    const float z = (float)k / (float)(nz - 1);
    float v = 0.f;
    for (int b = 0; b < nb; ++b) {
      const float* q = prm + 5 * b;
      const float dx = x - q[0], dy = y - q[1], dz = z - q[2];
      const float r2 = dx * dx + dy * dy + dz * dz;
      v += q[4] * expf(-r2 / (2.f * q[3] * q[3]));
    }
    out[id] = v;
  }
}

__device__ __forceinline__ float fade(float t) { return t * t * t * (t * (t * 6.f - 15.f) + 10.f); }
__device__ __forceinline__ float lerpf(float t, float a, float b) { return a + t * (b - a); }
__device__ __forceinline__ float grad(int h, float x, float y, float z) {
  h &= 15;
  const float u = h < 8 ? x : y;
  const float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
  return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}

__device__ float perlin(const unsigned char* P, float x, float y, float z) {
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
  x -= fx;
  y -= fy;
  z -= fz;
  const float u = fade(x), v = fade(y), w = fade(z);
  const int A = P[X] + Y, AA = P[A & 255] + Z, AB = P[(A + 1) & 255] + Z;
  const int B = P[(X + 1) & 255] + Y, BA = P[B & 255] + Z, BB = P[(B + 1) & 255] + Z;
  return lerpf(w,
               lerpf(v, lerpf(u, grad(P[AA & 255], x, y, z), grad(P[BA & 255], x - 1, y, z)),
                     lerpf(u, grad(P[AB & 255], x, y - 1, z), grad(P[BB & 255], x - 1, y - 1, z))),
               lerpf(v, lerpf(u, grad(P[(AA + 1) & 255], x, y, z - 1), grad(P[(BA + 1) & 255], x - 1, y, z - 1)),
                     lerpf(u, grad(P[(AB + 1) & 255], x, y - 1, z - 1),
                           grad(P[(BB + 1) & 255], x - 1, y - 1, z - 1))));
}

__global__ void k_noise(float* __restrict__ out, int nx, int ny, int nz, const unsigned char* __restrict__ perm,
                        int octaves, float f0, float lac, float gain) {
  __shared__ unsigned char P[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) P[i] = perm[i];
  __syncthreads();
  const int64_t total = (int64_t)nx * ny * nz;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total;
       id += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = id / ((int64_t)nx * ny);
    const int64_t r = id - k * (int64_t)nx * ny;
    const int j = (int)(r / nx), i = (int)(r - (int64_t)j * nx);
    const float x = (float)i / (float)(nx - 1);
    const float y = (float)j / (float)(ny - 1);
    const float z = (float)k / (float)(nz - 1);
    float f = f0, a = 1.f, v = 0.f;
    for (int o = 0; o < octaves; ++o) {
      v += a * perlin(P, x * f, y * f, z * f);
      f *= lac;
      a *= gain;
    }
    out[id] = v;
  }
}

__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fdecode(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void k_minmax(const float* __restrict__ d, int64_t n, unsigned* mm) {
  unsigned lo = 0xffffffffu, hi = 0u;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned k = fkey(d[i]);
    lo = min(lo, k);
    hi = max(hi, k);
  }
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}

__global__ void k_rescale(float* __restrict__ d, int64_t n, const unsigned* mm) {
  const float lo = fdecode(mm[0]), hi = fdecode(mm[1]);
  const float inv = (hi > lo) ? 1.f / (hi - lo) : 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float v = (d[i] - lo) * inv;
    d[i] = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
  }
}

static unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = 148 * 32;
  return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

cudaError_t launch_generate_blobs(float* out, const int n[3], const float* d_params, int nblobs,
                                  cudaStream_t st) {
  const int64_t total = (int64_t)n[0] * n[1] * n[2];
  k_blobs<<<grid_for(total), 256, 0, st>>>(out, n[0], n[1], n[2], d_params, nblobs);
  return cudaGetLastError();
}

cudaError_t launch_generate_noise(float* out, const int n[3], const unsigned char* d_perm, int octaves,
                                  float base_freq, float lacunarity, float gain, cudaStream_t st) {
  const int64_t total = (int64_t)n[0] * n[1] * n[2];
  k_noise<<<grid_for(total), 256, 0, st>>>(out, n[0], n[1], n[2], d_perm, octaves, base_freq, lacunarity,
                                           gain);
  return cudaGetLastError();
}

cudaError_t launch_normalise01(float* data, int64_t count, unsigned* d_minmax, cudaStream_t st) {
  const unsigned init[2] = {0xffffffffu, 0u};
  cudaError_t e = cudaMemcpyAsync(d_minmax, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  k_minmax<<<grid_for(count), 256, 0, st>>>(data, count, d_minmax);
  k_rescale<<<grid_for(count), 256, 0, st>>>(data, count, d_minmax);
  return cudaGetLastError();
}

}  // namespace beams
