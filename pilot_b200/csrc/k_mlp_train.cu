// k_mlp_train.cu — the learned form's training: data from the exact light
// march, bfloat16-weight / float32-accumulate forward and backward passes, Adam.
//
// Data: 2^k samples (position uniform in the volume, one of L lights on a
// Fibonacci sphere at 2x the diagonal from the centre) labelled with the exact
// light march's transmittance 1 - o at that position (the march of
// TransmittanceMap.h:279-332 run to an arbitrary point instead of a vertex).
// Training: minibatch MSE on T with Adam on float32 master weights; forward
// products use bfloat16-rounded weights and activations, as inference does.
// Compiled with -fmad=false like every kernel file (the exact march needs it).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "exact_device.cuh"
#include "kernels.h"
#include "mlp_common.cuh"
#include "mlp_host.h"

namespace beams {
namespace mlp {

__device__ __forceinline__ unsigned hash32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float uniform01(unsigned seed, unsigned i, unsigned k) {
  return (float)(hash32(seed ^ hash32(hash32(i) + k * 0x9e3779b9u)) >> 8) * (1.f / 16777216.f);
}

// ---- data: exact transmittance at random points ---------------------------------
// Normalised colour-map alpha of the field at P (one light-march sample).
__device__ float alpha_at(const ExactGeo& g, const float4* __restrict__ quads, const float4* T0, const float4* T1,
                          const float4* T2, const float* s_a, const float P[3]) {
  const unsigned qx = (unsigned)(g.n[0] - 1), qz = (unsigned)(g.n[0] - 1) * (unsigned)(g.n[1] - 1);
  float4 e0, e1, e2;
  const int c0 = find_cell_bsearch_t(T0, g.n[0] - 2, g.org[0], g.invh[0], P[0], e0);
  const int c1 = find_cell_bsearch_t(T1, g.n[1] - 2, g.org[1], g.invh[1], P[1], e1);
  const int c2 = find_cell_bsearch_t(T2, g.n[2] - 2, g.org[2], g.invh[2], P[2], e2);
  float vals[8];
  QuadLoad<float4>::cell(quads, (unsigned)c2 * qz + (unsigned)c1 * qx + (unsigned)c0, qx, qz, vals);
  float scalar = hex_interp(vals, div_rn_markstein(P[0] - e0.x, e0.z, e0.w), div_rn_markstein(P[1] - e1.x, e1.z, e1.w),
                            div_rn_markstein(P[2] - e2.x, e2.z, e2.w));
  scalar = (scalar - g.min_scalar) * g.inv_delta;
  const int n1 = g.tf_n - 1;
  return s_a[tf_index_clamped(scalar * (float)n1, n1)];
}

// sample i: position (world) in xyz, light index in w; target transmittance.
// A fraction `focus` of the positions is rejection-sampled (16 tries) where the
// colour map's alpha is non-zero: the shading only reads T where samples
// composite, so the network's capacity goes there.
__global__ void __launch_bounds__(256) k_gen_data(const ExactGeo g, const float4* __restrict__ quads,
                                                  const float4* __restrict__ tab, const float4* __restrict__ tf,
                                                  const float4* __restrict__ lights, int nlights, unsigned seed,
                                                  float focus, float4* __restrict__ samples,
                                                  float* __restrict__ target, int n) {
  extern __shared__ float4 s_dyn[];
  float4* s_tab = s_dyn;
  float* s_a = (float*)(s_dyn + g.max_off[0]);
  for (int i = threadIdx.x; i < g.max_off[0]; i += blockDim.x) s_tab[i] = tab[i];
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_a[i] = (g.max_alpha > 0.f) ? tf[i].w / g.max_alpha : 0.f;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int li = (int)(hash32(seed + 7919u * (unsigned)i) % (unsigned)nlights);
    float P[3];
    const int tries = (uniform01(seed, (unsigned)i, 3u) < focus) ? 16 : 1;
    for (int t = 0; t < tries; ++t) {
      const unsigned k = 4u + 3u * (unsigned)t;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        P[a] = g.minp[a] + uniform01(seed, (unsigned)i, k + (unsigned)a) * (g.maxp[a] - g.minp[a]);
      if (tries == 1 || alpha_at(g, quads, s_tab + g.ax_off[0], s_tab + g.ax_off[1], s_tab + g.ax_off[2], s_a, P) > 0.f)
        break;
    }
    const float4 Lw = lights[li];
    const float L[3] = {Lw.x, Lw.y, Lw.z};
    const float o = point_opacity(g, quads, s_tab + g.ax_off[0], s_tab + g.ax_off[1], s_tab + g.ax_off[2], s_a,
                                  L, P);
    samples[i] = make_float4(P[0], P[1], P[2], (float)li);
    target[i] = 1.f - o;
  }
}

// ---- encoding --------------------------------------------------------------------
__global__ void k_features(const float4* __restrict__ samples, const float4* __restrict__ lfeat, Encoding enc,
                           __nv_bfloat16* __restrict__ X, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 s = samples[i];
    const float4 lf = lfeat[(int)s.w];
    const float p[3] = {s.x, s.y, s.z}, l[3] = {lf.x, lf.y, lf.z};
    __nv_bfloat16* row = X + (size_t)i * kIn;
    encode(enc, p, l, [&](int j, float v) { row[j] = __float2bfloat16_rn(v); });
  }
}

// ---- dense layers (CUDA cores, float32 accumulation) -------------------------------
// Y[b][n] = bf16(relu(b[n] + sum_k X[b][k] * bf16(W[k][n]))), 32 rows per block.
__global__ void __launch_bounds__(256) k_linear_fwd(const __nv_bfloat16* __restrict__ X, const float* __restrict__ W,
                                                    const float* __restrict__ bias, __nv_bfloat16* __restrict__ Y,
                                                    int n, int K) {
  __shared__ float sW[kIn * kHid];
  __shared__ float sX[32 * (kIn + 1)];
  for (int i = threadIdx.x; i < K * kHid; i += blockDim.x) sW[i] = bf16r(W[i]);
  const int r0 = blockIdx.x * 32;
  for (int i = threadIdx.x; i < 32 * K; i += blockDim.x) {
    const int r = i / K, k = i - r * K;
    sX[r * (kIn + 1) + k] = (r0 + r < n) ? __bfloat162float(X[(size_t)(r0 + r) * K + k]) : 0.f;
  }
  __syncthreads();
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;  // 2 rows x 4 cols per thread
  float acc[2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int k = 0; k < K; ++k) {
    float xv[2], wv[4];
#pragma unroll
    for (int i = 0; i < 2; ++i) xv[i] = sX[(tr * 2 + i) * (kIn + 1) + k];
#pragma unroll
    for (int j = 0; j < 4; ++j) wv[j] = sW[k * kHid + tc * 4 + j];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(xv[i], wv[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int r = r0 + tr * 2 + i;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = tc * 4 + j;
      const float v = acc[i][j] + bias[c];
      Y[(size_t)r * kHid + c] = __float2bfloat16_rn(v > 0.f ? v : 0.f);
    }
  }
}

// Head, loss and the first backward step: z = b5 + h4 . bf16(w5), T = sigmoid(z);
// loss += (T - t)^2; dz = scale * 2 (T - t) T (1 - T);
// dH4[b][k] = dz * bf16(w5[k]) * (h4[b][k] > 0).
__global__ void k_head(const __nv_bfloat16* __restrict__ H4, const float* __restrict__ P,
                       const float* __restrict__ target, float* __restrict__ Tout, float* __restrict__ dH4,
                       float* __restrict__ dz_out, float* __restrict__ loss, int n, float scale) {
  float lsum = 0.f;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    const __nv_bfloat16* h = H4 + (size_t)b * kHid;
    float z = P[oB5];
    for (int k = 0; k < kHid; ++k) z = fmaf(__bfloat162float(h[k]), bf16r(P[oW5 + k]), z);
    const float T = 1.f / (1.f + expf(-z));
    if (Tout) Tout[b] = T;
    if (target) {
      const float d = T - target[b];
      lsum += d * d;
      const float dz = scale * 2.f * d * T * (1.f - T);
      if (dz_out) dz_out[b] = dz;
      if (dH4)
        for (int k = 0; k < kHid; ++k)
          dH4[(size_t)b * kHid + k] = (__bfloat162float(h[k]) > 0.f) ? dz * bf16r(P[oW5 + k]) : 0.f;
    }
  }
  if (loss) {
    lsum += __shfl_xor_sync(0xffffffffu, lsum, 16);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, 8);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, 4);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, 2);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, 1);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum);
  }
}

// dX[b][k] = (sum_n dY[b][n] * bf16(W[k][n])) * (X[b][k] > 0), 64 rows per block.
__global__ void __launch_bounds__(256) k_linear_dgrad(const float* __restrict__ dY, const float* __restrict__ W,
                                                      const __nv_bfloat16* __restrict__ X, float* __restrict__ dX,
                                                      int n, int K) {
  __shared__ float sW[kIn * kHid];
  __shared__ float sD[64 * (kHid + 1)];
  for (int i = threadIdx.x; i < K * kHid; i += blockDim.x) sW[i] = bf16r(W[i]);
  const int r0 = blockIdx.x * 64;
  for (int i = threadIdx.x; i < 64 * kHid; i += blockDim.x) {
    const int r = i / kHid, c = i - r * kHid;
    sD[r * (kHid + 1) + c] = (r0 + r < n) ? dY[(size_t)(r0 + r) * kHid + c] : 0.f;
  }
  __syncthreads();
  for (int o = threadIdx.x; o < 64 * K; o += blockDim.x) {
    const int r = o / K, k = o - r * K;
    if (r0 + r >= n) continue;
    float acc = 0.f;
    for (int c = 0; c < kHid; ++c) acc = fmaf(sD[r * (kHid + 1) + c], sW[k * kHid + c], acc);
    const float xv = __bfloat162float(X[(size_t)(r0 + r) * K + k]);
    dX[(size_t)(r0 + r) * K + k] = xv > 0.f ? acc : 0.f;
  }
}

// G_W[k][n] += sum_b X[b][k] dY[b][n]; G_b[n] += sum_b dY[b][n]; 256 rows per block.
__global__ void __launch_bounds__(256) k_linear_wgrad(const __nv_bfloat16* __restrict__ X, const float* __restrict__ dY,
                                                      float* __restrict__ GW, float* __restrict__ Gb, int n, int K) {
  __shared__ float sX[32 * kIn];
  __shared__ float sD[32 * kHid];
  const int b0 = blockIdx.x * 256;
  const int nout = K * kHid;
  float acc[28];  // K*64/256 <= 28 outputs per thread
  float bacc = 0.f;
#pragma unroll
  for (int j = 0; j < 28; ++j) acc[j] = 0.f;
  for (int c0 = 0; c0 < 256; c0 += 32) {
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * K; i += blockDim.x) {
      const int r = i / K, k = i - r * K;
      const int b = b0 + c0 + r;
      sX[r * kIn + k] = (b < n) ? __bfloat162float(X[(size_t)b * K + k]) : 0.f;
    }
    for (int i = threadIdx.x; i < 32 * kHid; i += blockDim.x) {
      const int r = i / kHid, c = i - r * kHid;
      const int b = b0 + c0 + r;
      sD[i] = (b < n) ? dY[(size_t)b * kHid + c] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 28; ++j) {
      const int o = threadIdx.x + j * 256;
      if (o >= nout) break;
      const int k = o / kHid, c = o - k * kHid;
      float a = acc[j];
      for (int r = 0; r < 32; ++r) a = fmaf(sX[r * kIn + k], sD[r * kHid + c], a);
      acc[j] = a;
    }
    if (threadIdx.x < kHid)
      for (int r = 0; r < 32; ++r) bacc += sD[r * kHid + threadIdx.x];
  }
#pragma unroll
  for (int j = 0; j < 28; ++j) {
    const int o = threadIdx.x + j * 256;
    if (o >= nout) break;
    atomicAdd(GW + o, acc[j]);
  }
  if (threadIdx.x < kHid) atomicAdd(Gb + threadIdx.x, bacc);
}

// Head gradients: G_w5[k] += sum_b dz[b] h4[b][k]; G_b5 += sum_b dz[b].
__global__ void k_head_wgrad(const __nv_bfloat16* __restrict__ H4, const float* __restrict__ dz,
                             float* __restrict__ G, int n) {
  const int k = threadIdx.x;  // 64 threads
  float a = 0.f, bz = 0.f;
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const float d = dz[b];
    a = fmaf(d, __bfloat162float(H4[(size_t)b * kHid + k]), a);
    bz += d;
  }
  atomicAdd(G + oW5 + k, a);
  if (k == 0) atomicAdd(G + oB5, bz);
}

__global__ void k_adam(float* __restrict__ P, float* __restrict__ G, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = G[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    G[i] = 0.f;
  }
}

}  // namespace mlp

// ---------------------------------------------------------------------------
// host side: the training driver
// ---------------------------------------------------------------------------
using namespace mlp;

static unsigned grid_cap(size_t n, int per) {
  size_t b = (n + per - 1) / per;
  return (unsigned)(b < 65535 * 8 ? (b ? b : 1) : 65535 * 8);
}

cudaError_t mlp_gen_data(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                         const float4* lights, int nlights, unsigned seed, float focus, float4* samples,
                         float* target, int n, cudaStream_t st) {
  const size_t smem = (size_t)g.max_off[0] * sizeof(float4) + (size_t)g.tf_n * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_gen_data, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_gen_data<<<148 * 8, 256, smem, st>>>(g, quads, tab, tf, lights, nlights, seed, focus, samples, target, n);
  return cudaGetLastError();
}

cudaError_t mlp_features(const float4* samples, const float4* lfeat, const Encoding& enc, __nv_bfloat16* X, int n,
                         cudaStream_t st) {
  k_features<<<grid_cap(n, 256), 256, 0, st>>>(samples, lfeat, enc, X, n);
  return cudaGetLastError();
}

// Forward (and, with G != null, backward) of n rows X (n x 112 bf16): on the
// tensor cores when w.err is set, else on the CUDA cores (the reference path).
cudaError_t mlp_fwd_bwd(const float* P, float* G, const __nv_bfloat16* X, const float* target, int n,
                        const TrainWS& w, cudaStream_t st) {
  const unsigned rf = (unsigned)((n + 31) / 32);
  const unsigned rb = (unsigned)((n + 63) / 64);
  const int Ks[4] = {kIn, kHid, kHid, kHid};
  const int oW[4] = {oW1, oW2, oW3, oW4}, oB[4] = {oB1, oB2, oB3, oB4};
  if (w.err) {
    // forward, loss and backward fused on the tcgen05 tensor cores (k_mlp_tc.cu)
    return mlp_train_step_tc(P, G, X, target, n, 1.f / (float)n, w.T, w.loss, w.err, st);
  }
  {
    const __nv_bfloat16* in = X;
    for (int l = 0; l < 4; ++l) {
      k_linear_fwd<<<rf, 256, 0, st>>>(in, P + oW[l], P + oB[l], w.H[l], n, Ks[l]);
      in = w.H[l];
    }
  }
  k_head<<<grid_cap(n, 256), 256, 0, st>>>(w.H[3], P, target, w.T, G ? w.dB : nullptr, G ? w.dz : nullptr, w.loss, n,
                                           1.f / (float)n);
  if (!G) return cudaGetLastError();
  k_head_wgrad<<<256, 64, 0, st>>>(w.H[3], w.dz, G, n);
  // dB holds dH4; walk the layers down
  float* cur = w.dB;
  for (int l = 3; l >= 0; --l) {
    const __nv_bfloat16* Xl = (l == 0) ? X : w.H[l - 1];
    k_linear_wgrad<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(Xl, cur, G + oW[l], G + oB[l], n, Ks[l]);
    if (l > 0) {
      // dH_{l-1} into the other scratch (n x 64), alternating dA/dB
      float* nxt = (cur == w.dB) ? w.dA : w.dB;
      k_linear_dgrad<<<rb, 256, 0, st>>>(cur, P + oW[l], Xl, nxt, n, kHid);
      cur = nxt;
    }
  }
  return cudaGetLastError();
}

cudaError_t mlp_adam(float* P, float* G, float* m, float* v, float lr, int t, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.99f;
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  k_adam<<<grid_cap(kParams, 256), 256, 0, st>>>(P, G, m, v, kParams, lr, b1, b2, 1e-8f, c1, c2);
  return cudaGetLastError();
}

}  // namespace beams
