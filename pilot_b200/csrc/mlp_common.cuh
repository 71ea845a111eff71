// mlp_common.cuh — the transmittance network shared by training and inference.
//
// T(p, light) = sigmoid(w5 . h4 + b5), h_l = relu(W_l h_{l-1} + b_l) for four
// hidden layers of width 64, and h0 = the 112-wide input encoding:
//   [0..2]    u*2 - 1, u = (p - bounds.min) / extent (position in the volume)
//   [3..5]    the light's direction from the volume centre (unit vector)
//   [6..101]  sin(pi f_k u_a), cos(pi f_k u_a), axis a = 0..2, k = 0..15,
//             f_k = 2^(7k/15) (1 to 128 half-cycles over the volume)
//   [102..111] zero padding (the tensor-core K step is 16)
// Weights and activations are rounded to bfloat16 where they enter a product;
// products accumulate in float32. Parameters are stored as float32 masters in
// one flat vector with the offsets below (W_l row-major [in][out]).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace beams {
namespace mlp {

constexpr int kIn = 112;
constexpr int kUsed = 102;
constexpr int kHid = 64;
constexpr int kFreq = 16;
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + kIn * kHid;
constexpr int oW2 = oB1 + kHid;
constexpr int oB2 = oW2 + kHid * kHid;
constexpr int oW3 = oB2 + kHid;
constexpr int oB3 = oW3 + kHid * kHid;
constexpr int oW4 = oB3 + kHid;
constexpr int oB4 = oW4 + kHid * kHid;
constexpr int oW5 = oB4 + kHid;
constexpr int oB5 = oW5 + kHid;
constexpr int kParams = oB5 + 1;
constexpr int kMaxLights = 64;

// Volume-relative encoding of one sample.
struct Encoding {
  float bmin[3];
  float inv_ext[3];
};

__device__ __forceinline__ float freq(int k) { return exp2f((float)(7 * k) / 15.f); }

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// sin(pi x), cos(pi x): x is reduced to r = x - 2 rint(x/2) in [-1, 1] (exact in
// float), then the hardware sine and cosine take pi r (|pi r| <= pi, where
// their absolute error is about 2^-21); the features are rounded to bfloat16.
__device__ __forceinline__ void sincospi_fast(float x, float* s, float* c) {
  const float r = x - 2.f * rintf(0.5f * x);
  __sincosf(3.14159265358979f * r, s, c);
}

// A sin/cos feature pair, c in [6, kUsed): the branch of feature_pair below.
__device__ __forceinline__ void sincos_pair(const float u[3], int c, const float* fk, float& a, float& b) {
  const int q = c - 6, ax = q >> 5, k = (q & 31) >> 1;
  sincospi_fast(fk[k] * u[ax], &a, &b);
}

// The (even) feature pair starting at column c of the encoding; fk[k] holds
// freq(k) (a table filled once per block by the same function, so the
// features are identical to computing it here).
__device__ __forceinline__ void feature_pair(const float u[3], const float l[3], int c, float& a, float& b,
                                             const float* fk = nullptr) {
  if (c >= 6 && c < kUsed) {
    const int q = c - 6, ax = q >> 5, k = (q & 31) >> 1;
    sincospi_fast((fk ? fk[k] : freq(k)) * u[ax], &a, &b);
  } else if (c == 0) {
    a = u[0] * 2.f - 1.f;
    b = u[1] * 2.f - 1.f;
  } else if (c == 2) {
    a = u[2] * 2.f - 1.f;
    b = l[0];
  } else if (c == 4) {
    a = l[1];
    b = l[2];
  } else {
    a = 0.f;
    b = 0.f;
  }
}

// Writes the kIn features of position p (world space) under light feature l.
__device__ __forceinline__ void normalised(const Encoding& e, const float p[3], float u[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) u[a] = (p[a] - e.bmin[a]) * e.inv_ext[a];
}

template <typename Out>
__device__ __forceinline__ void encode(const Encoding& e, const float p[3], const float l[3], Out&& out) {
  float u[3];
  normalised(e, p, u);
#pragma unroll 1
  for (int c = 0; c < kIn; c += 2) {
    float a, b;
    feature_pair(u, l, c, a, b);
    out(c, a);
    out(c + 1, b);
  }
}

}  // namespace mlp
}  // namespace beams
