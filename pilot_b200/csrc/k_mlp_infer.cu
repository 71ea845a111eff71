// k_mlp_infer.cu — the learned form's render: the view march with the
// transmittance network in place of the map lookup.
//
// The shading transmittance never feeds back into the march: the reference's
// alpha accumulation and early termination (LightedVolumeRenderer.cxx:464-492)
// use the TF alpha only. So each ray marches ahead, buffering its lit samples'
// TF colour and premultiplied alpha, and the network is evaluated at "knots":
// the first lit sample and then every `knot`-th lit sample (and the last). The
// samples between two knots take T interpolated linearly along the ray, then
// composite in the reference order. With knot = 1 every lit sample is
// evaluated.
//
// The network runs on the tensor cores: each warp evaluates its 32 rays'
// knots as two 16-row tiles with mma.sync m16n8k16 (bfloat16 in, float32
// accumulate). The encoding is computed straight into A-fragment registers,
// each layer's float32 output (bias, ReLU, rounded to bfloat16) becomes the
// next layer's A fragment in registers, and the weights sit in shared memory
// pre-packed in B-fragment order (one conflict-free 8-byte load per mma).
// Compiled with -fmad=false like every kernel file.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "exact_device.cuh"
#include "kernels.h"
#include "mlp_common.cuh"

namespace beams {
namespace mlp {

// Offset of layer l's packed B fragments (uint2 entries).
__host__ __device__ constexpr int off_l(int l) {
  return l == 0 ? 0 : (l == 1 ? 7 * 8 * 32 : (l == 2 ? 7 * 8 * 32 + 4 * 8 * 32 : 7 * 8 * 32 + 2 * 4 * 8 * 32));
}
constexpr int kPacked = 7 * 8 * 32 + 3 * 4 * 8 * 32;  // uint2 entries
constexpr int kAux = 4 * kHid + kHid + 1;             // biases, w5, b5

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma16816(float c[4], const unsigned a[4], const uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// B fragments of W_l (row-major [in][64]) for every (k-tile, n-tile, lane):
// lane (g = lane/4, t = lane%4) holds rows 16kt+2t, +1 and 16kt+2t+8, +9 of
// column 8nt+g, bfloat16 pairs (low half = lower row). The fragments of
// n-tiles 2j and 2j+1 sit side by side for each lane, so one 16-byte load
// fetches both: uint2 index ((kt*4 + j)*32 + lane)*2 + (nt & 1) in the layer.
__global__ void k_pack_weights(const float* __restrict__ P, uint2* __restrict__ W, float* __restrict__ aux) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kPacked) {
    int l = 0;
    while (l < 3 && i >= off_l(l + 1)) ++l;
    const int rel = i - off_l(l);
    const int lane = (rel >> 1) & 31, nt = 2 * ((rel >> 6) & 3) + (rel & 1), kt = rel >> 8;
    const int g = lane >> 2, t = lane & 3;
    const int woff = (l == 0) ? oW1 : (l == 1 ? oW2 : (l == 2 ? oW3 : oW4));
    const int col = 8 * nt + g, r0 = 16 * kt + 2 * t;
    const float* w = P + woff;
    W[i] = make_uint2(pack_bf16(w[r0 * kHid + col], w[(r0 + 1) * kHid + col]),
                      pack_bf16(w[(r0 + 8) * kHid + col], w[(r0 + 9) * kHid + col]));
  }
  if (i < kAux) {
    float v;
    if (i < 4 * kHid) {
      const int l = i / kHid, c = i - l * kHid;
      v = P[(l == 0 ? oB1 : (l == 1 ? oB2 : (l == 2 ? oB3 : oB4))) + c];
    } else if (i < 5 * kHid) {
      v = bf16r(P[oW5 + (i - 4 * kHid)]);
    } else {
      v = P[oB5];
    }
    aux[i] = v;
  }
}

// Bias, ReLU, bfloat16: C fragments of n-tiles 2j, 2j+1 become A fragment j.
__device__ __forceinline__ void to_a(const float C[8][4], const float* bias, int t, unsigned A[4][4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c0 = 16 * j + 2 * t, c1 = c0 + 8;
    const float b00 = bias[c0], b01 = bias[c0 + 1], b10 = bias[c1], b11 = bias[c1 + 1];
    A[j][0] = pack_bf16(fmaxf(C[2 * j][0] + b00, 0.f), fmaxf(C[2 * j][1] + b01, 0.f));
    A[j][1] = pack_bf16(fmaxf(C[2 * j][2] + b00, 0.f), fmaxf(C[2 * j][3] + b01, 0.f));
    A[j][2] = pack_bf16(fmaxf(C[2 * j + 1][0] + b10, 0.f), fmaxf(C[2 * j + 1][1] + b11, 0.f));
    A[j][3] = pack_bf16(fmaxf(C[2 * j + 1][2] + b10, 0.f), fmaxf(C[2 * j + 1][3] + b11, 0.f));
  }
}

// T for the calling lane's row (lane = row of the warp's 32-row batch); every
// lane of the warp must call it. kp: this lane's knot position; lf: light feature.
__device__ __forceinline__ float mlp_eval_warp(const Encoding& enc, const float kp[3], const float lf[3],
                                               const uint2* __restrict__ sW, const float* __restrict__ sAux,
                                               const float* __restrict__ s_freq) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float mine = 0.f;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const int ra = mt * 16 + g, rb = ra + 8;
    float pa[3], pb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      pa[d] = __shfl_sync(0xffffffffu, kp[d], ra);
      pb[d] = __shfl_sync(0xffffffffu, kp[d], rb);
    }
    float ua[3], ub[3];
    normalised(enc, pa, ua);
    normalised(enc, pb, ub);
    float C[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n) C[n][0] = C[n][1] = C[n][2] = C[n][3] = 0.f;
    // layer 1: K = 112 (7 k-tiles), features computed into A fragments
#pragma unroll 1
    for (int kt = 0; kt < 7; ++kt) {
      const int c0 = 16 * kt + 2 * t, c1 = c0 + 8;
      float x0, x1, y0, y1, z0, z1, w0, w1;
      if (kt >= 1 && kt <= 5) {  // columns 16..95: sin/cos features only
        sincos_pair(ua, c0, s_freq, x0, x1);
        sincos_pair(ub, c0, s_freq, y0, y1);
        sincos_pair(ua, c1, s_freq, z0, z1);
        sincos_pair(ub, c1, s_freq, w0, w1);
      } else {
        feature_pair(ua, lf, c0, x0, x1, s_freq);
        feature_pair(ub, lf, c0, y0, y1, s_freq);
        feature_pair(ua, lf, c1, z0, z1, s_freq);
        feature_pair(ub, lf, c1, w0, w1, s_freq);
      }
      const unsigned a[4] = {pack_bf16(x0, x1), pack_bf16(y0, y1), pack_bf16(z0, z1), pack_bf16(w0, w1)};
      const uint4* wb = reinterpret_cast<const uint4*>(sW + off_l(0) + kt * 256) + lane;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint4 w = wb[j * 32];
        mma16816(C[2 * j], a, make_uint2(w.x, w.y));
        mma16816(C[2 * j + 1], a, make_uint2(w.z, w.w));
      }
    }
    unsigned A[4][4];
    to_a(C, sAux, t, A);
    // layers 2..4: K = 64 (4 k-tiles)
#pragma unroll 1
    for (int l = 1; l < 4; ++l) {
#pragma unroll
      for (int n = 0; n < 8; ++n) C[n][0] = C[n][1] = C[n][2] = C[n][3] = 0.f;
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        const uint4* wb = reinterpret_cast<const uint4*>(sW + off_l(l) + kt * 256) + lane;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint4 w = wb[j * 32];
          mma16816(C[2 * j], A[kt], make_uint2(w.x, w.y));
          mma16816(C[2 * j + 1], A[kt], make_uint2(w.z, w.w));
        }
      }
      to_a(C, sAux + l * kHid, t, A);
    }
    // head: z = b5 + h4 . w5 over this lane's 16 columns, reduced over the quad
    // A[j][0] / A[j][2] hold row ra columns 16j+2t(+1) / 16j+8+2t(+1); [1]/[3] row rb
    const float* w5 = sAux + 4 * kHid;
    float za = 0.f, zb = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c0 = 16 * j + 2 * t, c1 = c0 + 8;
      const __nv_bfloat162 h0 = *reinterpret_cast<const __nv_bfloat162*>(&A[j][0]);
      const __nv_bfloat162 h1 = *reinterpret_cast<const __nv_bfloat162*>(&A[j][1]);
      const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&A[j][2]);
      const __nv_bfloat162 h3 = *reinterpret_cast<const __nv_bfloat162*>(&A[j][3]);
      za = fmaf(__low2float(h0), w5[c0], za);
      za = fmaf(__high2float(h0), w5[c0 + 1], za);
      za = fmaf(__low2float(h2), w5[c1], za);
      za = fmaf(__high2float(h2), w5[c1 + 1], za);
      zb = fmaf(__low2float(h1), w5[c0], zb);
      zb = fmaf(__high2float(h1), w5[c0 + 1], zb);
      zb = fmaf(__low2float(h3), w5[c1], zb);
      zb = fmaf(__high2float(h3), w5[c1 + 1], zb);
    }
    za += __shfl_xor_sync(0xffffffffu, za, 1);
    za += __shfl_xor_sync(0xffffffffu, za, 2);
    zb += __shfl_xor_sync(0xffffffffu, zb, 1);
    zb += __shfl_xor_sync(0xffffffffu, zb, 2);
    const float b5 = sAux[5 * kHid];
    const float Ta = 1.f / (1.f + __expf(-(za + b5)));
    const float Tb = 1.f / (1.f + __expf(-(zb + b5)));
    // row r of this tile: r - mt*16 < 8 -> Ta of lane 4(r-mt*16); else Tb of lane 4(r-mt*16-8)
    const int rr = lane - mt * 16;
    const int src = (rr >= 0 && rr < 16) ? 4 * (rr & 7) : 0;
    const float va = __shfl_sync(0xffffffffu, Ta, src);
    const float vb = __shfl_sync(0xffffffffu, Tb, src);
    if (rr >= 0 && rr < 16) mine = (rr < 8) ? va : vb;
  }
  return mine;
}

}  // namespace mlp

using namespace mlp;

constexpr int kKnotMax = 64;  // lit samples between two network evaluations, at most

__device__ __forceinline__ int next_warp_tile_mlp(unsigned* counter) {
  unsigned t = 0;
  if ((threadIdx.x & 31) == 0) t = atomicAdd(counter, 1u);
  return (int)__shfl_sync(0xffffffffu, t, 0);
}

// View march shaded by the network (see the file comment).
template <typename QuadT>
__global__ void __launch_bounds__(256, 2) k_view_march_mlp(const ExactGeo g, const QuadT* __restrict__ quads,
                                                           const float4* __restrict__ tab,
                                                           const float4* __restrict__ tf,
                                                           const uint2* __restrict__ Wp,
                                                           const float* __restrict__ aux, Encoding enc,
                                                           float lf0, float lf1, float lf2, int knot,
                                                           float4* __restrict__ out, Counters* __restrict__ cnt,
                                                           MlpProbe probe, MlpPass pass) {
  extern __shared__ float4 s_dyn[];
  const int nfield = g.max_off[0];
  float4* s_tab = s_dyn;
  float4* s_tf = s_dyn + nfield;
  uint2* sW = reinterpret_cast<uint2*>(s_tf + g.tf_n);
  float* sAux = reinterpret_cast<float*>(sW + kPacked);
  // per warp, the TF indices of the round's pending lit samples: [warp][j][lane]
  unsigned short* s_idx = reinterpret_cast<unsigned short*>(sAux + ((kAux + 3) & ~3)) +
                          (threadIdx.x >> 5) * (kKnotMax * 32) + (threadIdx.x & 31);
  for (int i = threadIdx.x; i < nfield; i += blockDim.x) s_tab[i] = tab[i];
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  for (int i = threadIdx.x; i < kPacked; i += blockDim.x) sW[i] = Wp[i];
  for (int i = threadIdx.x; i < kAux; i += blockDim.x) sAux[i] = aux[i];
  __shared__ float s_freq[kFreq];  // the encoding's frequencies, once per block
  if (threadIdx.x < kFreq) s_freq[threadIdx.x] = freq(threadIdx.x);
  __syncthreads();
  const float lf[3] = {lf0, lf1, lf2};
  const int tiles_x = (g.width + 7) >> 3;
  const int nprobe = probe.nqx * probe.nqy;
  const int ntiles = pass.probes_only ? (nprobe + 31) >> 5 : tiles_x * ((g.height + 3) >> 2);
  const unsigned qx = (unsigned)(g.n[0] - 1), qz = (unsigned)(g.n[0] - 1) * (unsigned)(g.n[1] - 1);
  const int n1 = g.tf_n - 1;
  unsigned lit = 0, hit = 0, evals = 0, rows = 0;
  for (int tile = next_warp_tile_mlp(&cnt->tiles_view); tile < ntiles; tile = next_warp_tile_mlp(&cnt->tiles_view)) {
    const int lane = threadIdx.x & 31;
    int x, y;
    if (pass.probes_only) {
      // probe q = 32 tile + lane; lanes past the grid get no pixel
      const int q = tile * 32 + lane;
      x = q < nprobe ? (q % probe.nqx) * probe.P + probe.h : g.width;
      y = q < nprobe ? (q / probe.nqx) * probe.P + probe.h : g.height;
    } else {
      const int x0 = (tile % tiles_x) * 8, y0 = (tile / tiles_x) * 4;
      // an 8x4 tile lies inside one fallback tile: the exact path renders it
      if (pass.skip && pass.skip[(y0 / kFallbackTile) * pass.ftx + x0 / kFallbackTile] != 0u) continue;
      x = x0 + (lane & 7);
      y = y0 + (lane >> 3);
    }
    // a probe pixel records its compositing samples for the exact-march check
    const bool is_probe = probe.P > 0 && x < g.width && y < g.height && x % probe.P == probe.h &&
                          y % probe.P == probe.h && x / probe.P < probe.nqx && y / probe.P < probe.nqy;
    float4* prec = is_probe ? probe.rec + (size_t)((y / probe.P) * probe.nqx + x / probe.P) * probe.cap * 2 : nullptr;
    int pn = 0;
    float4 color = make_float4(0.f, 0.f, 0.f, 0.f);
    float o[3] = {0.f, 0.f, 0.f}, d[3] = {0.f, 0.f, 1.f}, minD = 0.f, maxD = -1.f;
    bool done = true;
    if (x < g.width && y < g.height && ray_setup(g, x, y, o, d, minD, maxD)) {
      done = false;
      hit += 1;
    }
    const float qd = (maxD - minD) / g.sd;
    long long budget = (!done && qd < 1e9f) ? (long long)qd + 16 : (done ? 0ll : 1000000000ll);
    float dist = minD + g.mesh_eps;
    float p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
    while (!done && !inside_vol(g, p) && dist < maxD && budget-- > 0) {
      dist += g.sd;
      p[0] = o[0] + dist * d[0];
      p[1] = o[1] + dist * d[1];
      p[2] = o[2] + dist * d[2];
    }
    const float sdx = g.sd * d[0], sdy = g.sd * d[1], sdz = g.sd * d[2];
    float bl[3] = {0.f, 0.f, 0.f}, inv[3] = {0.f, 0.f, 0.f};
    bool newCell = true;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    float s0 = 0.f, s1m0 = 0.f, s2m3 = 0.f, s3 = 0.f, s4 = 0.f, s5m4 = 0.f, s6m7 = 0.f, s7 = 0.f;
    float Tprev = 1.f;
    bool have_prev = false;
    // march state lives across rounds; each round gathers up to `need` lit samples
    while (__any_sync(0xffffffffu, !done)) {
      // The round's lit samples are kept as their TF indices only (16 bits in
      // shared memory); compositing replays the alpha recurrence from the
      // round's starting alpha, which gives back each sample's premultiplied
      // alpha bit for bit.
      const float cw0 = color.w;
      int nb = 0;
      float kp[3] = {p[0], p[1], p[2]};
      const int need = have_prev ? knot : 1;
      while (!done && nb < need) {
        if (!(inside_vol(g, p) && dist < maxD && budget-- > 0)) {
          done = true;
          break;
        }
        const float mint = mn(tx, mn(ty, tz));
        const float maxt = mx(tx, mx(ty, tz));
        if (maxt > 1.f || mint < 0.f) newCell = true;
        if (newCell) {
          int c[3];
          locate_view_cell(g, s_tab, p, c, inv, bl);
          float v[8];
          QuadLoad<QuadT>::cell(quads, (unsigned)c[2] * qz + (unsigned)c[1] * qx + (unsigned)c[0], qx, qz, v);
          s0 = v[0];
          s3 = v[3];
          s4 = v[4];
          s7 = v[7];
          s6m7 = v[6] - v[7];
          s5m4 = v[5] - v[4];
          s1m0 = v[1] - v[0];
          s2m3 = v[2] - v[3];
          tx = (p[0] - bl[0]) * inv[0];
          ty = (p[1] - bl[1]) * inv[1];
          tz = (p[2] - bl[2]) * inv[2];
          newCell = false;
        }
        const float l76 = s7 + tx * s6m7;
        const float l45 = s4 + tx * s5m4;
        const float top = l45 + ty * (l76 - l45);
        const float l01 = s0 + tx * s1m0;
        const float l32 = s3 + tx * s2m3;
        const float bot = l01 + ty * (l32 - l01);
        float fs = bot + tz * (top - bot);
        fs = (fs - g.min_scalar) * g.inv_delta;
        const float fi = fs * (float)n1;
        if (fi > -1.f && fi < (float)(n1 + 1)) {
          const int ti = trunc_small(fmaxf(fi, 0.f));  // (int)fi: fi in (-1, n1 + 1)
          const float4 tfc = s_tf[ti];
          const float sa = tfc.w * (1.f - color.w);
          s_idx[nb * 32] = (unsigned short)ti;
          if (is_probe && sa > 0.f) {
            if (pn < probe.cap) {
              prec[2 * pn] = make_float4(p[0], p[1], p[2], 1.f);
              prec[2 * pn + 1] = make_float4(tfc.x, tfc.y, tfc.z, sa);
            }
            ++pn;
          }
          kp[0] = p[0];
          kp[1] = p[1];
          kp[2] = p[2];
          ++nb;
          color.w = sa + color.w;
          ++lit;
        }
        dist += g.sd;
        p[0] = p[0] + sdx;
        p[1] = p[1] + sdy;
        p[2] = p[2] + sdz;
        tx = (p[0] - bl[0]) * inv[0];
        ty = (p[1] - bl[1]) * inv[1];
        tz = (p[2] - bl[2]) * inv[2];
        if (color.w >= g.cutoff) done = true;
      }
      const float Tk = mlp_eval_warp(enc, kp, lf, sW, sAux, s_freq);
      rows += 32;
      if (nb > 0) {
        ++evals;
        const float inv_nb = 1.f / (float)nb;
        float cw = cw0;
        for (int j = 0; j < nb; ++j) {
          const float T = have_prev ? Tprev + (Tk - Tprev) * ((float)(j + 1) * inv_nb) : Tk;
          const float4 b = s_tf[s_idx[j * 32]];
          const float sa = b.w * (1.f - cw);
          cw = sa + cw;
          const float sc0 = clamp01(b.x * (T * g.light_color[0]));
          const float sc1 = clamp01(b.y * (T * g.light_color[1]));
          const float sc2 = clamp01(b.z * (T * g.light_color[2]));
          color.x = color.x + sc0 * sa;
          color.y = color.y + sc1 * sa;
          color.z = color.z + sc2 * sa;
        }
        Tprev = Tk;
        have_prev = true;
      }
    }
    if (x < g.width && y < g.height) out[(size_t)y * g.width + x] = color;
    if (is_probe) probe.count[(y / probe.P) * probe.nqx + x / probe.P] = pn;
  }
  if (!pass.probes_only) {
    warp_add(&cnt->lit_samples, lit);
    warp_add(&cnt->rays_hit, hit);
  }
  warp_add(&cnt->mlp_samples, evals);
  if ((threadIdx.x & 31) == 0 && rows) atomicAdd(&cnt->mlp_rows, (unsigned long long)rows);
}

cudaError_t launch_pack_weights(const float* P, uint2* W, float* aux, cudaStream_t st) {
  k_pack_weights<<<(kPacked + 255) / 256, 256, 0, st>>>(P, W, aux);
  return cudaGetLastError();
}

size_t mlp_packed_bytes() { return (size_t)kPacked * sizeof(uint2) + (size_t)kAux * sizeof(float); }

cudaError_t launch_view_march_mlp(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                  const uint2* W, const float* aux, const Encoding& enc, const float lf[3], int knot,
                                  float4* out, Counters* cnt, const MlpProbe& probe, const MlpPass& pass,
                                  cudaStream_t st) {
  if (knot < 1 || knot > kKnotMax) return cudaErrorInvalidValue;
  if (pass.probes_only && (probe.P < 1 || !probe.rec || !probe.count)) return cudaErrorInvalidValue;
  const size_t smem = (size_t)g.max_off[0] * sizeof(float4) + (size_t)g.tf_n * sizeof(float4) +
                      (size_t)kPacked * sizeof(uint2) + (size_t)((kAux + 3) & ~3) * sizeof(float) +
                      (size_t)8 * kKnotMax * 32 * sizeof(unsigned short);
  cudaError_t e = cudaFuncSetAttribute(k_view_march_mlp<float4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_view_march_mlp<float4>, 256, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = pass.probes_only ? (probe.nqx * probe.nqy + 31) / 32 : ((g.width + 7) >> 3) * ((g.height + 3) >> 2);
  int grid = sms * per_sm;
  const int need = (ntiles + 7) / 8;
  if (grid > need) grid = need;
  if (grid < 1) return cudaSuccess;
  k_view_march_mlp<float4><<<grid, 256, smem, st>>>(g, quads, tab, tf, W, aux, enc, lf[0], lf[1], lf[2], knot, out,
                                                    cnt, probe, pass);
  return cudaGetLastError();
}

}  // namespace beams
