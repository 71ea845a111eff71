// k_exact.cu — exact-form kernels.
//
// K1 light_march: one thread per map vertex ((M+1)^3), restating
//   TransmittanceMapGenerator::operator() (beams/rendering/TransmittanceMap.h:279-332)
//   with the light ray built in registers (LightRayOperations.h:32-43).
// K2 view_march: one thread per pixel, 8x4-pixel warp tiles, restating
//   CalcRayStart (LightedVolumeRenderer.cxx:644-718) and Sampler::operator()
//   (LightedVolumeRenderer.cxx:346-498) with the map lookup of
//   TransmittanceMapEstimator::GetEstimateUsingVertices (TransmittanceMap.h:166-197).
// K2c view_march_cells: SamplerCellAssoc::operator() (LightedVolumeRenderer.cxx:540-641).
//
// Compiled with -fmad=false (see exact_device.cuh).
#include <cuda_runtime.h>

#include "exact_device.cuh"
#include "kernels.h"

namespace beams {

constexpr int kMaxTF = 1024;

// ---------------------------------------------------------------------------
// K1
// ---------------------------------------------------------------------------
template <typename FieldT>
__global__ void __launch_bounds__(256) k_light_march(const ExactGeo g, const FieldT* __restrict__ field,
                                                     const float4* __restrict__ tf,
                                                     float* __restrict__ map, int64_t nvert,
                                                     Counters* __restrict__ cnt) {
  __shared__ float s_a[kMaxTF];  // TF alpha / max alpha (TransmittanceMap.h:329)
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x)
    s_a[i] = (g.max_alpha > 0.f) ? tf[i].w / g.max_alpha : 0.f;
  __syncthreads();

  const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned ns = 0;
  if (id < nvert) {
    float V[3], L[3];
    map_vertex(g, id, V);
    light_origin(g, V, L);
    const float v[3] = {V[0] - L[0], V[1] - L[1], V[2] - L[2]};
    const float rs = 1.f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const float dir[3] = {v[0] * rs, v[1] * rs, v[2] * rs};
    float tmin, tmax;
    segment_aabb(g, L, V, tmin, tmax);
    const float st[3] = {L[0] + tmin * dir[0], L[1] + tmin * dir[1], L[2] + tmin * dir[2]};
    float s[3] = {st[0], st[1], st[2]};
    const float len2 = (tmax - tmin) * (tmax - tmin);
    const float sdx = g.step * dir[0], sdy = g.step * dir[1], sdz = g.step * dir[2];
    const int n1 = g.tf_n - 1;
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    float o = 0.f;
    for (int b = g.light_budget; b > 0; --b) {
      const float q0 = s[0] - st[0], q1 = s[1] - st[1], q2 = s[2] - st[2];
      if (!(q0 * q0 + q1 * q1 + q2 * q2 <= len2)) break;
      s[0] = s[0] + sdx;
      s[1] = s[1] + sdy;
      s[2] = s[2] + sdz;
      if (!inside_vol(g, s)) break;
      int c[3];
      float pc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        c[d] = find_cell_bsearch(g, d, s[d]);
        const float lo = coord(g, d, c[d]);
        const float hi = coord(g, d, c[d] + 1);
        pc[d] = (s[d] - lo) / (hi - lo);
      }
      const int64_t i0 = (int64_t)c[2] * nxy + (int64_t)c[1] * nx + c[0];
      float vals[8];
      vals[0] = FieldLoad<FieldT>::ld(field, i0);
      vals[1] = FieldLoad<FieldT>::ld(field, i0 + 1);
      vals[2] = FieldLoad<FieldT>::ld(field, i0 + 1 + nx);
      vals[3] = FieldLoad<FieldT>::ld(field, i0 + nx);
      vals[4] = FieldLoad<FieldT>::ld(field, i0 + nxy);
      vals[5] = FieldLoad<FieldT>::ld(field, i0 + nxy + 1);
      vals[6] = FieldLoad<FieldT>::ld(field, i0 + nxy + 1 + nx);
      vals[7] = FieldLoad<FieldT>::ld(field, i0 + nxy + nx);
      float scalar = hex_interp(vals, pc[0], pc[1], pc[2]);
      scalar = (scalar - g.min_scalar) * g.inv_delta;
      const int idx = tf_index_clamped(scalar * (float)n1, n1);
      o = o + (1.f - o) * s_a[idx];
      ++ns;
      // o == 1 is a fixed point of o + (1-o)a: the remaining samples cannot change it.
      if (o == 1.f) break;
    }
    map[id] = o;
  }
  warp_add(&cnt->light_samples, ns);
}

// ---------------------------------------------------------------------------
// K2 (point field)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tile_pixel(const ExactGeo& g, int& x, int& y) {
  // 16x16-pixel blocks of 8 warps; each warp owns an 8x4 tile.
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_x = (g.width + 15) >> 4;
  const int bx = blockIdx.x % tiles_x, by = blockIdx.x / tiles_x;
  x = (bx << 4) + ((w & 1) << 3) + (lane & 7);
  y = (by << 4) + ((w >> 1) << 2) + (lane >> 3);
}

template <typename FieldT, bool USE_MAP>
__device__ __forceinline__ void view_march_pixel(const ExactGeo& g, const FieldT* __restrict__ field,
                                                 const float4* s_tf, const float* __restrict__ map,
                                                 int x, int y, float4& color, unsigned& lit,
                                                 unsigned& hit) {
  color = make_float4(0.f, 0.f, 0.f, 0.f);
  float o[3], d[3], minD, maxD;
  if (!ray_setup(g, x, y, o, d, minD, maxD)) return;
  hit = 1;
  const float qd = (maxD - minD) / g.sd;
  long long budget = (qd < 1e9f) ? (long long)qd + 16 : 1000000000ll;
  float dist = minD + g.mesh_eps;
  float p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
  while (!inside_vol(g, p) && dist < maxD && budget-- > 0) {
    dist += g.sd;
    p[0] = o[0] + dist * d[0];
    p[1] = o[1] + dist * d[1];
    p[2] = o[2] + dist * d[2];
  }
  const float sdx = g.sd * d[0], sdy = g.sd * d[1], sdz = g.sd * d[2];
  float bl[3] = {0.f, 0.f, 0.f};
  bool newCell = true;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  float s0 = 0.f, s1m0 = 0.f, s2m3 = 0.f, s3 = 0.f, s4 = 0.f, s5m4 = 0.f, s6m7 = 0.f, s7 = 0.f;
  int c[3] = {0, 0, 0};
  float inv[3] = {0.f, 0.f, 0.f};
  const int n1 = g.tf_n - 1;
  const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
  while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
    const float mint = mn(tx, mn(ty, tz));
    const float maxt = mx(tx, mx(ty, tz));
    if (maxt > 1.f || mint < 0.f) newCell = true;
    if (newCell) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (p[k] == g.maxp[k]) {
          c[k] = g.n[k] - 2;  // the reference leaves invSpacing[k] unchanged here
        } else {
          c[k] = find_cell_walk(g, k, p[k]);
          inv[k] = 1.f / (coord(g, k, c[k] + 1) - coord(g, k, c[k]));
        }
        bl[k] = coord(g, k, c[k]);
      }
      const int64_t i0 = (int64_t)c[2] * nxy + (int64_t)c[1] * nx + c[0];
      s0 = FieldLoad<FieldT>::ld(field, i0);
      const float s1 = FieldLoad<FieldT>::ld(field, i0 + 1);
      const float s2 = FieldLoad<FieldT>::ld(field, i0 + 1 + nx);
      s3 = FieldLoad<FieldT>::ld(field, i0 + nx);
      s4 = FieldLoad<FieldT>::ld(field, i0 + nxy);
      const float s5 = FieldLoad<FieldT>::ld(field, i0 + nxy + 1);
      const float s6 = FieldLoad<FieldT>::ld(field, i0 + nxy + 1 + nx);
      s7 = FieldLoad<FieldT>::ld(field, i0 + nxy + nx);
      s6m7 = s6 - s7;
      s5m4 = s5 - s4;
      s1m0 = s1 - s0;
      s2m3 = s2 - s3;
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
      const float4 tfc = s_tf[(int)fi];
      float sc0 = tfc.x, sc1 = tfc.y, sc2 = tfc.z;
      const float sa = tfc.w * (1.f - color.w);
      if (USE_MAP) {
        const float tr = 1.f - map_opacity<float>(g, map, p);
        sc0 = sc0 * (tr * g.light_color[0]);
        sc1 = sc1 * (tr * g.light_color[1]);
        sc2 = sc2 * (tr * g.light_color[2]);
      }
      sc0 = clamp01(sc0);
      sc1 = clamp01(sc1);
      sc2 = clamp01(sc2);
      color.x = color.x + sc0 * sa;
      color.y = color.y + sc1 * sa;
      color.z = color.z + sc2 * sa;
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
    if (color.w >= g.cutoff) break;
  }
}

template <typename FieldT, bool USE_MAP>
__global__ void __launch_bounds__(256) k_view_march(const ExactGeo g, const FieldT* __restrict__ field,
                                                    const float4* __restrict__ tf,
                                                    const float* __restrict__ map,
                                                    float4* __restrict__ out,
                                                    Counters* __restrict__ cnt) {
  __shared__ float4 s_tf[kMaxTF];
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  int x, y;
  tile_pixel(g, x, y);
  unsigned lit = 0, hit = 0;
  if (x < g.width && y < g.height) {
    float4 color;
    view_march_pixel<FieldT, USE_MAP>(g, field, s_tf, map, x, y, color, lit, hit);
    out[(int64_t)y * g.width + x] = color;
  }
  warp_add(&cnt->lit_samples, lit);
  warp_add(&cnt->rays_hit, hit);
}

// ---------------------------------------------------------------------------
// K2c (cell field, unlit)
// ---------------------------------------------------------------------------
template <typename FieldT>
__global__ void __launch_bounds__(256) k_view_march_cells(const ExactGeo g,
                                                          const FieldT* __restrict__ field,
                                                          const float4* __restrict__ tf,
                                                          float4* __restrict__ out,
                                                          Counters* __restrict__ cnt) {
  __shared__ float4 s_tf[kMaxTF];
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  int x, y;
  tile_pixel(g, x, y);
  unsigned lit = 0, hit = 0;
  if (x < g.width && y < g.height) {
    float4 color = make_float4(0.f, 0.f, 0.f, 0.f);
    float o[3], d[3], minD, maxD;
    if (ray_setup(g, x, y, o, d, minD, maxD)) {
      hit = 1;
      const float qd = (maxD - minD) / g.sd;
      long long budget = (qd < 1e9f) ? (long long)qd + 16 : 1000000000ll;
      float dist = minD + g.mesh_eps;
      float p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
      while (!inside_vol(g, p) && dist < maxD && budget-- > 0) {
        dist += g.sd;
        p[0] = o[0] + dist * d[0];
        p[1] = o[1] + dist * d[1];
        p[2] = o[2] + dist * d[2];
      }
      const float sdx = g.sd * d[0], sdy = g.sd * d[1], sdz = g.sd * d[2];
      bool newCell = true;
      float tx = 2.f, ty = 2.f, tz = 2.f;
      float4 sc = make_float4(0.f, 0.f, 0.f, 0.f);
      float bl[3] = {0.f, 0.f, 0.f};
      float inv[3] = {0.f, 0.f, 0.f};
      int c[3] = {0, 0, 0};
      const int n1 = g.tf_n - 1;
      const int64_t cx = g.n[0] - 1, cxy = (int64_t)(g.n[0] - 1) * (g.n[1] - 1);
      while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
        const float mint = mn(tx, mn(ty, tz));
        const float maxt = mx(tx, mx(ty, tz));
        if (maxt > 1.f || mint < 0.f) newCell = true;
        if (newCell) {
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            if (p[k] == g.maxp[k]) {
              c[k] = g.n[k] - 2;
            } else {
              c[k] = find_cell_walk(g, k, p[k]);
              inv[k] = 1.f / (coord(g, k, c[k] + 1) - coord(g, k, c[k]));
            }
            bl[k] = coord(g, k, c[k]);
          }
          const int64_t cid = (int64_t)c[2] * cxy + (int64_t)c[1] * cx + c[0];
          const float v = FieldLoad<FieldT>::ld(field, cid);
          const float nsv = (v - g.min_scalar) * g.inv_delta;
          sc = s_tf[tf_index_clamped(nsv * (float)n1, n1)];
          tx = (p[0] - bl[0]) * inv[0];
          ty = (p[1] - bl[1]) * inv[1];
          tz = (p[2] - bl[2]) * inv[2];
          newCell = false;
        }
        const float alpha = sc.w * (1.f - color.w);
        color.x = color.x + sc.x * alpha;
        color.y = color.y + sc.y * alpha;
        color.z = color.z + sc.z * alpha;
        color.w = alpha + color.w;
        ++lit;
        dist += g.sd;
        p[0] = p[0] + sdx;
        p[1] = p[1] + sdy;
        p[2] = p[2] + sdz;
        if (color.w >= g.cutoff) break;
        tx = (p[0] - bl[0]) * inv[0];
        ty = (p[1] - bl[1]) * inv[1];
        tz = (p[2] - bl[2]) * inv[2];
      }
      color.x = mn(color.x, 1.f);
      color.y = mn(color.y, 1.f);
      color.z = mn(color.z, 1.f);
      color.w = mn(color.w, 1.f);
    }
    out[(int64_t)y * g.width + x] = color;
  }
  warp_add(&cnt->lit_samples, lit);
  warp_add(&cnt->rays_hit, hit);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t launch_light_march_f32(const ExactGeo& g, const float* field, const float4* tf,
                                   float* map, Counters* cnt, cudaStream_t st) {
  const int64_t nvert = (int64_t)g.pd[0] * g.pd[1] * g.pd[2];
  const int64_t blocks = (nvert + 255) / 256;
  k_light_march<float><<<(unsigned)blocks, 256, 0, st>>>(g, field, tf, map, nvert, cnt);
  return cudaGetLastError();
}

cudaError_t launch_view_march_f32(const ExactGeo& g, const float* field, const float4* tf,
                                  const float* map, float4* out, Counters* cnt, cudaStream_t st) {
  const int blocks = ((g.width + 15) >> 4) * ((g.height + 15) >> 4);
  if (g.assoc_cells) {
    k_view_march_cells<float><<<blocks, 256, 0, st>>>(g, field, tf, out, cnt);
  } else if (g.use_map) {
    k_view_march<float, true><<<blocks, 256, 0, st>>>(g, field, tf, map, out, cnt);
  } else {
    k_view_march<float, false><<<blocks, 256, 0, st>>>(g, field, tf, nullptr, out, cnt);
  }
  return cudaGetLastError();
}

}  // namespace beams
