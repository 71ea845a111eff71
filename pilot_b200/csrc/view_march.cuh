// view_march.cuh — the per-pixel view march (K2's body), shared by the exact
// and precision forms' K2 and by the learned form's probe of its pixels.
// Restates CalcRayStart (LightedVolumeRenderer.cxx:644-718) and
// Sampler::operator() (LightedVolumeRenderer.cxx:346-498).
#pragma once
#include <type_traits>

#include "exact_device.cuh"

namespace beams {

// 8x4-pixel warp tiles; tiles_x = ceil(width / 8).
__device__ __forceinline__ void tile_pixel(int tiles_x, int tile, int& x, int& y) {
  const int lane = threadIdx.x & 31;
  const int bx = tile % tiles_x, by = tile / tiles_x;
  x = (bx << 3) + (lane & 7);
  y = (by << 2) + (lane >> 3);
}

// Next warp tile from the frame's counter (one atomic per warp tile).
__device__ __forceinline__ int next_warp_tile(unsigned* counter) {
  unsigned t = 0;
  if ((threadIdx.x & 31) == 0) t = atomicAdd(counter, 1u);
  return (int)__shfl_sync(0xffffffffu, t, 0);
}

// A view-march observer: called once per lit sample with its position, TF
// entry and premultiplied alpha (the default observes nothing).
struct NoRecord {
  __device__ __forceinline__ void operator()(const float*, const float4&, float) {}
};

// A view-march observer that marks, for every lit sample of premultiplied
// alpha above 0, the map cell that the shading looks up (the cell of
// map_interp_t: truncate min(max((p - origin) / spacing, 0), pd - 2) per axis),
// one byte per cell, skipping repeats of the previous sample's cell. A sample
// of alpha 0 adds exactly 0 times its shading, so the map value it reads only
// has to be finite (the masked builds zero a newly allocated map). A masked map build then lists every vertex with a marked cell
// around it (the same vertex set as marking the 8 corners, with one store per
// cell).
struct CellMarker {
  float morig[3], minv[3];
  int pd[3];
  unsigned char* mask;
  unsigned last;
  __device__ __forceinline__ void operator()(const float* p, const float4&, float sa) {
    if (!(sa > 0.f)) return;
    int c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float t = (p[d] - morig[d]) * minv[d];
      c[d] = trunc_small(fminf(fmaxf(t, 0.f), (float)(pd[d] - 2)));
    }
    const unsigned mx = (unsigned)(pd[0] - 1), mxy = mx * (unsigned)(pd[1] - 1);
    const unsigned id = (unsigned)c[2] * mxy + (unsigned)c[1] * mx + (unsigned)c[0];
    if (id == last) return;
    last = id;
    mask[id] = 1;
  }
};

// SKIP: samples in macro-cells whose occupancy is 0 (every value there maps to
// an in-range TF entry of alpha 0) only advance and count as lit: their
// premultiplied alpha is 0, so they change neither colour nor alpha.
template <typename QuadT, bool USE_MAP, typename MapT, typename Rec = NoRecord, bool SKIP = false, bool MULTI = false,
          bool RECT = false>
__device__ __forceinline__ void view_march_pixel(const ExactGeo& g, const QuadT* __restrict__ quads,
                                                 const float4* s_tab, const float4* s_tf,
                                                 const MapT* __restrict__ map, int x, int y, float4& color,
                                                 unsigned& lit, unsigned& hit, Rec* rec = nullptr,
                                                 const unsigned char* __restrict__ occ = nullptr) {
  color = make_float4(0.f, 0.f, 0.f, 0.f);
  float o[3], d[3], minD, maxD;
  if (!ray_setup(g, x, y, o, d, minD, maxD)) return;
  hit += 1;
  const float qd = (maxD - minD) / g.sd;
  int budget = (qd < 1e9f) ? (int)qd + 16 : 1000000000;  // qd <= 1e6: the sample distance is checked on the host
  float dist = minD + g.mesh_eps;
  float p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
  while (!inside_vol(g, p) && dist < maxD && budget-- > 0) {
    dist += g.sd;
    p[0] = o[0] + dist * d[0];
    p[1] = o[1] + dist * d[1];
    p[2] = o[2] + dist * d[2];
  }
  const float sdx = g.sd * d[0], sdy = g.sd * d[1], sdz = g.sd * d[2];
  unsigned qx, qz;
  QuadLoad<QuadT>::strides(g, qx, qz);
  float bl[3] = {0.f, 0.f, 0.f};
  bool newCell = true;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  float s0 = 0.f, s1m0 = 0.f, s2m3 = 0.f, s3 = 0.f, s4 = 0.f, s5m4 = 0.f, s6m7 = 0.f, s7 = 0.f;
  int c[3] = {0, 0, 0};
  float inv[3] = {0.f, 0.f, 0.f};
  const int n1 = g.tf_n - 1;
  while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
    if (SKIP && !occupied(g, occ, p)) {
      ++lit;
      dist += g.sd;
      p[0] = p[0] + sdx;
      p[1] = p[1] + sdy;
      p[2] = p[2] + sdz;
      tx = (p[0] - bl[0]) * inv[0];
      ty = (p[1] - bl[1]) * inv[1];
      tz = (p[2] - bl[2]) * inv[2];
      continue;  // colour unchanged, so the cutoff test cannot newly pass
    }
    const float mint = mn(tx, mn(ty, tz));
    const float maxt = mx(tx, mx(ty, tz));
    if (maxt > 1.f || mint < 0.f) newCell = true;
    if (newCell) {
      if constexpr (RECT) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float4* T = s_tab + g.ax_off[k];
          float4 e;
          if (p[k] == g.maxp[k]) {
            c[k] = g.n[k] - 2;  // the reference leaves invSpacing[k] unchanged here
            e = T[c[k]];
          } else {
            c[k] = find_cell_walk_rect(T, g.n[k] - 2, p[k], e);
            inv[k] = e.w;  // 1.f / (coord(c+1) - coord(c)), IEEE
          }
          bl[k] = e.x;
        }
      } else {
        locate_view_cell(g, s_tab, p, c, inv, bl);
      }
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
      const float4 tfc = s_tf[trunc_small(fmaxf(fi, 0.f))];  // (int)fi: fi in (-1, n1 + 1)
      float sc0 = tfc.x, sc1 = tfc.y, sc2 = tfc.z;
      const float sa = tfc.w * (1.f - color.w);
      if (rec) (*rec)(p, tfc, sa);
      if (USE_MAP && MULTI) {
        float est[3];
        map_light_sum(g, s_tab, (const float*)map, p, est);
        sc0 = sc0 * est[0];
        sc1 = sc1 * est[1];
        sc2 = sc2 * est[2];
      } else if (USE_MAP) {
        // exact form: 1 - opacity (TransmittanceMap.h:195); precision form: stored transmittance
        const float mv = map_interp_t<MapT>(g, s_tab, map, p);
        const float tr = (sizeof(MapT) == 2) ? mv : 1.f - mv;
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

}  // namespace beams
