// exact_device.cuh — device restatement of the reference's per-sample math.
//
// Every translation unit that includes this header is compiled with
// -fmad=false: a*b+c stays two IEEE roundings, as in the reference's x86-64
// build, and the explicit fmaf() calls below are the only fused operations
// (lcl's lerp uses std::fma). Division and sqrtf are IEEE (no fast-math).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "beams_params.h"

namespace beams {

// vtkm::Min / vtkm::Max on the host are std::min / std::max.
template <typename T> __device__ __forceinline__ T mn(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T mx(T a, T b) { return (a < b) ? b : a; }
__device__ __forceinline__ float clamp01(float x) { return x < 0.f ? 0.f : (x > 1.f ? 1.f : x); }

// lcl::internal::lerp(a, b, t) = fma(t, b, fma(-t, a, a)).
__device__ __forceinline__ float lerp_lcl(float a, float b, float t) {
  return fmaf(t, b, fmaf(-t, a, a));
}

// vtkm::exec::CellInterpolate on a hexahedron (lcl trilinear, VTK corner order).
__device__ __forceinline__ float hex_interp(const float v[8], float px, float py, float pz) {
  const float vbf = lerp_lcl(v[0], v[1], px);
  const float vbb = lerp_lcl(v[3], v[2], px);
  const float vtf = lerp_lcl(v[4], v[5], px);
  const float vtb = lerp_lcl(v[7], v[6], px);
  const float vb = lerp_lcl(vbf, vbb, py);
  const float vt = lerp_lcl(vtf, vtb, py);
  return lerp_lcl(vb, vt, pz);
}

// Rectilinear coordinate i on axis d (float32 counting array).
__device__ __forceinline__ float coord(const ExactGeo& g, int d, int i) {
  return g.org[d] + g.h[d] * (float)i;
}

__device__ __forceinline__ float vtx_coord(const ExactGeo& g, int d, int i) {
  return g.morig[d] + g.msp[d] * (float)i;
}

// Field loads. The exact form reads float32; the precision form reads 16-bit.
template <typename FieldT> struct FieldLoad;
template <> struct FieldLoad<float> {
  static __device__ __forceinline__ float ld(const float* __restrict__ f, int64_t i) { return __ldg(f + i); }
};

// SegmentAABB (Intersections.cxx:9-48). The slab ratios are formed in double
// because vtkm::Bounds holds doubles, then stored to float.
__device__ __forceinline__ void segment_aabb_b(const double bmin[3], const double bmax[3], const float a[3],
                                               const float b[3], float& tmin, float& tmax) {
  float dir[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const float len = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  dir[0] = dir[0] / len;
  dir[1] = dir[1] / len;
  dir[2] = dir[2] / len;
  tmin = 0.f;
  tmax = __int_as_float(0x7f800000);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float t0 = (float)((bmin[d] - (double)a[d]) / (double)dir[d]);
    const float t1 = (float)((bmax[d] - (double)a[d]) / (double)dir[d]);
    tmin = mx(tmin, mn(t0, t1));
    tmax = mn(tmax, mx(t0, t1));
  }
  if (tmin < 0.f) tmin = 1e-4f;
  if (tmax > len) tmax = len;
}

__device__ __forceinline__ void segment_aabb(const ExactGeo& g, const float a[3], const float b[3], float& tmin,
                                             float& tmax) {
  segment_aabb_b(g.bmin, g.bmax, a, b, tmin, tmax);
}

// GetEstimateUsingVerticesT of another brick's Phase-1 map at p
// (TransmittanceMap.h:93-112, :200-229; TransmittanceFetcher2 :505-508).
__device__ __forceinline__ float brick_map_opacity(const BrickRef& R, const float p[3]) {
  int c[3];
  float pc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float t = (p[d] - R.morig[d]) * R.minv[d];
    if (t < 0.f) t = 0.f;
    if (t >= (float)(R.pd[d] - 1)) t = (float)(R.pd[d] - 2);
    c[d] = (int)t;
    const float lo = R.morig[d] + R.msp[d] * (float)c[d];
    const float hi = R.morig[d] + R.msp[d] * (float)(c[d] + 1);
    pc[d] = (p[d] - lo) / (hi - lo);
  }
  const unsigned px = (unsigned)R.pd[0], pxy = (unsigned)R.pd[0] * (unsigned)R.pd[1];
  const float* m = R.map + ((unsigned)c[2] * pxy + (unsigned)c[1] * px + (unsigned)c[0]);
  float v[8] = {__ldg(m), __ldg(m + 1), __ldg(m + 1 + px), __ldg(m + px), __ldg(m + pxy), __ldg(m + pxy + 1),
                __ldg(m + pxy + 1 + px), __ldg(m + pxy + px)};
  return hex_interp(v, pc[0], pc[1], pc[2]);
}

// Cross-brick shadow prefix of one vertex ray (the reference's Phases 2-3,
// LightedVolumeRenderer.cxx:968-1235, TransmittanceMap.h:387-453): every other
// brick the segment light->vertex crosses (SegmentAABB hit, glancing hits
// included) contributes its Phase-1 map opacity at the segment's exit point;
// contributions are over-composited in increasing exit distance (HitSort;
// ties by brick id). The over operator on opacity is a product of
// transmittances, so no cross-brick exchange or sort of hit lists is needed.
__device__ __forceinline__ float stitch_prefix(const BrickRef* __restrict__ refs, int nrefs, int self,
                                               const float L[3], const float V[3], const float dir[3]) {
  float ht[kMaxBricks], ho[kMaxBricks];
  int hb[kMaxBricks];
  int nh = 0;
  for (int c = 0; c < nrefs; ++c) {
    if (c == self) continue;
    const BrickRef& R = refs[c];
    float tmin, tmax;
    segment_aabb_b(R.bmin, R.bmax, L, V, tmin, tmax);
    if (!(tmin <= tmax)) continue;
    const float P[3] = {L[0] + dir[0] * tmax, L[1] + dir[1] * tmax, L[2] + dir[2] * tmax};
    const float op = brick_map_opacity(R, P);
    int j = nh++;
    while (j > 0 && (tmax < ht[j - 1] || (tmax == ht[j - 1] && c < hb[j - 1]))) {
      ht[j] = ht[j - 1];
      ho[j] = ho[j - 1];
      hb[j] = hb[j - 1];
      --j;
    }
    ht[j] = tmax;
    ho[j] = op;
    hb[j] = c;
  }
  float o = 0.f;
  for (int i = 0; i < nh; ++i) o = o + (1.f - o) * ho[i];
  return o;
}

// Map vertex position (uniform point coordinates of the opacity map).
__device__ __forceinline__ void map_vertex(const ExactGeo& g, int64_t id, float V[3]) {
  const int64_t px = g.pd[0], pxy = (int64_t)g.pd[0] * g.pd[1];
  const int64_t k = id / pxy;
  const int64_t r = id - k * pxy;
  const int64_t j = r / px;
  const int64_t i = r - j * px;
  V[0] = vtx_coord(g, 0, (int)i);
  V[1] = vtx_coord(g, 1, (int)j);
  V[2] = vtx_coord(g, 2, (int)k);
}

__device__ __forceinline__ void light_origin(const ExactGeo& g, const float V[3], float L[3]) {
  if (g.light_kind == 0) {
    L[0] = g.light[0];
    L[1] = g.light[1];
    L[2] = g.light[2];
  } else {
    L[0] = V[0] - g.light[0] * g.dir_dist;
    L[1] = V[1] - g.light[1] * g.dir_dist;
    L[2] = V[2] - g.light[2] * g.dir_dist;
  }
}

// Entry i of the cell tables: {lo, hi, hi - lo, RN(1 / (hi - lo))} of field
// cell i (axes in order) or, past max_off[0], of map cell i - max_off[0].
__device__ __forceinline__ float4 table_entry(const ExactGeo& g, int i) {
  float lo, hi;
  if (i < g.max_off[0]) {
    const int d = (i >= g.ax_off[2]) ? 2 : (i >= g.ax_off[1] ? 1 : 0);
    const int c = i - g.ax_off[d];
    lo = coord(g, d, c);
    hi = coord(g, d, c + 1);
  } else {
    const int d = (i >= g.max_off[2]) ? 2 : (i >= g.max_off[1] ? 1 : 0);
    const int c = i - g.max_off[d];
    lo = vtx_coord(g, d, c);
    hi = vtx_coord(g, d, c + 1);
  }
  const float w = hi - lo;
  return make_float4(lo, hi, w, 1.f / w);
}

// (int)x for x in [0, 2^23), computed on the FMA pipe instead of the
// conversion unit: 2^23 + x rounded toward zero has the integer part of x in
// its mantissa (its exponent is fixed in [2^23, 2^24)). Callers clamp first, so
// NaN has become 0 before it arrives here.
__device__ __forceinline__ int trunc_small(float x) {
  return __float_as_int(__fadd_rz(x, 8388608.f)) - 0x4B000000;
}

// Correctly rounded division x / w given r = RN(1/w), after Markstein's
// theorem (P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990): with r the
// correctly rounded reciprocal and q a faithful quotient, the residual
// e = x - q*w is exact under fma and RN(q + e*r) is the correctly rounded
// quotient. One refinement makes q faithful, the second rounds it. Valid for
// normal operands whose quotient neither overflows nor underflows, which
// holds for the parametric coordinates here (|x| <= 2w, w a cell width);
// beams_selftest(BEAMS_SELFTEST_DIVISION) checks it against IEEE division.
__device__ __forceinline__ float div_rn_markstein(float x, float w, float r) {
  float q = x * r;
  float e = fmaf(-q, w, x);
  q = fmaf(e, r, q);
  e = fmaf(-q, w, x);
  return fmaf(e, r, q);
}

// Cell tables: T[c] = {coord(c), coord(c+1), coord(c+1)-coord(c), RN(1/(coord(c+1)-coord(c)))}.
//
// Light-march cell search: RectilinearMeshOracle's binary search
// (RectilinearMeshOracle.h:154-176) returns the smallest cell c with
// val <= coord(c+1). The seed (val - org) / h is that cell for counting
// coordinates except within an ulp of a cell face, where the bounded walk
// below settles it. At c == 0 a point on the lower face stays in cell 0 and
// inside the volume val <= coord(cmax+1), so one test per side suffices.
__device__ __forceinline__ int find_cell_bsearch_t(const float4* T, int cmax, float org, float invh,
                                                   float val, float4& e) {
  int c = trunc_small(fminf(fmaxf((val - org) * invh, 0.f), (float)cmax));
  e = T[c];
  if (val <= e.x || val > e.y) {
    while (c > 0 && val <= e.x) e = T[--c];
    while (c < cmax && val > e.y) e = T[++c];
  }
  return c;
}

// The bounded walk that settles a seeded light-march cell guess (the smallest
// c with val <= coord(c+1), RectilinearMeshOracle.h:154-176), for the rare
// sample within an ulp of a cell face; kept out of line (noinline) so that the
// march's common path carries none of its code.
static __device__ __noinline__ int walk_cell_bsearch(const float4* T, int cmax, float val, int c) {
  float4 e = T[c];
  while (c > 0 && val <= e.x) e = T[--c];
  while (c < cmax && val > e.y) e = T[++c];
  return c;
}
static __device__ __noinline__ int3 walk_cells_bsearch(const float4* T0, const float4* T1, const float4* T2, int m0,
                                                       int m1, int m2, float v0, float v1, float v2, int c0, int c1,
                                                       int c2) {
  return make_int3(walk_cell_bsearch(T0, m0, v0, c0), walk_cell_bsearch(T1, m1, v1, c1),
                   walk_cell_bsearch(T2, m2, v2, c2));
}

// Searches for explicit (non-uniform) rectilinear coordinates, where no seed
// from a uniform spacing is close: the light march's binary search
// (RectilinearMeshOracle.h:154-176, smallest c with val <= coord(c+1)) and the
// view march's cell lookup (the unique c with coord(c) <= p < coord(c+1) that
// RectilinearLocator::LocateCell walks to, LightedVolumeRenderer.cxx:119-165),
// both over the shared-memory cell table.
__device__ __forceinline__ int find_cell_bsearch_rect(const float4* T, int cmax, float val, float4& e) {
  int lo = 0, hi = cmax;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (val <= T[mid].y) hi = mid;
    else lo = mid + 1;
  }
  e = T[lo];
  return lo;
}
__device__ __forceinline__ int find_cell_walk_rect(const float4* T, int cmax, float p, float4& e) {
  int lo = 0, hi = cmax;  // largest c with coord(c) <= p
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (T[mid].x <= p) lo = mid;
    else hi = mid - 1;
  }
  e = T[lo];
  return lo;
}

// View-march cell search: RectilinearLocator::LocateCell (LightedVolumeRenderer.cxx:119-165)
// walks to the unique cell with coord(c) <= p < coord(c+1).
__device__ __forceinline__ int find_cell_walk_t(const float4* T, int cmax, float org, float invh, float p,
                                                float4& e) {
  int c = trunc_small(fminf(fmaxf((p - org) * invh, 0.f), (float)cmax));
  e = T[c];
  if (p < e.x || p >= e.y) {
    while (c > 0 && p < e.x) e = T[--c];
    while (c < cmax && p >= e.y) e = T[++c];
  }
  return c;
}

// The view march's walk (the unique c with coord(c) <= p < coord(c+1)) that
// settles seeded guesses off by a face, out of line like walk_cells_bsearch.
static __device__ __noinline__ int walk_cell_view(const float4* T, int cmax, float p, int c) {
  float4 e = T[c];
  while (c > 0 && p < e.x) e = T[--c];
  while (c < cmax && p >= e.y) e = T[++c];
  return c;
}
static __device__ __noinline__ int3 walk_cells_view(const float4* T0, const float4* T1, const float4* T2, int m0,
                                                    int m1, int m2, float v0, float v1, float v2, int c0, int c1,
                                                    int c2) {
  return make_int3(walk_cell_view(T0, m0, v0, c0), walk_cell_view(T1, m1, v1, c1), walk_cell_view(T2, m2, v2, c2));
}

// The view march's cell location on a uniform grid when a sample leaves its
// cell (RectilinearLocator::LocateCell, LightedVolumeRenderer.cxx:119-165):
// seeded guesses, one branch testing the three axes, the rare walk out of line.
// On a max face the cell is the last one and inv[k] is left as it was (the
// reference keeps the previous invSpacing there); bl[k] = the cell's lower
// coordinate.
__device__ __forceinline__ void locate_view_cell(const ExactGeo& g, const float4* s_tab, const float p[3], int c[3],
                                                 float inv[3], float bl[3]) {
  float4 e[3];
  bool off = false;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    c[k] = trunc_small(fminf(fmaxf((p[k] - g.org[k]) * g.invh[k], 0.f), (float)(g.n[k] - 2)));
    e[k] = s_tab[g.ax_off[k] + c[k]];
    off = off | (p[k] < e[k].x) | (p[k] >= e[k].y);
  }
  if (off) {
    const int3 cc = walk_cells_view(s_tab + g.ax_off[0], s_tab + g.ax_off[1], s_tab + g.ax_off[2], g.n[0] - 2,
                                    g.n[1] - 2, g.n[2] - 2, p[0], p[1], p[2], c[0], c[1], c[2]);
    c[0] = cc.x;
    c[1] = cc.y;
    c[2] = cc.z;
#pragma unroll
    for (int k = 0; k < 3; ++k) e[k] = s_tab[g.ax_off[k] + c[k]];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (p[k] == g.maxp[k]) {
      c[k] = g.n[k] - 2;
      e[k] = s_tab[g.ax_off[k] + c[k]];
    } else {
      inv[k] = e[k].w;  // 1.f / (coord(c+1) - coord(c)), IEEE
    }
    bl[k] = e[k].x;
  }
}

// TF index of the light march (TransmittanceMap.h:322-326): truncate, clamp to
// [0, n1]; saturating, NaN -> 0. Clamping in float first gives the same index:
// (-1, 0) truncates to 0 either way and [n1, n1+1) to n1.
__device__ __forceinline__ int tf_index_clamped(float fi, int n1) {
  return trunc_small(fminf(fmaxf(fi, 0.f), (float)n1));
}
// The same with the top index given as a float (n1f = (float)n1).
__device__ __forceinline__ int tf_index_clamped_f(float fi, float n1f) {
  return trunc_small(fminf(fmaxf(fi, 0.f), n1f));
}

// Pinhole camera ray through pixel centre (x, y).
__device__ __forceinline__ void camera_ray(const ExactGeo& g, int x, int y, float o[3], float d[3]) {
  const float sx = ((float)x + 0.5f) * g.kx - g.cx;
  const float sy = ((float)y + 0.5f) * g.ky - g.cy;
  float v[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = (g.cf[k] + sx * g.cr[k]) + sy * g.cu[k];
  const float len = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d[k] = v[k] / len;
    o[k] = g.cam_pos[k];
  }
}

// CalcRayStart (LightedVolumeRenderer.cxx:644-718) in S = float (the reference)
// or S = double (t_enter/t_exit set up in FP64, then rounded to float).
template <typename S>
__device__ __forceinline__ bool slab_t(const S o[3], const S d[3], const double bmin[3],
                                       const double bmax[3], S& minD, S& maxD) {
  S lo[3], hi[3];
  const S eps = (sizeof(S) == 4) ? (S)1e-8f : (S)1e-8;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const S inv = S(1) / ((fabs(d[k]) < eps) ? eps : d[k]);
    const S od = o[k] * inv;
    lo[k] = (S)bmin[k] * inv - od;
    hi[k] = (S)bmax[k] * inv - od;
  }
  minD = mx(mx(mx(mn(lo[1], hi[1]), mn(lo[0], hi[0])), mn(lo[2], hi[2])), minD);
  const S exitD = mn(mn(mx(lo[1], hi[1]), mx(lo[0], hi[0])), mx(lo[2], hi[2]));
  maxD = mn(maxD, exitD);
  return !(maxD < minD);
}

// The ray enters with MinDistance 0 and MaxDistance +inf, or the canvas depth
// limit of its pixel when one is set; the slab test narrows both.
__device__ __forceinline__ bool ray_setup(const ExactGeo& g, int x, int y, float o[3], float d[3],
                                          float& minD, float& maxD) {
  camera_ray(g, x, y, o, d);
  const float lim = g.ray_max ? __ldg(g.ray_max + (size_t)y * g.width + x) : __int_as_float(0x7f800000);
  if (g.slab_fp64) {
    const double od[3] = {(double)o[0], (double)o[1], (double)o[2]};
    const double dd[3] = {(double)d[0], (double)d[1], (double)d[2]};
    double lo = 0.0, hi = (double)lim;
    const bool hit = slab_t<double>(od, dd, g.bmin, g.bmax, lo, hi);
    minD = (float)lo;
    maxD = (float)hi;
    return hit;
  }
  minD = 0.f;
  maxD = lim;
  return slab_t<float>(o, d, g.bmin, g.bmax, minD, maxD);
}

__device__ __forceinline__ bool inside_vol(const ExactGeo& g, const float p[3]) {
  return !(p[0] < g.minp[0] || p[0] > g.maxp[0] || p[1] < g.minp[1] || p[1] > g.maxp[1] ||
           p[2] < g.minp[2] || p[2] > g.maxp[2]);
}

template <typename MapT> __device__ __forceinline__ float ld_map(const MapT* p);
template <> __device__ __forceinline__ float ld_map<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_map<__half>(const __half* p) { return __half2float(__ldg(p)); }

// TransmittanceLocator::LocateCell + GetEstimateUsingVerticesT
// (TransmittanceMap.h:93-112, :200-229): the map value interpolated at p
// (opacity in the exact form, transmittance in the precision form).
// MT = map cell tables.
template <typename MapT>
__device__ __forceinline__ float map_interp_t(const ExactGeo& g, const float4* MT, const MapT* __restrict__ map,
                                              const float p[3]) {
  int c[3];
  float pc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // the reference clamps t to [0, pd-2] when t >= pd-1 and truncates; the
    // cell is the same as truncating min(max(t, 0), pd-2)
    const float t = (p[d] - g.morig[d]) * g.minv[d];
    c[d] = trunc_small(fminf(fmaxf(t, 0.f), (float)(g.pd[d] - 2)));
    const float4 e = MT[g.max_off[d] + c[d]];
    pc[d] = div_rn_markstein(p[d] - e.x, e.z, e.w);
  }
  const unsigned px = (unsigned)g.pd[0], pxy = (unsigned)g.pd[0] * (unsigned)g.pd[1];
  const MapT* m = map + ((unsigned)c[2] * pxy + (unsigned)c[1] * px + (unsigned)c[0]);
  float v[8];
  v[0] = ld_map(m);
  v[1] = ld_map(m + 1);
  v[2] = ld_map(m + 1 + px);
  v[3] = ld_map(m + px);
  v[4] = ld_map(m + pxy);
  v[5] = ld_map(m + pxy + 1);
  v[6] = ld_map(m + pxy + 1 + px);
  v[7] = ld_map(m + pxy + px);
  return hex_interp(v, pc[0], pc[1], pc[2]);
}

// The multi-light shading term at p: sum over the maps of (1 - opacity_l) *
// light_colors[l], in light order. The cell and parametric coordinates are the
// same for every map (one map grid), so they are located once.
__device__ __forceinline__ void map_light_sum(const ExactGeo& g, const float4* MT, const float* __restrict__ map,
                                              const float p[3], float est[3]) {
  int c[3];
  float pc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float t = (p[d] - g.morig[d]) * g.minv[d];
    c[d] = trunc_small(fminf(fmaxf(t, 0.f), (float)(g.pd[d] - 2)));
    const float4 e = MT[g.max_off[d] + c[d]];
    pc[d] = div_rn_markstein(p[d] - e.x, e.z, e.w);
  }
  const unsigned px = (unsigned)g.pd[0], pxy = (unsigned)g.pd[0] * (unsigned)g.pd[1];
  const size_t nv = (size_t)pxy * (unsigned)g.pd[2];
  const float* m = map + ((unsigned)c[2] * pxy + (unsigned)c[1] * px + (unsigned)c[0]);
  for (int l = 0; l < g.n_lights; ++l, m += nv) {
    const float v[8] = {__ldg(m), __ldg(m + 1), __ldg(m + 1 + px), __ldg(m + px),
                        __ldg(m + pxy), __ldg(m + pxy + 1), __ldg(m + pxy + 1 + px), __ldg(m + pxy + px)};
    const float tr = 1.f - hex_interp(v, pc[0], pc[1], pc[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float t = tr * g.light_colors[l][d];
      est[d] = (l == 0) ? t : est[d] + t;
    }
  }
}

// Shared-memory form of the light-aligned brick order for bricks of 2^bl
// vertices per edge: {nb_w, nb_u, nb_v, axis_w, axis_u, axis_v, shear_u, shear_v}.
__device__ __forceinline__ void brick_order_setup(const ExactGeo& g, int bl, int* s_bo) {
  int nb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) nb[d] = (g.pd[d] + (1 << bl) - 1) >> bl;
  for (int k = 0; k < 3; ++k) {
    s_bo[k] = nb[g.bo_axis[k]];
    s_bo[3 + k] = g.bo_axis[k];
  }
  s_bo[6] = g.bo_shear[0];
  s_bo[7] = g.bo_shear[1];
}

// Brick bi of that order -> brick coordinates. Read through volatile loads so
// the parameters stay in shared memory rather than in registers.
__device__ __forceinline__ void pencil_brick(int bi, const int* s_bo, int& bx, int& by, int& bz) {
  const volatile int* q = s_bo;
  const int nw = q[0], nu = q[1], nv = q[2];
  const int w = bi % nw, pe = bi / nw;
  int u = (pe % nu + ((w * q[6]) >> 16)) % nu;
  int v = (pe / nu + ((w * q[7]) >> 16)) % nv;
  u += (u < 0) ? nu : 0;
  v += (v < 0) ? nv : 0;
  const int aw = q[3], au = q[4];
  bx = aw == 0 ? w : (au == 0 ? u : v);
  by = aw == 1 ? w : (au == 1 ? u : v);
  bz = aw == 2 ? w : (au == 2 ? u : v);
}

// Quad layout of a point field: Q[z][y][x] = {f(x,y,z), f(x+1,y,z), f(x,y+1,z),
// f(x+1,y+1,z)} for x < nx-1, y < ny-1, so one cell is two 16-byte loads
// (z and z+1). VTK corner order 0..7 = lo.x lo.y lo.w lo.z hi.x hi.y hi.w hi.z.
// Cell (x, y, z) is entry qi = z qz + y qx + x; strides() gives qx and qz.
// FieldF32 reads the float32 field itself (x fastest, eight scalar loads per
// cell; qx = nx, qz = nx ny): the allocation-free entry point's layout.
template <typename Q> struct QuadLoad;
struct FieldF32 { float v; };
__device__ __forceinline__ void quad_strides(const ExactGeo& g, unsigned& qx, unsigned& qz) {
  qx = (unsigned)(g.n[0] - 1);
  qz = qx * (unsigned)(g.n[1] - 1);
}
template <> struct QuadLoad<FieldF32> {
  static __device__ __forceinline__ void strides(const ExactGeo& g, unsigned& qx, unsigned& qz) {
    qx = (unsigned)g.n[0];
    qz = qx * (unsigned)g.n[1];
  }
  static __device__ __forceinline__ void cell(const FieldF32* __restrict__ q, unsigned qi, unsigned qx, unsigned qz,
                                              float v[8]) {
    const float* f = reinterpret_cast<const float*>(q) + qi;
    v[0] = __ldg(f);
    v[1] = __ldg(f + 1);
    v[2] = __ldg(f + qx + 1);
    v[3] = __ldg(f + qx);
    v[4] = __ldg(f + qz);
    v[5] = __ldg(f + qz + 1);
    v[6] = __ldg(f + qz + qx + 1);
    v[7] = __ldg(f + qz + qx);
  }
};
// 16-bit quads (precision form): four binary16 or bfloat16 values in 8 bytes.
struct __align__(8) QuadBF16 { unsigned short v[4]; };
struct __align__(8) QuadF16 { unsigned short v[4]; };
__device__ __forceinline__ float bf16_lo(unsigned u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(unsigned u) { return __uint_as_float(u & 0xffff0000u); }
__device__ __forceinline__ float f16_lo(unsigned u) { return __half2float(__ushort_as_half((unsigned short)(u & 0xffffu))); }
__device__ __forceinline__ float f16_hi(unsigned u) { return __half2float(__ushort_as_half((unsigned short)(u >> 16))); }
template <> struct QuadLoad<QuadBF16> {
  static __device__ __forceinline__ void strides(const ExactGeo& g, unsigned& qx, unsigned& qz) { quad_strides(g, qx, qz); }
  static __device__ __forceinline__ void cell(const QuadBF16* __restrict__ q, unsigned qi, unsigned, unsigned qz, float v[8]) {
    const uint2 a = __ldg((const uint2*)(q + qi));
    const uint2 b = __ldg((const uint2*)(q + qi + qz));
    v[0] = bf16_lo(a.x); v[1] = bf16_hi(a.x); v[2] = bf16_hi(a.y); v[3] = bf16_lo(a.y);
    v[4] = bf16_lo(b.x); v[5] = bf16_hi(b.x); v[6] = bf16_hi(b.y); v[7] = bf16_lo(b.y);
  }
};
template <> struct QuadLoad<QuadF16> {
  static __device__ __forceinline__ void strides(const ExactGeo& g, unsigned& qx, unsigned& qz) { quad_strides(g, qx, qz); }
  static __device__ __forceinline__ void cell(const QuadF16* __restrict__ q, unsigned qi, unsigned, unsigned qz, float v[8]) {
    const uint2 a = __ldg((const uint2*)(q + qi));
    const uint2 b = __ldg((const uint2*)(q + qi + qz));
    v[0] = f16_lo(a.x); v[1] = f16_hi(a.x); v[2] = f16_hi(a.y); v[3] = f16_lo(a.y);
    v[4] = f16_lo(b.x); v[5] = f16_hi(b.x); v[6] = f16_hi(b.y); v[7] = f16_lo(b.y);
  }
};
template <> struct QuadLoad<float4> {
  static __device__ __forceinline__ void strides(const ExactGeo& g, unsigned& qx, unsigned& qz) { quad_strides(g, qx, qz); }
  static __device__ __forceinline__ void cell(const float4* __restrict__ q, unsigned qi, unsigned, unsigned qz, float v[8]) {
    const float4 a = __ldg(q + qi);
    const float4 b = __ldg(q + qi + qz);
    v[0] = a.x; v[1] = a.y; v[2] = a.w; v[3] = a.z;
    v[4] = b.x; v[5] = b.y; v[6] = b.w; v[7] = b.z;
  }
};

// Whether the macro-cell holding p may hold a non-zero TF alpha. The macro
// index comes from the approximate cell (p - org) / h; the occupancy of macro
// m covers cells [8m - 1, 8m + 8], so a cell search off by one stays covered.
__device__ __forceinline__ bool occupied(const ExactGeo& g, const unsigned char* __restrict__ occ, const float p[3]) {
  int m[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float f = fminf(fmaxf((p[d] - g.org[d]) * g.invh[d], 0.f), (float)(g.n[d] - 2));
    m[d] = trunc_small(f) >> kMacroLog2;
  }
  return __ldg(occ + ((size_t)m[2] * g.occ_n[1] + m[1]) * g.occ_n[0] + m[0]) != 0;
}

// The light march of TransmittanceMap.h:279-332 from L to an arbitrary point P
// (K1 runs it to map vertices): opacity accumulated over the same sample
// sequence. T0..T2: field cell tables; s_a: TF alpha / max alpha.
__device__ __forceinline__ float point_opacity(const ExactGeo& g, const float4* __restrict__ quads, const float4* T0,
                                               const float4* T1, const float4* T2, const float* s_a, const float L[3],
                                               const float P[3]) {
  const float v[3] = {P[0] - L[0], P[1] - L[1], P[2] - L[2]};
  const float rs = 1.f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const float dir[3] = {v[0] * rs, v[1] * rs, v[2] * rs};
  float tmin, tmax;
  segment_aabb(g, L, P, tmin, tmax);
  const float st[3] = {L[0] + tmin * dir[0], L[1] + tmin * dir[1], L[2] + tmin * dir[2]};
  float s[3] = {st[0], st[1], st[2]};
  const float len2 = (tmax - tmin) * (tmax - tmin);
  const int n1 = g.tf_n - 1;
  const unsigned qx = (unsigned)(g.n[0] - 1), qz = (unsigned)(g.n[0] - 1) * (unsigned)(g.n[1] - 1);
  float o = 0.f;
  for (int b = g.light_budget; b > 0; --b) {
    const float q0 = s[0] - st[0], q1 = s[1] - st[1], q2 = s[2] - st[2];
    if (!(q0 * q0 + q1 * q1 + q2 * q2 <= len2)) break;
    s[0] = s[0] + g.step * dir[0];
    s[1] = s[1] + g.step * dir[1];
    s[2] = s[2] + g.step * dir[2];
    if (!inside_vol(g, s)) break;
    float4 e0, e1, e2;
    const int c0 = find_cell_bsearch_t(T0, g.n[0] - 2, g.org[0], g.invh[0], s[0], e0);
    const int c1 = find_cell_bsearch_t(T1, g.n[1] - 2, g.org[1], g.invh[1], s[1], e1);
    const int c2 = find_cell_bsearch_t(T2, g.n[2] - 2, g.org[2], g.invh[2], s[2], e2);
    float vals[8];
    QuadLoad<float4>::cell(quads, (unsigned)c2 * qz + (unsigned)c1 * qx + (unsigned)c0, qx, qz, vals);
    float scalar = hex_interp(vals, div_rn_markstein(s[0] - e0.x, e0.z, e0.w), div_rn_markstein(s[1] - e1.x, e1.z, e1.w),
                              div_rn_markstein(s[2] - e2.x, e2.z, e2.w));
    scalar = (scalar - g.min_scalar) * g.inv_delta;
    o = o + (1.f - o) * s_a[tf_index_clamped(scalar * (float)n1, n1)];
    if (o == 1.f) break;
  }
  return o;
}

// Warp-aggregated counter increment (one atomic per warp). Must be reached by
// all 32 lanes of the warp (kernels keep out-of-range lanes alive with v = 0);
// blocks are one-dimensional.
__device__ __forceinline__ void warp_add(unsigned long long* dst, unsigned v) {
  const unsigned s = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(dst, (unsigned long long)s);
}

}  // namespace beams
