// beams_oracle.cpp — CPU restatement of the Beams lighted volume renderer.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline). The product
// library never links or calls this file.
//
// Each routine cites the reference lines it restates (paths within
// goodbadwolf/pilot). The template parameter T is float for the
// reference-faithful mode and double for the FP64 yardstick. The file must be
// compiled with -ffp-contract=off so that a*b+c stays two roundings, as in the
// reference's x86-64 build (no FMA target flags).
//
// VTK-m internals the reference calls, restated from their published
// definitions (VTK-m 1.9 / lcl); parity at these points is unpinned:
//  * vtkm::exec::CellInterpolate on a hexahedron = lcl trilinear in VTK corner
//    order with lerp(a,b,t) = fma(t, b, fma(-t, a, a)).
//  * WorldCoordinatesToParametricCoordinates on an axis-aligned hexahedron
//    = (p - min) / (max - min), componentwise.
//  * vtkm::Normal(v) = v * (1 / sqrt(dot(v,v))); vtkm::Magnitude = sqrt(dot).
//  * vtkm::Min/Max = std::min/std::max; vtkm::Clamp(x,lo,hi) = x<lo?lo:(x>hi?hi:x).
//  * ArrayHandleCounting / uniform point coordinates: origin + spacing * i.
//  * raytracing::Camera::CreateRays is replaced by the pinhole camera below
//    (rays through pixel centres, MinDistance 0, MaxDistance +inf).
//
// Deviations from the reference, each where the reference would hang or return
// NaN (the GPU library does the same):
//  * A view sample whose transfer-function index falls outside the table is
//    skipped but the ray still advances (LightedVolumeRenderer.cxx:456-459
//    `continue`s without advancing, which never terminates).
//  * Marches carry an iteration budget derived from the segment length, so a
//    step absorbed by float rounding cannot spin forever.
//  * A transfer function whose alphas are all 0 gives a light-march opacity of
//    0 instead of 0/0 (TransmittanceMap.h:329 divides by the max alpha).
//  * The TF index of the light march and of the cell-field march saturates for
//    |value| >= 2^63 instead of taking x86's indefinite-integer value.

#include "beams_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename T> inline T mn(T a, T b) { return (b < a) ? b : a; }
template <typename T> inline T mx(T a, T b) { return (a < b) ? b : a; }
template <typename T> inline T clamp01(T x) { return x < T(0) ? T(0) : (x > T(1) ? T(1) : x); }

inline float lerp(float a, float b, float t) { return std::fma(t, b, std::fma(-t, a, a)); }
inline double lerp(double a, double b, double t) { return std::fma(t, b, std::fma(-t, a, a)); }

// lcl Hexahedron interpolate: x-lerps of edges (0,1) (3,2) (4,5) (7,6), then y, then z.
template <typename T>
inline T hex_interp(const T v[8], T px, T py, T pz) {
  T vbf = lerp(v[0], v[1], px);
  T vbb = lerp(v[3], v[2], px);
  T vtf = lerp(v[4], v[5], px);
  T vtb = lerp(v[7], v[6], px);
  T vb = lerp(vbf, vbb, py);
  T vt = lerp(vtf, vtb, py);
  return lerp(vb, vt, pz);
}

template <typename T>
struct Geo {
  int n[3];
  std::vector<T> C[3];          // rectilinear coordinates (Spheres.cxx:144-156)
  T minp[3], maxp[3];
  double bmin[3], bmax[3];      // vtkm::Bounds of the coordinate system (double)
  T min_scalar, inv_delta;      // LightedVolumeRenderer.cxx:331-334, TransmittanceMap.h:254-261
  std::vector<T> tf;
  int tf_n;
  T max_alpha;                  // GetMaxAlpha, TransmittanceMap.h:515-525
  int pd[3];                    // map point dims M+1
  T morig[3], msp[3], minv[3];  // CreateDataSetForOpacityMap, TransmittanceMap.h:550-563
  T light_color[3];             // Color * Intensity, LightedVolumeRenderer.cxx:840
  // multi-light extension (off in the reference, which shades with Locations[0]
  // only, LightedVolumeRenderer.cxx:836-840): n_lights maps of map_nv vertices
  // stacked in light order, light l shaded with lcols[3l..3l+2]
  int n_lights = 1;
  int64_t map_nv = 0;
  std::vector<T> lcols;
  const float* ray_max = nullptr;  // canvas depth clipping, per pixel (width * height)
  T extent_mag;                 // BoundsMagnitude, Math.h:13-21
  T sd, mesh_eps, step, cutoff;
  int light_kind;
  T light[3];                   // point position or normalised travel direction
  T dir_dist;                   // directional light: origin placed this far back
  const float* field;
  int use_map;
  int slab_fp64;
  int precision;
  std::vector<T> tau;  // -ln(1 - a_i) per TF entry (precision form)
  // camera
  T cam_pos[3], cf[3], cr[3], cu[3], kx, cx, ky, cy;
  int width, height;
};

template <typename T>
void build_geo(const oracle_scene* s, Geo<T>& g) {
  for (int d = 0; d < 3; ++d) {
    g.n[d] = s->dims[d];
    g.C[d].resize(s->dims[d]);
    const T o = (T)s->origin[d], h = (T)s->spacing[d];
    for (int i = 0; i < s->dims[d]; ++i) g.C[d][i] = s->coords[d] ? (T)s->coords[d][i] : o + h * (T)i;
    g.minp[d] = g.C[d][0];
    g.maxp[d] = g.C[d][s->dims[d] - 1];
    g.bmin[d] = (double)g.C[d][0];
    g.bmax[d] = (double)g.C[d][s->dims[d] - 1];
  }
  const T fmin = (T)s->range[0], fmax = (T)s->range[1];
  g.min_scalar = fmin;
  g.inv_delta = ((fmax - fmin) != T(0)) ? T(1) / (fmax - fmin) : fmin;
  g.tf_n = s->tf_n;
  g.tf.resize(4 * (size_t)s->tf_n);
  g.max_alpha = T(0);
  for (int i = 0; i < s->tf_n; ++i) {
    for (int c = 0; c < 4; ++c) g.tf[4 * i + c] = (T)s->tf[4 * i + c];
    g.max_alpha = mx(g.max_alpha, g.tf[4 * i + 3]);
  }
  T ext[3];
  for (int d = 0; d < 3; ++d) ext[d] = (T)(g.bmax[d] - g.bmin[d]);
  g.extent_mag = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]);
  for (int d = 0; d < 3; ++d) {
    g.pd[d] = s->map_m[d] + 1;
    g.morig[d] = (T)g.bmin[d];
    g.msp[d] = ext[d] / (T)s->map_m[d];
    g.minv[d] = T(1) / g.msp[d];
    g.light_color[d] = (T)s->light_color[d] * (T)s->light_intensity;
  }
  g.sd = (s->sample_distance > 0.f) ? (T)s->sample_distance : g.extent_mag / (T)200;
  g.mesh_eps = g.extent_mag * (T)0.0001f;
  if (sizeof(T) == 8) g.mesh_eps = g.extent_mag * (T)0.0001;
  g.step = g.extent_mag / (T)s->light_steps;
  g.cutoff = (T)s->alpha_cutoff;
  g.light_kind = s->light_kind;
  if (s->light_kind == 0) {
    for (int d = 0; d < 3; ++d) g.light[d] = (T)s->light[d];
  } else {
    const double* L = s->light;
    const double len = std::sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
    for (int d = 0; d < 3; ++d) g.light[d] = (T)(L[d] / len);
  }
  g.dir_dist = T(2) * g.extent_mag;
  g.field = s->field;
  g.use_map = s->use_map;
  g.slab_fp64 = s->slab_fp64;
  g.precision = s->precision;
  g.ray_max = s->ray_max;
  g.tau.resize(s->tf_n);
  {
    float ma = 0.f;  // float32 max alpha, as the device derives it
    for (int i = 0; i < s->tf_n; ++i) ma = (ma < s->tf[4 * i + 3]) ? s->tf[4 * i + 3] : ma;
    for (int i = 0; i < s->tf_n; ++i) {
      // a_i = alpha / max alpha in float, then -ln(1 - a_i) in double, stored as float.
      const float a = (ma > 0.f) ? s->tf[4 * i + 3] / ma : 0.f;
      g.tau[i] = (a >= 1.f) ? std::numeric_limits<T>::infinity() : (T)(float)(-std::log1p(-(double)a));
    }
  }
  // Pinhole camera set up in double; per-pixel arithmetic in T.
  double f[3], r[3], u[3];
  for (int d = 0; d < 3; ++d) f[d] = s->cam_look[d] - s->cam_pos[d];
  double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (int d = 0; d < 3; ++d) f[d] /= fl;
  const double* up = s->cam_up;
  r[0] = f[1] * up[2] - f[2] * up[1];
  r[1] = f[2] * up[0] - f[0] * up[2];
  r[2] = f[0] * up[1] - f[1] * up[0];
  double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  for (int d = 0; d < 3; ++d) r[d] /= rl;
  u[0] = r[1] * f[2] - r[2] * f[1];
  u[1] = r[2] * f[0] - r[0] * f[2];
  u[2] = r[0] * f[1] - r[1] * f[0];
  const double th = std::tan(s->fov_y_deg * M_PI / 360.0);
  const double aspect = (double)s->width / (double)s->height;
  for (int d = 0; d < 3; ++d) {
    g.cam_pos[d] = (T)s->cam_pos[d];
    g.cf[d] = (T)f[d];
    g.cr[d] = (T)r[d];
    g.cu[d] = (T)u[d];
  }
  g.kx = (T)(2.0 * th * aspect / s->width);
  g.cx = (T)(th * aspect);
  g.ky = (T)(2.0 * th / s->height);
  g.cy = (T)th;
  g.width = s->width;
  g.height = s->height;
}

// ---- light march (TransmittanceMap.h:239-340, Intersections.cxx:9-48,
//      RectilinearMeshOracle.h:139-195, LightRayOperations.h:32-43) -------------

// SegmentAABB: the slab ratios are formed in double because vtkm::Bounds holds
// doubles (Intersections.cxx:27-40), then stored to T.
template <typename T>
void segment_aabb(const T a[3], const T b[3], const Geo<T>& g, T& tmin, T& tmax) {
  T dir[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const T len = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  for (int d = 0; d < 3; ++d) dir[d] = dir[d] / len;
  tmin = T(0);
  tmax = std::numeric_limits<T>::infinity();
  for (int d = 0; d < 3; ++d) {
    const T t0 = (T)((g.bmin[d] - (double)a[d]) / (double)dir[d]);
    const T t1 = (T)((g.bmax[d] - (double)a[d]) / (double)dir[d]);
    tmin = mx(tmin, mn(t0, t1));
    tmax = mn(tmax, mx(t0, t1));
  }
  if (tmin < T(0)) tmin = (T)1e-4f;
  if (tmax > len) tmax = len;
}

template <typename T>
inline T field_at(const Geo<T>& g, int64_t j) {
  const int64_t nv = (int64_t)g.n[0] * g.n[1] * g.n[2];
  if (j >= nv) j = nv - 1;
  return (T)g.field[j];
}

// Marches from light origin L to destination P; returns the accumulated opacity.
template <typename T>
T light_march_point(const Geo<T>& g, const T L[3], const T P[3], uint64_t& nsamples, T o0 = T(0)) {
  T v[3] = {P[0] - L[0], P[1] - L[1], P[2] - L[2]};
  const T rs = T(1) / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const T dir[3] = {v[0] * rs, v[1] * rs, v[2] * rs};
  T tmin, tmax;
  segment_aabb(L, P, g, tmin, tmax);
  const T start[3] = {L[0] + tmin * dir[0], L[1] + tmin * dir[1], L[2] + tmin * dir[2]};
  T sl[3] = {start[0], start[1], start[2]};
  const T len2 = (tmax - tmin) * (tmax - tmin);
  const int N1 = g.tf_n - 1;
  T o = o0;
  // Budget: the loop below advances by step each iteration inside the box.
  int budget = (int)(g.extent_mag / g.step) + 8;
  while (budget-- > 0) {
    const T q[3] = {sl[0] - start[0], sl[1] - start[1], sl[2] - start[2]};
    if (!(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= len2)) break;
    for (int d = 0; d < 3; ++d) sl[d] = sl[d] + g.step * dir[d];
    bool inside = true;
    for (int d = 0; d < 3; ++d)
      if (sl[d] < g.minp[d] || sl[d] > g.maxp[d]) inside = false;
    if (!inside) break;
    int c[3];
    T pc[3];
    for (int d = 0; d < 3; ++d) {
      int lo = 0, hi = g.n[d] - 2;
      const T val = sl[d];
      while (lo <= hi) {
        const int mid = (lo + hi) / 2;
        if (val <= g.C[d][mid + 1]) hi = mid - 1;
        else lo = mid + 1;
      }
      c[d] = lo;
      int j = lo + 1;
      if (j >= g.n[d]) j = lo;
      const T mnp = g.C[d][lo], mxp = g.C[d][j];
      pc[d] = (val - mnp) / (mxp - mnp);
    }
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    const int64_t i0 = (int64_t)c[2] * nxy + (int64_t)c[1] * nx + c[0];
    T vals[8];
    vals[0] = field_at(g, i0);
    vals[1] = field_at(g, i0 + 1);
    vals[2] = field_at(g, i0 + 1 + nx);
    vals[3] = field_at(g, i0 + nx);
    vals[4] = field_at(g, i0 + nxy);
    vals[5] = field_at(g, i0 + nxy + 1);
    vals[6] = field_at(g, i0 + nxy + 1 + nx);
    vals[7] = field_at(g, i0 + nxy + nx);
    T scalar = hex_interp(vals, pc[0], pc[1], pc[2]);
    scalar = (scalar - g.min_scalar) * g.inv_delta;
    const T fi = scalar * (T)N1;
    int idx;
    if (fi > T(-1) && fi < (T)(N1 + 1)) idx = (int)(int64_t)fi;
    else idx = (fi >= (T)(N1 + 1)) ? N1 : 0;
    if (idx < 0) idx = 0;
    if (idx > N1) idx = N1;
    const T a = (g.max_alpha > T(0)) ? g.tf[4 * idx + 3] / g.max_alpha : T(0);
    o = o + (T(1) - o) * a;
    ++nsamples;
  }
  return o;
}

// Precision form of the light march: same samples as light_march_point, but
// the opacity is accumulated as optical depth tau = sum -ln(1 - a_i) with Kahan
// compensation over the non-zero terms (a sample of alpha 0 adds nothing, not
// even its compensation step), a_i = 1 cuts the ray (T = 0), and the result is
// the transmittance exp(-tau) rounded to IEEE binary16 (returned as float).
template <typename T>
T light_march_point_tau(const Geo<T>& g, const T L[3], const T P[3], uint64_t& nsamples) {
  T v[3] = {P[0] - L[0], P[1] - L[1], P[2] - L[2]};
  const T rs = T(1) / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const T dir[3] = {v[0] * rs, v[1] * rs, v[2] * rs};
  T tmin, tmax;
  segment_aabb(L, P, g, tmin, tmax);
  const T start[3] = {L[0] + tmin * dir[0], L[1] + tmin * dir[1], L[2] + tmin * dir[2]};
  T sl[3] = {start[0], start[1], start[2]};
  const T len2 = (tmax - tmin) * (tmax - tmin);
  const int N1 = g.tf_n - 1;
  float sum = 0.f, comp = 0.f;
  bool cut = false;
  int budget = (int)(g.extent_mag / g.step) + 8;
  while (budget-- > 0) {
    const T q[3] = {sl[0] - start[0], sl[1] - start[1], sl[2] - start[2]};
    if (!(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= len2)) break;
    for (int d = 0; d < 3; ++d) sl[d] = sl[d] + g.step * dir[d];
    bool inside = true;
    for (int d = 0; d < 3; ++d)
      if (sl[d] < g.minp[d] || sl[d] > g.maxp[d]) inside = false;
    if (!inside) break;
    T pc[3];
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int lo = 0, hi = g.n[d] - 2;
      const T val = sl[d];
      while (lo <= hi) {
        const int mid = (lo + hi) / 2;
        if (val <= g.C[d][mid + 1]) hi = mid - 1;
        else lo = mid + 1;
      }
      c[d] = lo;
      pc[d] = (val - g.C[d][lo]) / (g.C[d][lo + 1] - g.C[d][lo]);
    }
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    const int64_t i0 = (int64_t)c[2] * nxy + (int64_t)c[1] * nx + c[0];
    T vals[8] = {field_at(g, i0), field_at(g, i0 + 1), field_at(g, i0 + 1 + nx), field_at(g, i0 + nx),
                 field_at(g, i0 + nxy), field_at(g, i0 + nxy + 1), field_at(g, i0 + nxy + 1 + nx),
                 field_at(g, i0 + nxy + nx)};
    T scalar = hex_interp(vals, pc[0], pc[1], pc[2]);
    scalar = (scalar - g.min_scalar) * g.inv_delta;
    const T fi = scalar * (T)N1;
    int idx;
    if (fi > T(-1) && fi < (T)(N1 + 1)) idx = (int)(int64_t)fi;
    else idx = (fi >= (T)(N1 + 1)) ? N1 : 0;
    idx = idx < 0 ? 0 : (idx > N1 ? N1 : idx);
    ++nsamples;
    const float ti = (float)g.tau[idx];
    if (std::isinf(ti)) {
      cut = true;
      break;
    }
    if (ti == 0.f) continue;
    const float y = ti - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
    if (sum >= 18.f) break;  // exp(-18) < 2^-25 rounds to 0 in binary16 however tau grows
  }
  const float tr = cut ? 0.f : (float)std::exp(-(double)sum);
  return (T)(float)(_Float16)tr;
}

template <typename T>
inline void map_vertex(const Geo<T>& g, int64_t id, T V[3]) {
  const int64_t px = g.pd[0], pxy = (int64_t)g.pd[0] * g.pd[1];
  const int64_t k = id / pxy, j = (id / px) % g.pd[1], i = id % px;
  V[0] = g.morig[0] + g.msp[0] * (T)i;
  V[1] = g.morig[1] + g.msp[1] * (T)j;
  V[2] = g.morig[2] + g.msp[2] * (T)k;
}

template <typename T>
inline void light_origin(const Geo<T>& g, const T V[3], T L[3]) {
  if (g.light_kind == 0) {
    for (int d = 0; d < 3; ++d) L[d] = g.light[d];
  } else {
    for (int d = 0; d < 3; ++d) L[d] = V[d] - g.light[d] * g.dir_dist;
  }
}

// Map value of one vertex: opacity (reference) or FP16 transmittance (precision form).
template <typename T>
T vertex_opacity(const Geo<T>& g, int64_t id, uint64_t& ns) {
  T V[3], L[3];
  map_vertex(g, id, V);
  light_origin(g, V, L);
  if (g.precision) return light_march_point_tau(g, L, V, ns);
  return light_march_point(g, L, V, ns);
}

// ---- map lookup (TransmittanceMap.h:93-112 LocateCell, :166-197 estimator) -----

template <typename T, typename MapGet>
inline T map_opacity_at(const Geo<T>& g, const T p[3], MapGet get);

template <typename T, typename MapGet>
inline void map_estimate(const Geo<T>& g, const T p[3], MapGet get, T est[3]) {
  if (g.n_lights > 1) {
    // sum over the lights of (1 - opacity_l) * colour_l, accumulated in light order
    for (int l = 0; l < g.n_lights; ++l) {
      const int64_t off = (int64_t)l * g.map_nv;
      auto gl = [&get, off](int64_t i) -> T { return get(i + off); };
      const T tr = T(1) - map_opacity_at(g, p, gl);
      for (int d = 0; d < 3; ++d) {
        const T t = tr * g.lcols[3 * l + d];
        est[d] = (l == 0) ? t : est[d] + t;
      }
    }
    return;
  }
  // precision form: the map holds transmittance, interpolated directly
  const T tr = g.precision ? map_opacity_at(g, p, get) : T(1) - map_opacity_at(g, p, get);
  for (int d = 0; d < 3; ++d) est[d] = tr * g.light_color[d];
}

// GetEstimateUsingVerticesT (TransmittanceMap.h:200-229): map opacity at p.
template <typename T, typename MapGet>
inline T map_opacity_at(const Geo<T>& g, const T p[3], MapGet get) {
  int64_t c[3];
  for (int d = 0; d < 3; ++d) {
    T t = (p[d] - g.morig[d]) * g.minv[d];
    if (t < T(0)) t = T(0);
    if (t >= (T)(g.pd[d] - 1)) t = (T)(g.pd[d] - 2);
    c[d] = (int64_t)t;
  }
  const int64_t px = g.pd[0], pxy = (int64_t)g.pd[0] * g.pd[1];
  const int64_t i0 = c[2] * pxy + c[1] * px + c[0];
  T pc[3];
  for (int d = 0; d < 3; ++d) {
    const T mnp = g.morig[d] + g.msp[d] * (T)c[d];
    const T mxp = g.morig[d] + g.msp[d] * (T)(c[d] + 1);
    pc[d] = (p[d] - mnp) / (mxp - mnp);
  }
  T v[8];
  v[0] = get(i0);
  v[1] = get(i0 + 1);
  v[2] = get(i0 + 1 + px);
  v[3] = get(i0 + px);
  v[4] = get(i0 + pxy);
  v[5] = get(i0 + pxy + 1);
  v[6] = get(i0 + pxy + 1 + px);
  v[7] = get(i0 + pxy + px);
  return hex_interp(v, pc[0], pc[1], pc[2]);
}

// ---- camera + slab (LightedVolumeRenderer.cxx:644-718) --------------------------

template <typename T>
void camera_ray(const Geo<T>& g, int x, int y, T o[3], T d[3]) {
  const T sx = ((T)x + (T)0.5f) * g.kx - g.cx;
  const T sy = ((T)y + (T)0.5f) * g.ky - g.cy;
  T v[3];
  for (int k = 0; k < 3; ++k) v[k] = (g.cf[k] + sx * g.cr[k]) + sy * g.cu[k];
  const T len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int k = 0; k < 3; ++k) {
    d[k] = v[k] / len;
    o[k] = g.cam_pos[k];
  }
}

template <typename S>
bool slab(const S o[3], const S d[3], const double bmin[3], const double bmax[3], S& minD, S& maxD) {
  S inv[3], od[3], lo[3], hi[3];
  const S eps = (sizeof(S) == 4) ? (S)1e-8f : (S)1e-8;
  for (int k = 0; k < 3; ++k) {
    inv[k] = S(1) / ((std::fabs(d[k]) < eps) ? eps : d[k]);
    od[k] = o[k] * inv[k];
    lo[k] = (S)bmin[k] * inv[k] - od[k];
    hi[k] = (S)bmax[k] * inv[k] - od[k];
  }
  minD = mx(mx(mx(mn(lo[1], hi[1]), mn(lo[0], hi[0])), mn(lo[2], hi[2])), minD);
  const S exitD = mn(mn(mx(lo[1], hi[1]), mx(lo[0], hi[0])), mx(lo[2], hi[2]));
  maxD = mn(maxD, exitD);
  return !(maxD < minD);
}

template <typename T>
bool ray_setup(const Geo<T>& g, int x, int y, T o[3], T d[3], T& minD, T& maxD) {
  camera_ray(g, x, y, o, d);
  // MaxDistance enters as the pixel's canvas limit (+inf without a depth buffer)
  const float lim = g.ray_max ? g.ray_max[(int64_t)y * g.width + x] : std::numeric_limits<float>::infinity();
  if (sizeof(T) == 4 && g.slab_fp64) {
    double od[3] = {(double)o[0], (double)o[1], (double)o[2]};
    double dd[3] = {(double)d[0], (double)d[1], (double)d[2]};
    double lo = 0.0, hi = (double)lim;
    const bool hit = slab(od, dd, g.bmin, g.bmax, lo, hi);
    minD = (T)lo;
    maxD = (T)hi;
    return hit;
  }
  minD = T(0);
  maxD = (T)lim;
  return slab(o, d, g.bmin, g.bmax, minD, maxD);
}

// ---- view march (LightedVolumeRenderer.cxx:346-498, locator :45-186) -------------

template <typename T>
inline bool inside_vol(const Geo<T>& g, const T p[3]) {
  for (int d = 0; d < 3; ++d)
    if (p[d] < g.minp[d] || p[d] > g.maxp[d]) return false;
  return true;
}

struct NoRecord {
  template <typename T> void operator()(const T*, const T*, T) const {}
};

// RectilinearLocator::LocateCell (LightedVolumeRenderer.cxx:108-156): per axis,
// a point on the max face takes the last cell and keeps the previous inverse
// spacing; otherwise the cell is walked from the previous one until
// min <= p < max, and invSpacing = 1 / (max - min).
template <typename T>
inline void locate_cell_walk(const Geo<T>& g, const T p[3], int c[3], T inv[3]) {
  for (int k = 0; k < 3; ++k) {
    if (p[k] == g.maxp[k]) {
      c[k] = g.n[k] - 2;
      continue;
    }
    const std::vector<T>& C = g.C[k];
    bool found = false;
    T minVal = C[c[k]];
    const int dirn = (p[k] - minVal >= T(0)) ? 1 : -1;
    T maxVal = C[c[k] + 1];
    while (!found) {
      if (p[k] >= minVal && p[k] < maxVal) {
        found = true;
        continue;
      }
      c[k] += dirn;
      const int nid = dirn == 1 ? c[k] + 1 : c[k];
      const T next = C[nid];
      if (dirn == 1) {
        minVal = maxVal;
        maxVal = next;
      } else {
        maxVal = minVal;
        minVal = next;
      }
    }
    inv[k] = T(1) / (maxVal - minVal);
  }
}

// rec(p, tf_rgba, sa) is called at every composited sample, before shading.
template <typename T, typename MapGet, typename Rec = NoRecord>
void march_pixel(const Geo<T>& g, int x, int y, MapGet get, T color[4], uint64_t& lit, Rec rec = Rec()) {
  color[0] = color[1] = color[2] = color[3] = T(0);
  T o[3], d[3], minD, maxD;
  if (!ray_setup(g, x, y, o, d, minD, maxD)) return;  // minDistance == -1
  const T q = (maxD - minD) / g.sd;
  int64_t budget = (q < (T)1e9) ? (int64_t)q + 16 : (int64_t)1000000000;
  T dist = minD + g.mesh_eps;
  T p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
  while (!inside_vol(g, p) && dist < maxD && budget-- > 0) {
    dist += g.sd;
    for (int k = 0; k < 3; ++k) p[k] = o[k] + dist * d[k];
  }
  T bl[3] = {0, 0, 0};
  bool newCell = true;
  T tx = 0, ty = 0, tz = 0;
  T s0 = 0, s1m0 = 0, s2m3 = 0, s3 = 0, s4 = 0, s5m4 = 0, s6m7 = 0, s7 = 0;
  int c[3] = {0, 0, 0};
  T inv[3] = {0, 0, 0};
  const int N1 = g.tf_n - 1;
  const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
  while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
    const T mint = mn(tx, mn(ty, tz));
    const T maxt = mx(tx, mx(ty, tz));
    if (maxt > T(1) || mint < T(0)) newCell = true;
    if (newCell) {
      locate_cell_walk(g, p, c, inv);
      const int64_t i0 = (int64_t)c[2] * nxy + (int64_t)c[1] * nx + c[0];
      bl[0] = g.C[0][c[0]];
      bl[1] = g.C[1][c[1]];
      bl[2] = g.C[2][c[2]];
      s0 = (T)g.field[i0];
      const T s1 = (T)g.field[i0 + 1];
      const T s2 = (T)g.field[i0 + 1 + nx];
      s3 = (T)g.field[i0 + nx];
      s4 = (T)g.field[i0 + nxy];
      const T s5 = (T)g.field[i0 + nxy + 1];
      const T s6 = (T)g.field[i0 + nxy + 1 + nx];
      s7 = (T)g.field[i0 + nxy + nx];
      s6m7 = s6 - s7;
      s5m4 = s5 - s4;
      s1m0 = s1 - s0;
      s2m3 = s2 - s3;
      tx = (p[0] - bl[0]) * inv[0];
      ty = (p[1] - bl[1]) * inv[1];
      tz = (p[2] - bl[2]) * inv[2];
      newCell = false;
    }
    const T l76 = s7 + tx * s6m7;
    const T l45 = s4 + tx * s5m4;
    const T top = l45 + ty * (l76 - l45);
    const T l01 = s0 + tx * s1m0;
    const T l32 = s3 + tx * s2m3;
    const T bot = l01 + ty * (l32 - l01);
    T fs = bot + tz * (top - bot);
    fs = (fs - g.min_scalar) * g.inv_delta;
    const T fi = fs * (T)N1;
    if (fi > T(-1) && fi < (T)(N1 + 1)) {
      const int idx = (int)(int64_t)fi;
      T sc[4] = {g.tf[4 * idx], g.tf[4 * idx + 1], g.tf[4 * idx + 2], g.tf[4 * idx + 3]};
      sc[3] *= (T(1) - color[3]);
      rec(p, sc, sc[3]);
      if (g.use_map) {
        T est[3];
        map_estimate(g, p, get, est);
        sc[0] = sc[0] * est[0];
        sc[1] = sc[1] * est[1];
        sc[2] = sc[2] * est[2];
      }
      sc[0] = clamp01(sc[0]);
      sc[1] = clamp01(sc[1]);
      sc[2] = clamp01(sc[2]);
      color[0] = color[0] + sc[0] * sc[3];
      color[1] = color[1] + sc[1] * sc[3];
      color[2] = color[2] + sc[2] * sc[3];
      color[3] = sc[3] + color[3];
      ++lit;
    }
    dist += g.sd;
    for (int k = 0; k < 3; ++k) p[k] = p[k] + g.sd * d[k];
    tx = (p[0] - bl[0]) * inv[0];
    ty = (p[1] - bl[1]) * inv[1];
    tz = (p[2] - bl[2]) * inv[2];
    if (color[3] >= g.cutoff) break;
  }
}

// SamplerCellAssoc::operator() (LightedVolumeRenderer.cxx:540-641): the unlit
// march of a cell-centred field ((n-1)^3 values, x fastest, cell id
// (c2 (ny-1) + c1) (nx-1) + c0, :252-255). The TF index of the cell value is
// truncated and clamped to [0, n-1] (:603-608); the colour is fetched once per
// cell, the cell is kept while tx, ty, tz stay in [0, 1] (starting from 2, so
// the first sample locates, :581-583), each sample composites
// a = A (1 - C.a), C.rgb += rgb a, C.a += a (:617-621), then the ray advances
// and breaks on C.a >= cutoff before tx/ty/tz are updated (:624-631); the
// result is clamped to 1 per channel (:632-635). Every composite is counted.
template <typename T>
void march_pixel_cells(const Geo<T>& g, int x, int y, T color[4], uint64_t& lit) {
  color[0] = color[1] = color[2] = color[3] = T(0);
  T o[3], d[3], minD, maxD;
  if (!ray_setup(g, x, y, o, d, minD, maxD)) return;  // minDistance == -1
  const T q = (maxD - minD) / g.sd;
  int64_t budget = (q < (T)1e9) ? (int64_t)q + 16 : (int64_t)1000000000;
  T dist = minD + g.mesh_eps;
  T p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
  while (!inside_vol(g, p) && dist < maxD && budget-- > 0) {
    dist += g.sd;
    for (int k = 0; k < 3; ++k) p[k] = o[k] + dist * d[k];
  }
  bool newCell = true;
  T tx = T(2), ty = T(2), tz = T(2);
  T sc[4] = {0, 0, 0, 0};
  T bl[3] = {0, 0, 0};
  T inv[3] = {0, 0, 0};
  int c[3] = {0, 0, 0};
  const int N1 = g.tf_n - 1;
  const int64_t cx = g.n[0] - 1, cxy = (int64_t)(g.n[0] - 1) * (g.n[1] - 1);
  while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
    const T mint = mn(tx, mn(ty, tz));
    const T maxt = mx(tx, mx(ty, tz));
    if (maxt > T(1) || mint < T(0)) newCell = true;
    if (newCell) {
      locate_cell_walk(g, p, c, inv);
      const int64_t cid = (int64_t)c[2] * cxy + (int64_t)c[1] * cx + c[0];
      const T s0 = (T)g.field[cid];
      const T ns = (s0 - g.min_scalar) * g.inv_delta;
      const T fi = ns * (T)N1;
      int idx;  // static_cast<vtkm::Id>, saturating (see the file header), then the clamp
      if (fi > T(-1) && fi < (T)(N1 + 1)) idx = (int)(int64_t)fi;
      else idx = (fi >= (T)(N1 + 1)) ? N1 : 0;
      if (idx < 0) idx = 0;
      if (idx > N1) idx = N1;
      for (int k = 0; k < 4; ++k) sc[k] = g.tf[4 * idx + k];
      for (int k = 0; k < 3; ++k) bl[k] = g.C[k][c[k]];  // GetMinPoint
      tx = (p[0] - bl[0]) * inv[0];
      ty = (p[1] - bl[1]) * inv[1];
      tz = (p[2] - bl[2]) * inv[2];
      newCell = false;
    }
    const T alpha = sc[3] * (T(1) - color[3]);
    color[0] = color[0] + sc[0] * alpha;
    color[1] = color[1] + sc[1] * alpha;
    color[2] = color[2] + sc[2] * alpha;
    color[3] = alpha + color[3];
    ++lit;
    dist += g.sd;
    for (int k = 0; k < 3; ++k) p[k] = p[k] + g.sd * d[k];
    if (color[3] >= g.cutoff) break;
    tx = (p[0] - bl[0]) * inv[0];
    ty = (p[1] - bl[1]) * inv[1];
    tz = (p[2] - bl[2]) * inv[2];
  }
  for (int k = 0; k < 4; ++k) color[k] = mn(color[k], T(1));
}

int nthreads(int t) {
#ifdef _OPENMP
  return t > 0 ? t : omp_get_max_threads();
#else
  (void)t;
  return 1;
#endif
}

bool valid(const oracle_scene* s) {
  if (!s || !s->field || !s->tf || s->tf_n < 1) return false;
  for (int d = 0; d < 3; ++d) {
    if (s->dims[d] < 2 || s->map_m[d] < 1) return false;
    if (!(s->spacing[d] > 0)) return false;
  }
  if (!(s->light_steps > 0) || !(s->alpha_cutoff > 0)) return false;
  return true;
}

template <typename T>
int light_march_all(const oracle_scene* s, T* out, int threads, uint64_t* samples) {
  if (!valid(s) || !out) return 1;
  Geo<T> g;
  build_geo(s, g);
  const int64_t nv = (int64_t)g.pd[0] * g.pd[1] * g.pd[2];
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads(threads)) reduction(+ : total)
  for (int64_t id = 0; id < nv; ++id) {
    uint64_t ns = 0;
    out[id] = vertex_opacity(g, id, ns);
    total += ns;
  }
  if (samples) *samples = total;
  return 0;
}

template <typename T>
int light_march_ids(const oracle_scene* s, const int64_t* ids, int64_t n, T* out, int threads,
                    uint64_t* samples) {
  if (!valid(s) || !out || !ids) return 1;
  Geo<T> g;
  build_geo(s, g);
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads(threads)) reduction(+ : total)
  for (int64_t i = 0; i < n; ++i) {
    uint64_t ns = 0;
    out[i] = vertex_opacity(g, ids[i], ns);
    total += ns;
  }
  if (samples) *samples = total;
  return 0;
}

template <typename T>
int view_march_cells(const oracle_scene* s, int x0, int y0, int w, int h, T* rgba, int threads,
                     uint64_t* lit_out) {
  if (!valid(s) || !rgba) return 1;
  if (x0 < 0 || y0 < 0 || x0 + w > s->width || y0 + h > s->height) return 1;
  Geo<T> g;
  build_geo(s, g);
  uint64_t lit = 0;
  const int64_t npx = (int64_t)w * h;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads(threads)) reduction(+ : lit)
  for (int64_t i = 0; i < npx; ++i) {
    const int yy = (int)(i / w), xx = (int)(i - (int64_t)yy * w);
    T c[4];
    uint64_t l = 0;
    march_pixel_cells(g, x0 + xx, y0 + yy, c, l);
    lit += l;
    for (int k = 0; k < 4; ++k) rgba[4 * i + k] = c[k];
  }
  if (lit_out) *lit_out = lit;
  return 0;
}

template <typename T>
int view_march(const oracle_scene* s, const T* map, int x0, int y0, int w, int h, T* rgba,
               int threads, uint64_t* lit_out, int n_lights = 1, const float* lcols = nullptr) {
  if (!valid(s) || !rgba) return 1;
  if (s->use_map && !map) return 1;
  if (x0 < 0 || y0 < 0 || x0 + w > s->width || y0 + h > s->height) return 1;
  Geo<T> g;
  build_geo(s, g);
  if (n_lights > 1) {
    if (!lcols || !s->use_map || s->precision) return 1;
    g.n_lights = n_lights;
    g.map_nv = (int64_t)g.pd[0] * g.pd[1] * g.pd[2];
    g.lcols.assign(lcols, lcols + 3 * (size_t)n_lights);
  }
  uint64_t lit = 0;
  auto get = [map](int64_t i) -> T { return map[i]; };
  const int64_t npx = (int64_t)w * h;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads(threads)) reduction(+ : lit)
  for (int64_t i = 0; i < npx; ++i) {
    const int yy = (int)(i / w), xx = (int)(i - (int64_t)yy * w);
    T c[4];
    uint64_t l = 0;
    march_pixel(g, x0 + xx, y0 + yy, get, c, l);
    lit += l;
    T* dst = rgba + 4 * i;
    dst[0] = c[0];
    dst[1] = c[1];
    dst[2] = c[2];
    dst[3] = c[3];
  }
  if (lit_out) *lit_out = lit;
  return 0;
}

}  // namespace


// ---- multi-block rendering (the reference's sort-last path on one host) ----------
//
// Phase 1: each block marches its own map from zero (TransmittanceMap.h:565-621).
// Phases 2-3 (LightedVolumeRenderer.cxx:968-1256, TransmittanceMap.h:342-513):
// for every vertex, each other block the segment light->vertex crosses
// (SegmentAABB hit, glancing hits included) contributes its Phase-1 map opacity
// at the segment's exit point (RayT = tMax); the contributions are
// over-composited in increasing RayT and the local march is re-run starting
// from that prefix. Phase 4: each block renders the full image clipped to its
// own bounds. Phase 5 (MapperLightedVolume.cxx:215-303): images are composited
// front to back in increasing |camera - block centre|.
namespace {

template <typename T>
int render_bricks(const oracle_scene* sc, int nb, T* maps_local, T* maps_final, T* imgs, T* rgba, int threads,
                  uint64_t* lit_out) {
  if (nb < 1 || !rgba) return 1;
  for (int b = 0; b < nb; ++b)
    if (!valid(&sc[b])) return 1;
  std::vector<Geo<T>> G(nb);
  for (int b = 0; b < nb; ++b) build_geo(&sc[b], G[b]);
  std::vector<std::vector<T>> local(nb), fin(nb);
  for (int b = 0; b < nb; ++b) {
    const int64_t nv = (int64_t)G[b].pd[0] * G[b].pd[1] * G[b].pd[2];
    local[b].resize(nv);
    fin[b].resize(nv);
    const Geo<T>& g = G[b];
    T* dst = local[b].data();
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads(threads))
    for (int64_t id = 0; id < nv; ++id) {
      uint64_t ns = 0;
      dst[id] = vertex_opacity(g, id, ns);
    }
  }
  for (int b = 0; b < nb; ++b) {
    const int64_t nv = (int64_t)G[b].pd[0] * G[b].pd[1] * G[b].pd[2];
    const Geo<T>& g = G[b];
    T* dst = fin[b].data();
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads(threads))
    for (int64_t id = 0; id < nv; ++id) {
      T V[3], L[3];
      map_vertex(g, id, V);
      light_origin(g, V, L);
      T v[3] = {V[0] - L[0], V[1] - L[1], V[2] - L[2]};
      const T rs = T(1) / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      const T dir[3] = {v[0] * rs, v[1] * rs, v[2] * rs};
      struct Hit { T t; int blk; T op; };
      Hit hits[64];
      int nh = 0;
      for (int c = 0; c < nb && nh < 64; ++c) {
        if (c == b) continue;
        T tmin, tmax;
        segment_aabb(L, V, G[c], tmin, tmax);
        if (!(tmin <= tmax)) continue;
        const T P[3] = {L[0] + dir[0] * tmax, L[1] + dir[1] * tmax, L[2] + dir[2] * tmax};
        const T* mc = local[c].data();
        const T op = map_opacity_at(G[c], P, [mc](int64_t i) -> T { return mc[i]; });
        hits[nh++] = Hit{tmax, c, op};
      }
      // HitSort (TransmittanceMap.h:371-385): increasing RayT; ties by block id.
      for (int i = 1; i < nh; ++i)
        for (int j = i; j > 0 && (hits[j].t < hits[j - 1].t ||
                                  (hits[j].t == hits[j - 1].t && hits[j].blk < hits[j - 1].blk)); --j)
          std::swap(hits[j], hits[j - 1]);
      T o = T(0);
      for (int i = 0; i < nh; ++i) o = o + (T(1) - o) * hits[i].op;
      uint64_t ns = 0;
      dst[id] = light_march_point(g, L, V, ns, o);
    }
  }
  const int W = sc[0].width, H = sc[0].height;
  const int64_t npx = (int64_t)W * H;
  std::vector<T> img((size_t)nb * npx * 4);
  uint64_t lit = 0;
  for (int b = 0; b < nb; ++b) {
    const Geo<T>& g = G[b];
    const T* mp = fin[b].data();
    auto get = [mp](int64_t i) -> T { return mp[i]; };
    T* out = img.data() + (size_t)b * npx * 4;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads(threads)) reduction(+ : lit)
    for (int64_t i = 0; i < npx; ++i) {
      const int yy = (int)(i / W), xx = (int)(i - (int64_t)yy * W);
      T c[4];
      uint64_t l = 0;
      march_pixel(g, xx, yy, get, c, l);
      lit += l;
      for (int k = 0; k < 4; ++k) out[4 * i + k] = c[k];
    }
  }
  // depth order: |camera - block centre| in float (MapperLightedVolume.cxx:221-241)
  std::vector<std::pair<float, int>> order;
  const float cam[3] = {(float)sc[0].cam_pos[0], (float)sc[0].cam_pos[1], (float)sc[0].cam_pos[2]};
  for (int b = 0; b < nb; ++b) {
    float c3[3];
    for (int d = 0; d < 3; ++d) c3[d] = (float)((G[b].bmin[d] + G[b].bmax[d]) * 0.5);
    const float dx = cam[0] - c3[0], dy = cam[1] - c3[1], dz = cam[2] - c3[2];
    order.push_back({std::sqrt(dx * dx + dy * dy + dz * dz), b});
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<float, int>& l, const std::pair<float, int>& r) { return l.first < r.first; });
  const T* first = img.data() + (size_t)order[0].second * npx * 4;
  for (int64_t i = 0; i < 4 * npx; ++i) rgba[i] = first[i];
  for (int k = 1; k < nb; ++k) {
    const T* bimg = img.data() + (size_t)order[k].second * npx * 4;
    for (int64_t j = 0; j < npx; ++j) {
      T* a = rgba + 4 * j;
      const T* bb = bimg + 4 * j;
      a[0] = a[0] + bb[0] * (T(1) - a[3]);
      a[1] = a[1] + bb[1] * (T(1) - a[3]);
      a[2] = a[2] + bb[2] * (T(1) - a[3]);
      a[3] = a[3] + bb[3] * (T(1) - a[3]);
    }
  }
  size_t off = 0;
  for (int b = 0; b < nb; ++b) {
    if (maps_local) std::copy(local[b].begin(), local[b].end(), maps_local + off);
    if (maps_final) std::copy(fin[b].begin(), fin[b].end(), maps_final + off);
    off += local[b].size();
  }
  if (imgs) std::copy(img.begin(), img.end(), imgs);
  if (lit_out) *lit_out = lit;
  return 0;
}

}  // namespace

extern "C" int oracle_render_bricks_f32(const oracle_scene* scenes, int nbricks, float* maps_local, float* maps_final,
                                        float* brick_images, float* rgba, int threads, uint64_t* lit) {
  return render_bricks<float>(scenes, nbricks, maps_local, maps_final, brick_images, rgba, threads, lit);
}
extern "C" int oracle_render_bricks_f64(const oracle_scene* scenes, int nbricks, double* maps_local,
                                        double* maps_final, double* brick_images, double* rgba, int threads,
                                        uint64_t* lit) {
  return render_bricks<double>(scenes, nbricks, maps_local, maps_final, brick_images, rgba, threads, lit);
}

// ---- synthetic inputs on the CPU (the reference arm's field) ---------------------
// Same float32 operation sequence as the library's device generator
// (gradient noise after Perlin's "Improving Noise", 2002), so the two agree.
namespace {
inline float nfade(float t) { return t * t * t * (t * (t * 6.f - 15.f) + 10.f); }
inline float nlerp(float t, float a, float b) { return a + t * (b - a); }
inline float ngrad(int h, float x, float y, float z) {
  h &= 15;
  const float u = h < 8 ? x : y;
  const float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
  return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
float nperlin(const unsigned char* P, float x, float y, float z) {
  const float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  const int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
  x -= fx;
  y -= fy;
  z -= fz;
  const float u = nfade(x), v = nfade(y), w = nfade(z);
  const int A = P[X] + Y, AA = P[A & 255] + Z, AB = P[(A + 1) & 255] + Z;
  const int B = P[(X + 1) & 255] + Y, BA = P[B & 255] + Z, BB = P[(B + 1) & 255] + Z;
  return nlerp(w,
               nlerp(v, nlerp(u, ngrad(P[AA & 255], x, y, z), ngrad(P[BA & 255], x - 1, y, z)),
                     nlerp(u, ngrad(P[AB & 255], x, y - 1, z), ngrad(P[BB & 255], x - 1, y - 1, z))),
               nlerp(v, nlerp(u, ngrad(P[(AA + 1) & 255], x, y, z - 1), ngrad(P[(BA + 1) & 255], x - 1, y, z - 1)),
                     nlerp(u, ngrad(P[(AB + 1) & 255], x, y - 1, z - 1),
                           ngrad(P[(BB + 1) & 255], x - 1, y - 1, z - 1))));
}
}  // namespace

extern "C" int oracle_generate_noise(float* out, int nx, int ny, int nz, const unsigned char* perm, int octaves,
                                     float f0, float lac, float gain, int threads) {
  if (!out || !perm || nx < 2 || ny < 2 || nz < 2 || octaves < 1) return 1;
  const int64_t total = (int64_t)nx * ny * nz;
  float lo = std::numeric_limits<float>::infinity(), hi = -lo;
#pragma omp parallel for schedule(static) num_threads(nthreads(threads)) reduction(min : lo) reduction(max : hi)
  for (int64_t id = 0; id < total; ++id) {
    const int64_t k = id / ((int64_t)nx * ny);
    const int64_t r = id - k * (int64_t)nx * ny;
    const int j = (int)(r / nx), i = (int)(r - (int64_t)j * nx);
    const float x = (float)i / (float)(nx - 1);
    const float y = (float)j / (float)(ny - 1);
    const float z = (float)k / (float)(nz - 1);
    float f = f0, a = 1.f, v = 0.f;
    for (int o = 0; o < octaves; ++o) {
      v += a * nperlin(perm, x * f, y * f, z * f);
      f *= lac;
      a *= gain;
    }
    out[id] = v;
    lo = std::min(lo, v);
    hi = std::max(hi, v);
  }
  const float inv = (hi > lo) ? 1.f / (hi - lo) : 0.f;
#pragma omp parallel for schedule(static) num_threads(nthreads(threads))
  for (int64_t id = 0; id < total; ++id) {
    const float v = (out[id] - lo) * inv;
    out[id] = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
  }
  return 0;
}

template <typename T>
static int light_march_points(const oracle_scene* s, const T* pts, int64_t n, const T* light_pos, T* out,
                              int threads) {
  if (!valid(s) || !pts || !out) return 1;
  Geo<T> g;
  build_geo(s, g);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads(threads))
  for (int64_t i = 0; i < n; ++i) {
    const T P[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    T L[3];
    if (light_pos) {
      L[0] = light_pos[3 * i];
      L[1] = light_pos[3 * i + 1];
      L[2] = light_pos[3 * i + 2];
    } else {
      light_origin(g, P, L);
    }
    uint64_t ns = 0;
    out[i] = light_march_point(g, L, P, ns);
  }
  return 0;
}

extern "C" {

int oracle_light_march_f32(const oracle_scene* s, float* out, int threads, uint64_t* samples) {
  return light_march_all<float>(s, out, threads, samples);
}
int oracle_light_march_f64(const oracle_scene* s, double* out, int threads, uint64_t* samples) {
  return light_march_all<double>(s, out, threads, samples);
}
int oracle_light_march_ids_f32(const oracle_scene* s, const int64_t* ids, int64_t n, float* out,
                               int threads, uint64_t* samples) {
  return light_march_ids<float>(s, ids, n, out, threads, samples);
}
int oracle_light_march_ids_f64(const oracle_scene* s, const int64_t* ids, int64_t n, double* out,
                               int threads, uint64_t* samples) {
  return light_march_ids<double>(s, ids, n, out, threads, samples);
}

int oracle_light_march_points_f64(const oracle_scene* s, const double* pts, int64_t n,
                                  const double* light_pos, double* out, int threads) {
  return light_march_points<double>(s, pts, n, light_pos, out, threads);
}
int oracle_light_march_points_f32(const oracle_scene* s, const float* pts, int64_t n, const float* light_pos,
                                  float* out, int threads) {
  return light_march_points<float>(s, pts, n, light_pos, out, threads);
}

int oracle_view_march_f32(const oracle_scene* s, const float* map, int x0, int y0, int w, int h,
                          float* rgba, int threads, uint64_t* lit) {
  return view_march<float>(s, map, x0, y0, w, h, rgba, threads, lit);
}
int oracle_view_march_f64(const oracle_scene* s, const double* map, int x0, int y0, int w, int h,
                          double* rgba, int threads, uint64_t* lit) {
  return view_march<double>(s, map, x0, y0, w, h, rgba, threads, lit);
}

int oracle_view_march_cells_f32(const oracle_scene* s, int x0, int y0, int w, int h, float* rgba_out, int threads,
                                uint64_t* lit_samples) {
  return view_march_cells(s, x0, y0, w, h, rgba_out, threads, lit_samples);
}
int oracle_view_march_cells_f64(const oracle_scene* s, int x0, int y0, int w, int h, double* rgba_out, int threads,
                                uint64_t* lit_samples) {
  return view_march_cells(s, x0, y0, w, h, rgba_out, threads, lit_samples);
}
int oracle_window_depth_to_distance(const oracle_scene* s, const float* depth, double near_plane,
                                    double far_plane, double* out) {
  if (!valid(s) || !depth || !out || !(near_plane > 0.0) || !(far_plane > near_plane)) return 1;
  Geo<double> g;
  build_geo(s, g);
  for (int y = 0; y < g.height; ++y)
    for (int x = 0; x < g.width; ++x) {
      const int64_t i = (int64_t)y * g.width + x;
      double dw = (double)depth[i];
      dw = (dw == dw) ? std::min(std::max(dw, 0.0), 1.0) : 1.0;
      const double z = 2.0 * dw - 1.0;
      const double t = 2.0 * far_plane * near_plane / ((far_plane + near_plane) - z * (far_plane - near_plane));
      const double sx = ((double)x + 0.5) * g.kx - g.cx, sy = ((double)y + 0.5) * g.ky - g.cy;
      double v[3];
      for (int k = 0; k < 3; ++k) v[k] = (g.cf[k] + sx * g.cr[k]) + sy * g.cu[k];
      out[i] = t * std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
  return 0;
}

// Multi-light extension: maps holds n_lights exact-form maps stacked in light
// order; light_colors holds colour * intensity per light (float32, n_lights x 3).
int oracle_view_march_multi_f32(const oracle_scene* s, const float* maps, int n_lights, const float* light_colors,
                                int x0, int y0, int w, int h, float* rgba, int threads, uint64_t* lit) {
  if (n_lights < 1) return 1;
  return view_march<float>(s, maps, x0, y0, w, h, rgba, threads, lit, n_lights, light_colors);
}

// FP64 view march whose map vertices are computed on first use (memoised), for
// crops of scenes whose full FP64 map would take too long on the CPU. Pixels
// are taken every `stride` pixels of the window; rgba_out holds
// ceil(w/stride)*ceil(h/stride)*4 values.
int oracle_view_march_lazy_f64(const oracle_scene* s, int x0, int y0, int w, int h, int stride,
                               double* rgba, int threads, uint64_t* lit_out) {
  if (!valid(s) || !rgba || stride < 1) return 1;
  if (x0 < 0 || y0 < 0 || x0 + w > s->width || y0 + h > s->height) return 1;
  Geo<double> g;
  build_geo(s, g);
  const int64_t nv = (int64_t)g.pd[0] * g.pd[1] * g.pd[2];
  std::vector<double> vals(s->use_map ? nv : 1);
  std::vector<std::atomic<uint8_t>> state(s->use_map ? nv : 1);
  for (auto& a : state) a.store(0, std::memory_order_relaxed);
  auto get = [&](int64_t i) -> double {
    if (state[i].load(std::memory_order_acquire) == 2) return vals[i];
    uint64_t ns = 0;
    const double v = vertex_opacity(g, i, ns);
    vals[i] = v;  // every writer stores the same value
    state[i].store(2, std::memory_order_release);
    return v;
  };
  const int ow = (w + stride - 1) / stride, oh = (h + stride - 1) / stride;
  uint64_t lit = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads(threads)) reduction(+ : lit)
  for (int yy = 0; yy < oh; ++yy) {
    for (int xx = 0; xx < ow; ++xx) {
      double c[4];
      uint64_t l = 0;
      march_pixel(g, x0 + xx * stride, y0 + yy * stride, get, c, l);
      lit += l;
      double* dst = rgba + 4 * ((int64_t)yy * ow + xx);
      for (int k = 0; k < 4; ++k) dst[k] = c[k];
    }
  }
  if (lit_out) *lit_out = lit;
  return 0;
}

// Lit samples of the pixel window in march order: for each sample its position
// (xyz), TF rgb and premultiplied alpha (7 floats); counts[i] per pixel. Stops
// at cap samples in total (returns 2 if the cap was hit). The shading is not
// applied, so any transmittance model can be composited from these records.
int oracle_record_samples_f32(const oracle_scene* s, int x0, int y0, int w, int h, float* rec, int64_t cap,
                              int* counts) {
  if (!valid(s) || !rec || !counts) return 1;
  Geo<float> g;
  build_geo(s, g);
  g.use_map = 0;
  int64_t n = 0;
  bool full = false;
  for (int yy = 0; yy < h; ++yy)
    for (int xx = 0; xx < w; ++xx) {
      float c[4];
      uint64_t l = 0;
      int cnt = 0;
      auto r = [&](const float* p, const float* sc, float sa) {
        if (n >= cap) {
          full = true;
          return;
        }
        float* d = rec + 7 * n;
        d[0] = p[0]; d[1] = p[1]; d[2] = p[2];
        d[3] = sc[0]; d[4] = sc[1]; d[5] = sc[2]; d[6] = sa;
        ++n;
        ++cnt;
      };
      march_pixel(g, x0 + xx, y0 + yy, [](int64_t) { return 0.f; }, c, l, r);
      counts[yy * w + xx] = cnt;
    }
  return full ? 2 : 0;
}

int oracle_ray_setup_f32(const oracle_scene* s, int x, int y, float out[8]) {
  if (!valid(s) || !out) return 1;
  Geo<float> g;
  build_geo(s, g);
  float o[3], d[3], lo, hi;
  const bool hit = ray_setup(g, x, y, o, d, lo, hi);
  for (int k = 0; k < 3; ++k) {
    out[k] = o[k];
    out[3 + k] = d[k];
  }
  out[6] = hit ? lo : -1.f;
  out[7] = hi;
  return 0;
}

// SphereFieldGenerator::operator() (beams/sources/Spheres.cxx:36-91), float32,
// with vtkm::Lerp(a, b, t) taken as a + t * (b - a) (VTK-m not vendored here).
int oracle_generate_spheres(float* out, int nx, int ny, int nz, const float origin[3], const float spacing[3],
                            const float* e, int ne, float def, int has_floor, float floor_y, float floor_v) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || ne < 0 || (ne > 0 && !e)) return 1;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const float p[3] = {origin[0] + spacing[0] * (float)x, origin[1] + spacing[1] * (float)y,
                            origin[2] + spacing[2] * (float)z};
        float sum = 0.f, cnt = 0.f;
        for (int k = 0; k < ne; ++k) {
          const float* s = e + 8 * k;
          const float d0 = s[0] - p[0], d1 = s[1] - p[1], d2 = s[2] - p[2];
          float a = ((d0 * d0) / (s[3] * s[3])) + ((d1 * d1) / (s[4] * s[4]));
          a = a + ((d2 * d2) / (s[5] * s[5]));
          a = std::sqrt(a);
          if (a <= 1.f) {
            sum = sum + (s[6] + a * (s[7] - s[6]));
            cnt = cnt + 1.f;
          }
        }
        float v = cnt > 0.f ? sum / cnt : def;
        if (has_floor && p[1] < floor_y) v = floor_v;
        out[((size_t)z * ny + y) * nx + x] = v;
      }
  return 0;
}

int oracle_composite_f32(const float* images, int nimages, int npix, const int* order, float* out) {
  if (!images || !order || !out || nimages < 1 || npix < 0) return 1;
  const float* first = images + (int64_t)order[0] * npix * 4;
  std::memcpy(out, first, sizeof(float) * 4 * (size_t)npix);
  for (int i = 1; i < nimages; ++i) {
    const float* b = images + (int64_t)order[i] * npix * 4;
    for (int64_t j = 0; j < npix; ++j) {
      float* a = out + 4 * j;
      const float* bb = b + 4 * j;
      a[0] = a[0] + bb[0] * (1.0f - a[3]);
      a[1] = a[1] + bb[1] * (1.0f - a[3]);
      a[2] = a[2] + bb[2] * (1.0f - a[3]);
      a[3] = a[3] + bb[3] * (1.0f - a[3]);
    }
  }
  return 0;
}

}  // extern "C"
