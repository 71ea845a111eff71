// beams_api.cu — the C ABI (include/beams_b200.h): renderer state, parameter
// derivation and frame orchestration. Host code only; kernels live in k_*.cu.
//
// Phase structure of one frame follows LightedVolumeRenderer::RenderOnDevice
// (beams/rendering/LightedVolumeRenderer.cxx:910-1372): the map is built once
// (the reference's Phase 3 re-runs Phase 1 from zero opacity when there is a
// single block, :1210-1256, which yields the same map), then the view march.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/beams_b200.h"
#include "beams_params.h"
#include "kernels.h"
#include "renderer.h"

using beams::Counters;
using beams::ExactGeo;

namespace {
thread_local std::string g_tls_error;
}

namespace beams {

beams_status fail(beams_renderer* r, beams_status s, const std::string& msg) {
  if (r) r->err = msg;
  else g_tls_error = msg;
  return s;
}

beams_status cuda_fail(beams_renderer* r, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a sticky-free error so the next call starts clean
  return fail(r, e == cudaErrorMemoryAllocation ? BEAMS_ERR_OOM : BEAMS_ERR_CUDA, m);
}

// Allocation-failure injection for tests (beams_test_fail_allocation): the
// n-th following buffer allocation reports out-of-memory instead of allocating.
static std::atomic<int> g_fail_alloc_in{0};

beams_status ensure_buffer(beams_renderer* r, void** buf, size_t* cap, size_t bytes, const char* what) {
  if (*cap >= bytes && *buf) return BEAMS_OK;
  if (*buf) {
    cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
  }
  int pending = g_fail_alloc_in.load();
  while (pending > 0 && !g_fail_alloc_in.compare_exchange_weak(pending, pending - 1)) {
  }
  if (pending == 1) return fail(r, BEAMS_ERR_OOM, std::string(what) + ": out of device memory (injected)");
  cudaError_t e = cudaMalloc(buf, bytes);
  if (e != cudaSuccess) {
    *buf = nullptr;
    return cuda_fail(r, e, what);
  }
  *cap = bytes;
  return BEAMS_OK;
}

beams_status ensure_masked_map(beams_renderer* r, float** buf, size_t* cap, size_t bytes, cudaStream_t st,
                               bool clear) {
  const bool fresh = clear || !(*buf && *cap >= bytes);
  beams_status s = ensure_buffer(r, (void**)buf, cap, bytes, "allocating map");
  if (s != BEAMS_OK || !fresh) return s;
  cudaError_t e = cudaMemsetAsync(*buf, 0, bytes, st);
  if (e != cudaSuccess) return cuda_fail(r, e, "clearing map");
  return BEAMS_OK;
}

static bool finite3(const double* v) {
  return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

// Light l's part of the kernel parameters (Color * Intensity, LightedVolumeRenderer.cxx:840).
static void geo_set_light(ExactGeo& g, const Light& L) {
  g.light_kind = L.kind;
  for (int d = 0; d < 3; ++d) g.light_color[d] = L.color[d] * L.intensity;
  if (L.kind == 0) {
    for (int d = 0; d < 3; ++d) g.light[d] = (float)L.v[d];
  } else {
    const double len = std::sqrt(L.v[0] * L.v[0] + L.v[1] * L.v[1] + L.v[2] * L.v[2]);
    for (int d = 0; d < 3; ++d) g.light[d] = (float)(L.v[d] / len);
  }
  // the map build's brick order follows the light's travel direction at the
  // volume centre, in map-vertex units (see ExactGeo::bo_axis)
  double e[3];
  for (int d = 0; d < 3; ++d) {
    const double c = 0.5 * (g.bmin[d] + g.bmax[d]);
    const double t = (L.kind == 0) ? c - L.v[d] : L.v[d];
    e[d] = (g.msp[d] > 0.f) ? t / (double)g.msp[d] : 0.0;
  }
  int w = 2;
  for (int d = 0; d < 3; ++d)
    if (std::fabs(e[d]) > std::fabs(e[w])) w = d;
  const int u = (w == 0) ? 1 : 0, v = (w == 2) ? 1 : 2;
  g.bo_axis[0] = w;
  g.bo_axis[1] = u;
  g.bo_axis[2] = v;
  const bool ok = std::fabs(e[w]) > 0.0 && std::isfinite(e[w]);
  g.bo_shear[0] = ok ? (int)std::lround(65536.0 * e[u] / e[w]) : 0;
  g.bo_shear[1] = ok ? (int)std::lround(65536.0 * e[v] / e[w]) : 0;
}

// Derives the kernel parameters exactly as the reference derives them
// (float32 arithmetic; see the cited lines in beams_params.h).
beams_status make_geo_vol(beams_renderer* r, const beams_volume& v, const beams_camera* cam, ExactGeo& g) {
  std::memset(&g, 0, sizeof(g));
  g.bo_axis[0] = 2;  // z-pencils until a light sets the order
  g.bo_axis[1] = 0;
  g.bo_axis[2] = 1;
  // the renderer's own volume may carry explicit rectilinear coordinates
  const bool rect = r->rect && &v == &r->vol;
  g.rect = rect ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    g.n[d] = v.dims[d];
    if (rect) {
      // MinPoint / MaxPoint are the first and last coordinates
      // (LightedVolumeRenderer.cxx:77-87); the uniform fields keep the average spacing
      g.minp[d] = r->coords[d].front();
      g.maxp[d] = r->coords[d].back();
      g.org[d] = g.minp[d];
      g.h[d] = (g.maxp[d] - g.minp[d]) / (float)(v.dims[d] - 1);
    } else {
      g.org[d] = (float)v.origin[d];
      g.h[d] = (float)v.spacing[d];
      g.minp[d] = g.org[d] + g.h[d] * 0.f;
      g.maxp[d] = g.org[d] + g.h[d] * (float)(v.dims[d] - 1);
    }
    g.invh[d] = 1.f / g.h[d];
    g.bmin[d] = (double)g.minp[d];
    g.bmax[d] = (double)g.maxp[d];
  }
  const float fmin = (float)v.range[0], fmax = (float)v.range[1];
  g.min_scalar = fmin;
  g.inv_delta = ((fmax - fmin) != 0.f) ? 1.f / (fmax - fmin) : fmin;
  g.tf_n = r->tf_n;
  float ma = 0.f;
  for (int i = 0; i < r->tf_n; ++i) {
    const float a = r->tf[4 * i + 3];
    ma = (ma < a) ? a : ma;
  }
  g.max_alpha = ma;
  float ext[3];
  for (int d = 0; d < 3; ++d) ext[d] = (float)(g.bmax[d] - g.bmin[d]);
  g.extent_mag = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]);
  for (int d = 0; d < 3; ++d) {
    g.pd[d] = r->map_m[d] + 1;
    g.morig[d] = (float)g.bmin[d];
    g.msp[d] = ext[d] / (float)r->map_m[d];
    g.minv[d] = 1.f / g.msp[d];
  }
  g.sd = (r->sample_distance > 0.f) ? r->sample_distance : g.extent_mag / 200.f;
  // Bounds every view ray's iteration count (and so the kernel's run time).
  if (!(g.extent_mag / g.sd <= 1.0e6f))
    return fail(r, BEAMS_ERR_INVALID_ARG, "sample distance is below 1e-6 of the volume diagonal");
  g.mesh_eps = g.extent_mag * 0.0001f;
  g.step = g.extent_mag / r->light_steps;
  g.cutoff = r->cutoff;
  g.light_budget = (int)(g.extent_mag / g.step) + 8;
  g.light_brick_log2 = r->light_brick_log2;
  occupancy_dims(g.n, g.occ_n);
  g.dir_dist = 2.f * g.extent_mag;
  if (!r->lights.empty()) geo_set_light(g, r->lights[0]);
  g.n_lights = 1;
  for (int d = 0; d < 3; ++d) g.light_colors[0][d] = g.light_color[d];
  if (r->multi_light && r->lights.size() > 1) {
    g.n_lights = (int)r->lights.size();
    for (int l = 0; l < g.n_lights; ++l)
      for (int d = 0; d < 3; ++d) g.light_colors[l][d] = r->lights[l].color[d] * r->lights[l].intensity;
  }
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    g.ax_off[d] = off;
    off += g.n[d] - 1;
  }
  for (int d = 0; d < 3; ++d) {
    g.max_off[d] = off;
    off += r->map_m[d];
  }
  g.ntab = off;
  geo_loop_constants(g);
  g.slab_fp64 = r->slab_fp64;
  g.use_map = r->use_map ? 1 : 0;
  g.assoc_cells = (v.assoc == BEAMS_ASSOC_CELLS) ? 1 : 0;
  if (cam) {
    double f[3], rr[3], u[3];
    for (int d = 0; d < 3; ++d) f[d] = cam->look_at[d] - cam->position[d];
    const double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (int d = 0; d < 3; ++d) f[d] /= fl;
    const double* up = cam->up;
    rr[0] = f[1] * up[2] - f[2] * up[1];
    rr[1] = f[2] * up[0] - f[0] * up[2];
    rr[2] = f[0] * up[1] - f[1] * up[0];
    const double rl = std::sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
    if (!(fl > 0) || !(rl > 0)) return fail(r, BEAMS_ERR_INVALID_ARG, "camera: degenerate view or up vector");
    for (int d = 0; d < 3; ++d) rr[d] /= rl;
    u[0] = rr[1] * f[2] - rr[2] * f[1];
    u[1] = rr[2] * f[0] - rr[0] * f[2];
    u[2] = rr[0] * f[1] - rr[1] * f[0];
    const double th = std::tan(cam->fov_y_deg * M_PI / 360.0);
    const double aspect = (double)cam->width / (double)cam->height;
    for (int d = 0; d < 3; ++d) {
      g.cam_pos[d] = (float)cam->position[d];
      g.cf[d] = (float)f[d];
      g.cr[d] = (float)rr[d];
      g.cu[d] = (float)u[d];
    }
    g.kx = (float)(2.0 * th * aspect / cam->width);
    g.cx = (float)(th * aspect);
    g.ky = (float)(2.0 * th / cam->height);
    g.cy = (float)th;
    g.width = cam->width;
    g.height = cam->height;
    g.win[0] = 0;
    g.win[1] = 0;
    g.win[2] = cam->width;
    g.win[3] = cam->height;
  }
  return BEAMS_OK;
}

// The pixels whose rays can meet the box [bmin, bmax]: the bounding rectangle
// of its corners projected through the pinhole camera (the projection of a box
// in front of the camera is the convex hull of its corners'), widened by two
// pixels, which is far more than the rounding of a ray's direction. A corner at
// or behind the camera plane gives the whole image. Returns false when the
// window is empty.
static bool brick_window(const ExactGeo& g, int win[4]) {
  win[0] = 0;
  win[1] = 0;
  win[2] = g.width;
  win[3] = g.height;
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
  for (int k = 0; k < 8; ++k) {
    const double c[3] = {(k & 1) ? g.bmax[0] : g.bmin[0], (k & 2) ? g.bmax[1] : g.bmin[1],
                         (k & 4) ? g.bmax[2] : g.bmin[2]};
    double v[3], zf = 0, xr = 0, yu = 0;
    for (int d = 0; d < 3; ++d) v[d] = c[d] - (double)g.cam_pos[d];
    for (int d = 0; d < 3; ++d) {
      zf += v[d] * g.cf[d];
      xr += v[d] * g.cr[d];
      yu += v[d] * g.cu[d];
    }
    if (!(zf > 1e-6 * (std::fabs(xr) + std::fabs(yu) + 1e-30))) return true;  // whole image
    // pixel x of direction cf + sx cr + sy cu: (x + 0.5) kx - cx = sx
    const double px = (xr / zf + g.cx) / g.kx - 0.5, py = (yu / zf + g.cy) / g.ky - 0.5;
    xmin = std::min(xmin, px);
    xmax = std::max(xmax, px);
    ymin = std::min(ymin, py);
    ymax = std::max(ymax, py);
  }
  const double x0 = std::max(0.0, std::floor(xmin) - 2.0), y0 = std::max(0.0, std::floor(ymin) - 2.0);
  const double x1 = std::min((double)g.width, std::ceil(xmax) + 3.0);
  const double y1 = std::min((double)g.height, std::ceil(ymax) + 3.0);
  if (!(x1 > x0 && y1 > y0)) {
    win[2] = win[3] = 0;
    return false;
  }
  win[0] = (int)x0;
  win[1] = (int)y0;
  win[2] = (int)(x1 - x0);
  win[3] = (int)(y1 - y0);
  return true;
}

beams_status make_geo(beams_renderer* r, const beams_camera* cam, ExactGeo& g) {
  return make_geo_vol(r, r->vol, cam, g);
}

beams_status validate_camera(beams_renderer* r, const beams_camera* cam) {
  if (!cam) return fail(r, BEAMS_ERR_INVALID_ARG, "camera is NULL");
  if (cam->width < 1 || cam->height < 1 || cam->width > 16384 || cam->height > 16384)
    return fail(r, BEAMS_ERR_INVALID_ARG, "camera: width/height must be in [1, 16384]");
  if (!(cam->fov_y_deg > 0.0 && cam->fov_y_deg < 180.0))
    return fail(r, BEAMS_ERR_INVALID_ARG, "camera: fov_y_deg must be in (0, 180)");
  if (!finite3(cam->position) || !finite3(cam->look_at) || !finite3(cam->up))
    return fail(r, BEAMS_ERR_INVALID_ARG, "camera: non-finite vector");
  return BEAMS_OK;
}

// Key of the inputs a map depends on; a cached map is reused only on a match.
static void map_key(const beams_renderer* r, MapKey& k) {
  std::memset(&k, 0, sizeof(k));
  k.volume_version = r->volume_version;
  k.tf_version = r->tf_version;
  for (int d = 0; d < 3; ++d) k.m[d] = r->map_m[d];
  k.steps = r->light_steps;
  k.form = r->form;
  if (!r->lights.empty()) {
    k.light_kind = r->lights[0].kind;
    for (int d = 0; d < 3; ++d) k.light[d] = r->lights[0].v[d];
  }
  k.n_lights = (r->multi_light && r->lights.size() > 1) ? (int)r->lights.size() : 1;
  for (int l = 1; l < k.n_lights && l < kMaxMultiLights; ++l) {
    k.extra_kind[l] = r->lights[l].kind;
    for (int d = 0; d < 3; ++d) k.extra[l][d] = r->lights[l].v[d];
  }
}

// Derived layouts of one field: cell tables and (point fields) the quad copy.
static beams_status prepare_layouts_for(beams_renderer* r, const ExactGeo& g, int assoc, const void* d_field,
                                        unsigned long long version, float4** d_tab, size_t* tab_cap,
                                        unsigned long long tab_key[4], float4** d_quads, size_t* quads_cap,
                                        unsigned long long* quads_version, int& launches) {
  const unsigned long long key[4] = {version, (unsigned long long)r->map_m[0], (unsigned long long)r->map_m[1],
                                     (unsigned long long)r->map_m[2]};
  if (std::memcmp(key, tab_key, sizeof(key)) != 0) {
    beams_status s = ensure_buffer(r, (void**)d_tab, tab_cap, (size_t)g.ntab * sizeof(float4), "allocating cell tables");
    if (s != BEAMS_OK) return s;
    cudaError_t e = launch_build_tables(g, *d_tab, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "cell table build");
    ++launches;
    std::memcpy(tab_key, key, sizeof(key));
  }
  if (assoc == BEAMS_ASSOC_POINTS && *quads_version != version) {
    const size_t nq = (size_t)(g.n[0] - 1) * (g.n[1] - 1) * g.n[2];
    beams_status s = ensure_buffer(r, (void**)d_quads, quads_cap, nq * sizeof(float4), "allocating quad field");
    if (s != BEAMS_OK) return s;
    cudaError_t e = launch_build_quads(d_field, BEAMS_F32, *d_quads, BEAMS_F32, g.n, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "quad field build");
    ++launches;
    *quads_version = version;
  }
  return BEAMS_OK;
}

// Element type of the quad field the current form reads: float32 quads in the
// exact form, bfloat16/binary16 quads in the precision form.
static int quad_dtype(const beams_renderer* r) {
  if (r->form != BEAMS_FORM_PRECISION) return BEAMS_F32;
  return (r->vol.dtype == BEAMS_BF16 || r->vol.dtype == BEAMS_F16) ? r->vol.dtype : r->prec_dtype;
}

// Builds the derived layouts the kernels read: cell tables (per frame geometry)
// and, for point fields, the 4-corner quad copy of the field in the form's dtype.
beams_status prepare_layouts(beams_renderer* r, const ExactGeo& g, int& launches) {
  const unsigned long long key[4] = {r->volume_version, (unsigned long long)r->map_m[0],
                                     (unsigned long long)r->map_m[1], (unsigned long long)r->map_m[2]};
  if (std::memcmp(key, r->tab_key, sizeof(key)) != 0) {
    beams_status s = ensure_buffer(r, (void**)&r->d_tab, &r->tab_cap, (size_t)g.ntab * sizeof(float4),
                                   "allocating cell tables");
    if (s != BEAMS_OK) return s;
    cudaError_t e = launch_build_tables(g, r->d_tab, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "cell table build");
    ++launches;
    if (g.rect) {
      // explicit coordinates: the field axes' entries {lo, hi, hi - lo, RN(1 / (hi - lo))}
      std::vector<float4> fe((size_t)g.max_off[0]);
      for (int d = 0; d < 3; ++d)
        for (int c = 0; c + 1 < g.n[d]; ++c) {
          const float lo = r->coords[d][c], hi = r->coords[d][c + 1], w = hi - lo;
          fe[(size_t)g.ax_off[d] + c] = make_float4(lo, hi, w, 1.f / w);
        }
      e = cudaMemcpyAsync(r->d_tab, fe.data(), fe.size() * sizeof(float4), cudaMemcpyHostToDevice, r->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
      if (e != cudaSuccess) return cuda_fail(r, e, "coordinate table upload");
    }
    std::memcpy(r->tab_key, key, sizeof(key));
  }
  const int qd = quad_dtype(r);
  const unsigned long long qkey = r->volume_version * 4ull + (unsigned long long)qd;
  if (r->vol.assoc == BEAMS_ASSOC_POINTS && r->quads_version != qkey) {
    const size_t nq = (size_t)(g.n[0] - 1) * (g.n[1] - 1) * g.n[2];
    const size_t qbytes = (qd == BEAMS_F32) ? sizeof(float4) : 8;
    beams_status s = ensure_buffer(r, (void**)&r->d_quads, &r->quads_cap, nq * qbytes, "allocating quad field");
    if (s != BEAMS_OK) return s;
    cudaError_t e = launch_build_quads(r->d_field, r->vol.dtype, r->d_quads, qd, g.n, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "quad field build");
    ++launches;
    r->quads_version = qkey;
  }
  return BEAMS_OK;
}

// Occupancy of the current quads under the current colour map (rebuilt when either changes).
beams_status prepare_occupancy(beams_renderer* r, const ExactGeo& g, int& launches) {
  const int qd = quad_dtype(r);
  const unsigned long long key[2] = {r->volume_version * 4ull + (unsigned long long)qd, r->tf_version};
  if (key[0] == r->occ_key[0] && key[1] == r->occ_key[1]) return BEAMS_OK;
  const size_t nm = (size_t)g.occ_n[0] * g.occ_n[1] * g.occ_n[2];
  beams_status s = ensure_buffer(r, (void**)&r->d_occ, &r->occ_cap, nm, "allocating occupancy grid");
  if (s != BEAMS_OK) return s;
  cudaError_t e = launch_build_occupancy(g, qd, r->d_quads, r->d_tf, r->d_occ, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "occupancy build");
  ++launches;
  r->occ_key[0] = key[0];
  r->occ_key[1] = key[1];
  return BEAMS_OK;
}

beams_status build_map(beams_renderer* r, const ExactGeo& g, int& launches, bool& built) {
  built = false;
  MapKey key;
  map_key(r, key);
  if (r->reuse_map && r->map_valid && std::memcmp(&key, &r->map_key, sizeof(key)) == 0) return BEAMS_OK;
  const size_t nvert = (size_t)g.pd[0] * g.pd[1] * g.pd[2];
  const bool prec = r->form == BEAMS_FORM_PRECISION;
  const int nl = g.n_lights > 1 ? g.n_lights : 1;  // the multi-light extension: one map per light
  beams_status s = ensure_buffer(r, (void**)&r->d_map, &r->map_cap, nl * nvert * (prec ? 2 : sizeof(float)),
                                 "allocating map");
  if (s != BEAMS_OK) return s;
  r->map_valid = false;
  const unsigned char* occ = nullptr;
  if (r->empty_skip && !g.rect) {  // the occupancy grid indexes uniform macro-cells
    s = prepare_occupancy(r, g, launches);
    if (s != BEAMS_OK) return s;
    occ = r->d_occ;
  }
  cudaError_t e = prec ? launch_light_march_prec(g, quad_dtype(r), r->d_quads, r->d_tab, r->d_tf, r->d_tau,
                                                 (__half*)r->d_map, r->d_cnt, r->stream, occ)
                       : launch_light_march_f32(g, (const float4*)r->d_quads, r->d_tab, r->d_tf, r->d_map, r->d_cnt,
                                                r->stream, nullptr, 0, -1, nullptr, occ);
  if (e != cudaSuccess) return cuda_fail(r, e, "light_march launch");
  ++launches;
  for (int l = 1; l < nl; ++l) {
    ExactGeo gl = g;
    geo_set_light(gl, r->lights[l]);
    e = launch_light_march_f32(gl, (const float4*)r->d_quads, r->d_tab, r->d_tf, r->d_map + (size_t)l * nvert,
                               r->d_cnt, r->stream, nullptr, 0, -1, nullptr, occ);
    if (e != cudaSuccess) return cuda_fail(r, e, "light_march launch");
    ++launches;
  }
  r->map_key = key;
  r->map_valid = true;
  r->map_count = nl * nvert;
  r->map_is_half = prec;
  built = true;
  return BEAMS_OK;
}

// The exact form's lazy map (beams_set_lazy_shadow_map). The view rays' samples
// and their order do not depend on the map (early termination reads only the
// colour map's alpha), so a view march without shading marks the map cells
// the frame reads, and the light march builds only the vertices of marked
// cells: the image equals the full map's bit for bit. The map itself is
// partial, so it is neither kept for reuse nor readable.
static void mark_key(const beams_renderer* r, const ExactGeo& g, MarkKey& k) {
  std::memset(&k, 0, sizeof(k));
  k.volume_version = r->volume_version;
  k.tf_version = r->tf_version;
  k.depth_version = r->depth_set ? r->depth_version : 0;
  for (int d = 0; d < 3; ++d) {
    k.cam[d] = g.cam_pos[d];
    k.cam[3 + d] = g.cf[d];
    k.cam[6 + d] = g.cr[d];
    k.cam[9 + d] = g.cu[d];
    k.morig[d] = g.morig[d];
    k.minv[d] = g.minv[d];
    k.pd[d] = g.pd[d];
  }
  k.k[0] = g.kx;
  k.k[1] = g.cx;
  k.k[2] = g.ky;
  k.k[3] = g.cy;
  k.sd = g.sd;
  k.mesh_eps = g.mesh_eps;
  k.cutoff = g.cutoff;
  k.min_scalar = g.min_scalar;
  k.inv_delta = g.inv_delta;
  k.size[0] = g.width;
  k.size[1] = g.height;
  for (int i = 0; i < 4; ++i) k.win[i] = g.win[i];
  k.slab_fp64 = g.slab_fp64;
  k.form = r->form;
  k.quad_dtype = quad_dtype(r);
}

static beams_status build_map_lazy(beams_renderer* r, const ExactGeo& g, int& launches) {
  const size_t nvert = (size_t)g.pd[0] * g.pd[1] * g.pd[2];
  const int nl = g.n_lights > 1 ? g.n_lights : 1;
  const bool prec = r->form == BEAMS_FORM_PRECISION;  // binary16 transmittance
  // the buffer is cleared when its format changes too: float32 data read as
  // binary16 can hold NaN or infinity patterns
  beams_status s = ensure_masked_map(r, &r->d_map, &r->map_cap, nl * nvert * (prec ? 2 : sizeof(float)), r->stream,
                                     r->map_is_half != prec);
  if (s != BEAMS_OK) return s;
  r->map_valid = false;
  r->map_is_half = prec;
  const size_t ncell = (size_t)(g.pd[0] - 1) * (g.pd[1] - 1) * (g.pd[2] - 1);
  s = ensure_buffer(r, (void**)&r->d_cell_mask, &r->cell_mask_cap, ncell, "allocating the map cell mask");
  if (s != BEAMS_OK) return s;
  const unsigned char* occ = nullptr;       // the light march's empty-space skip
  const unsigned char* view_occ = nullptr;  // the marking pass skips as the view march does
  if ((r->empty_skip || r->view_skip) && !g.rect) {
    s = prepare_occupancy(r, g, launches);
    if (s != BEAMS_OK) return s;
    occ = r->empty_skip ? r->d_occ : nullptr;
    view_occ = r->view_skip ? r->d_occ : nullptr;
  }
  s = ensure_buffer(r, (void**)&r->d_vlist, &r->vlist_cap, marked_list_bytes(g.pd),
                    "allocating the map vertex list");
  if (s != BEAMS_OK) return s;
  const float4* quads = (const float4*)r->d_quads;
  // mode 2 keeps the marks while the view's inputs are unchanged (a light
  // orbit around a fixed camera re-marks nothing)
  MarkKey key;
  mark_key(r, g, key);
  cudaError_t e = cudaSuccess;
  if (!(r->keep_marks && r->marks_valid && std::memcmp(&key, &r->mark_key, sizeof(key)) == 0)) {
    r->marks_valid = false;
    e = cudaMemsetAsync(r->d_cell_mask, 0, ncell, r->stream);
    if (e == cudaSuccess)
      e = prec ? launch_mark_view_cells_prec(g, quad_dtype(r), r->d_quads, r->d_tab, r->d_tf, r->d_cell_mask,
                                             r->d_cnt, r->stream, view_occ)
               : launch_mark_view_cells(g, quads, r->d_tab, r->d_tf, r->d_cell_mask, r->d_cnt, nullptr, nullptr,
                                        r->stream, view_occ);
    if (e != cudaSuccess) return cuda_fail(r, e, "map cell marking launch");
    ++launches;
    r->mark_key = key;
    r->marks_valid = r->keep_marks;
  }
  e = launch_list_marked_vertices(g, r->d_cell_mask, nullptr, r->d_vlist, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "map vertex listing launch");
  launches += 2;  // the block pass and the list
  if (prec) {
    e = launch_light_march_prec(g, quad_dtype(r), r->d_quads, r->d_tab, r->d_tf, r->d_tau, (__half*)r->d_map,
                                r->d_cnt, r->stream, occ, r->d_vlist);
    if (e != cudaSuccess) return cuda_fail(r, e, "light_march launch");
    ++launches;
    return BEAMS_OK;
  }
  for (int l = 0; l < nl; ++l) {
    ExactGeo gl = g;
    if (l > 0) geo_set_light(gl, r->lights[l]);
    e = launch_light_march_f32(gl, quads, r->d_tab, r->d_tf, r->d_map + (size_t)l * nvert, r->d_cnt, r->stream,
                               nullptr, 0, -1, nullptr, occ, r->d_vlist);
    if (e != cudaSuccess) return cuda_fail(r, e, "light_march launch");
    ++launches;
  }
  return BEAMS_OK;
}

static beams_status check_sizes(beams_renderer* r, const beams_volume& v) {
  const double nq = (double)(v.dims[0] - 1) * (v.dims[1] - 1) * v.dims[2];
  if (nq >= 4294967296.0) return fail(r, BEAMS_ERR_UNSUPPORTED, "volume too large for 32-bit cell indexing");
  const double nv = (double)(r->map_m[0] + 1) * (r->map_m[1] + 1) * (r->map_m[2] + 1);
  if (nv >= 2147483648.0) return fail(r, BEAMS_ERR_UNSUPPORTED, "shadow map too large (vertices >= 2^31)");
  const int ntab = v.dims[0] + v.dims[1] + v.dims[2] - 3 + r->map_m[0] + r->map_m[1] + r->map_m[2];
  if ((size_t)(ntab + 1024) * 16 > 200 * 1024)
    return fail(r, BEAMS_ERR_UNSUPPORTED, "volume/map axes too long for the shared-memory cell tables");
  return BEAMS_OK;
}

beams_status mlp_set_render_options(beams_renderer* r, const beams_mlp_options* o);
beams_status mlp_render_view(beams_renderer* r, const ExactGeo& g, float4* out, int& launches);
bool mlp_ready(const beams_renderer* r);

beams_status check_ready(beams_renderer* r) {
  if (r->rect && (r->brick_mode || r->form == BEAMS_FORM_MLP || (r->multi_light && r->lights.size() > 1)))
    return fail(r, BEAMS_ERR_UNSUPPORTED,
                "explicit volume coordinates render in the exact and precision forms of a single volume "
                "with one light");
  if (r->multi_light && r->lights.size() > 1) {
    if (r->brick_mode || r->form != BEAMS_FORM_EXACT || (r->has_volume && r->vol.assoc != BEAMS_ASSOC_POINTS))
      return fail(r, BEAMS_ERR_UNSUPPORTED, "several lights render in the exact form of a point volume only");
    if ((int)r->lights.size() > kMaxMultiLights)
      return fail(r, BEAMS_ERR_UNSUPPORTED, "at most 8 lights in the multi-light extension");
  }
  if (r->brick_mode) {
    if (r->bricks.empty()) return fail(r, BEAMS_ERR_STATE, "no bricks set (beams_set_bricks)");
    if (r->tf_n < 1) return fail(r, BEAMS_ERR_STATE, "no colour map set (beams_set_color_map)");
    if (r->use_map && r->lights.empty()) return fail(r, BEAMS_ERR_STATE, "shadow map enabled but no light added");
    if (r->form != BEAMS_FORM_EXACT) return fail(r, BEAMS_ERR_UNSUPPORTED, "bricks render in the exact form only");
    for (auto& b : r->bricks) {
      beams_status s = check_sizes(r, b.vol);
      if (s != BEAMS_OK) return s;
    }
    return BEAMS_OK;
  }
  if (!r->has_volume) return fail(r, BEAMS_ERR_STATE, "no volume set (beams_set_volume)");
  if (r->tf_n < 1) return fail(r, BEAMS_ERR_STATE, "no colour map set (beams_set_color_map)");
  if (r->use_map && r->vol.assoc == BEAMS_ASSOC_POINTS && r->lights.empty())
    return fail(r, BEAMS_ERR_STATE, "shadow map enabled but no light added");
  if (r->form == BEAMS_FORM_EXACT && r->vol.dtype != BEAMS_F32)
    return fail(r, BEAMS_ERR_UNSUPPORTED, "the exact form needs a float32 volume");
  if (r->form == BEAMS_FORM_PRECISION && r->vol.assoc != BEAMS_ASSOC_POINTS)
    return fail(r, BEAMS_ERR_UNSUPPORTED, "the precision form renders point fields");
  if (r->form == BEAMS_FORM_MLP) {
    if (r->vol.dtype != BEAMS_F32 || r->vol.assoc != BEAMS_ASSOC_POINTS)
      return fail(r, BEAMS_ERR_UNSUPPORTED, "the MLP form renders float32 point fields");
    if (!r->use_map) return fail(r, BEAMS_ERR_STATE, "the MLP form shades: enable the shadow map");
  }
  const double nq = (double)(r->vol.dims[0] - 1) * (r->vol.dims[1] - 1) * r->vol.dims[2];
  if (nq >= 4294967296.0) return fail(r, BEAMS_ERR_UNSUPPORTED, "volume too large for 32-bit cell indexing");
  const double nv = (double)(r->map_m[0] + 1) * (r->map_m[1] + 1) * (r->map_m[2] + 1);
  if (nv >= 2147483648.0) return fail(r, BEAMS_ERR_UNSUPPORTED, "shadow map too large (vertices >= 2^31)");
  const int ntab = r->vol.dims[0] + r->vol.dims[1] + r->vol.dims[2] - 3 + r->map_m[0] + r->map_m[1] + r->map_m[2];
  if ((size_t)(ntab + 1024) * 16 > 200 * 1024)
    return fail(r, BEAMS_ERR_UNSUPPORTED, "volume/map axes too long for the shared-memory cell tables");
  return BEAMS_OK;
}

// Side streams, events and per-brick counters of the per-brick launches (created on first use).
static beams_status brick_lanes_ready(beams_renderer* r) {
  cudaError_t e = cudaSuccess;
  if (!r->brick_fork) e = cudaEventCreateWithFlags(&r->brick_fork, cudaEventDisableTiming);
  for (int l = 0; l < beams_renderer::kBrickLanes && e == cudaSuccess; ++l) {
    if (!r->brick_lane[l]) e = cudaStreamCreateWithFlags(&r->brick_lane[l], cudaStreamNonBlocking);
    if (e == cudaSuccess && !r->brick_join[l]) e = cudaEventCreateWithFlags(&r->brick_join[l], cudaEventDisableTiming);
  }
  if (e == cudaSuccess && !r->d_brick_cnt) e = cudaMalloc((void**)&r->d_brick_cnt, kMaxBricks * sizeof(Counters));
  if (e != cudaSuccess) return cuda_fail(r, e, "creating brick streams");
  return BEAMS_OK;
}

// The fork of work onto the lanes: every lane waits for what r->stream has queued so far.
static beams_status brick_lanes_fork(beams_renderer* r) {
  cudaError_t e = cudaEventRecord(r->brick_fork, r->stream);
  for (int l = 0; l < beams_renderer::kBrickLanes && e == cudaSuccess; ++l)
    e = cudaStreamWaitEvent(r->brick_lane[l], r->brick_fork, 0);
  if (e != cudaSuccess) return cuda_fail(r, e, "forking brick streams");
  return BEAMS_OK;
}

// r->stream waits for everything queued on the lanes (called on error paths too).
static cudaError_t brick_lanes_join(beams_renderer* r) {
  cudaError_t first = cudaSuccess;
  for (int l = 0; l < beams_renderer::kBrickLanes; ++l) {
    cudaError_t e = cudaEventRecord(r->brick_join[l], r->brick_lane[l]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(r->stream, r->brick_join[l], 0);
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  }
  return first;
}

// One frame of a multi-block scene: Phase 1 local maps, Phases 2-3 stitched
// maps, Phase 4 per-brick view marches, Phase 5 depth-ordered composite.
// Cell mask of the outer cell layer of a pd[0] x pd[1] x pd[2]-vertex map
// (cells with index 0 or pd-2 on some axis), built on the host once per map
// size: a masked K1 then builds exactly the vertices within one layer of a face.
static beams_status brick_shell_mask(beams_renderer* r, const int pd[3]) {
  if (r->d_shell_mask && std::memcmp(r->shell_pd, pd, sizeof(r->shell_pd)) == 0) return BEAMS_OK;
  const int mx = pd[0] - 1, my = pd[1] - 1, mz = pd[2] - 1;
  std::vector<unsigned char> h((size_t)mx * my * mz);
  for (int z = 0; z < mz; ++z)
    for (int y = 0; y < my; ++y)
      for (int x = 0; x < mx; ++x)
        h[((size_t)z * my + y) * mx + x] =
            (x == 0 || y == 0 || z == 0 || x == mx - 1 || y == my - 1 || z == mz - 1) ? 1 : 0;
  beams_status s = ensure_buffer(r, (void**)&r->d_shell_mask, &r->shell_cap, h.size(), "allocating the shell mask");
  if (s != BEAMS_OK) return s;
  cudaError_t e = cudaMemcpyAsync(r->d_shell_mask, h.data(), h.size(), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);  // h goes out of scope
  if (e != cudaSuccess) return cuda_fail(r, e, "copying the shell mask");
  std::memcpy(r->shell_pd, pd, sizeof(r->shell_pd));
  return BEAMS_OK;
}

// Within a phase the bricks' launches are independent and run on the lanes;
// the phases are joined on r->stream (Phase 3 reads every Phase-1 map, Phase 5
// every brick image).
beams_status render_bricks(beams_renderer* r, const beams_camera* cam, float4* out, int& launches) {
  const int nb = (int)r->bricks.size();
  std::vector<ExactGeo> G(nb);
  for (int b = 0; b < nb; ++b) {
    Brick& B = r->bricks[b];
    beams_status s = make_geo_vol(r, B.vol, cam, G[b]);
    if (s != BEAMS_OK) return s;
    s = prepare_layouts_for(r, G[b], B.vol.assoc, B.d_field, B.version, &B.d_tab, &B.tab_cap, B.tab_key,
                            &B.d_quads, &B.quads_cap, &B.quads_version, launches);
    if (s != BEAMS_OK) return s;
  }
  const size_t npix = (size_t)cam->width * cam->height;
  beams_status s = ensure_buffer(r, (void**)&r->d_brick_imgs, &r->brick_imgs_cap, (size_t)nb * npix * sizeof(float4),
                                 "allocating brick images");
  if (s != BEAMS_OK) return s;
  cudaError_t e;
  s = brick_lanes_ready(r);
  if (s != BEAMS_OK) return s;
  e = cudaMemsetAsync(r->d_brick_cnt, 0, nb * sizeof(Counters), r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "clearing brick counters");
  auto lane = [&](int b) { return r->brick_lane[b % beams_renderer::kBrickLanes]; };
  const bool lazy = r->lazy_map && r->use_map;
  auto lane_fail = [&](cudaError_t err, const char* what) {
    brick_lanes_join(r);
    return cuda_fail(r, err, what);
  };
  if (r->use_map) {
    std::vector<BrickRef> refs(nb);
    for (int b = 0; b < nb; ++b) {
      Brick& B = r->bricks[b];
      const size_t nv = (size_t)G[b].pd[0] * G[b].pd[1] * G[b].pd[2];
      s = ensure_buffer(r, (void**)&B.d_map_local, &B.local_cap, nv * sizeof(float), "allocating brick map");
      if (s == BEAMS_OK) s = ensure_masked_map(r, &B.d_map_final, &B.final_cap, nv * sizeof(float), r->stream, false);
      if (s != BEAMS_OK) return s;
      B.map_count = nv;
      BrickRef& R = refs[b];
      for (int d = 0; d < 3; ++d) {
        R.bmin[d] = G[b].bmin[d];
        R.bmax[d] = G[b].bmax[d];
        R.morig[d] = G[b].morig[d];
        R.msp[d] = G[b].msp[d];
        R.minv[d] = G[b].minv[d];
        R.pd[d] = G[b].pd[d];
      }
      R.map = B.d_map_local;
    }
    s = ensure_buffer(r, (void**)&r->d_refs, &r->refs_cap, nb * sizeof(BrickRef), "allocating brick table");
    if (s != BEAMS_OK) return s;
    e = cudaMemcpyAsync(r->d_refs, refs.data(), nb * sizeof(BrickRef), cudaMemcpyHostToDevice, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "copying brick table");
    // Phase 1: local maps. The stitch reads them only at segment exit points on
    // brick faces, so when no two bricks overlap only the vertices within one
    // layer of a face are built (the 512^3 field as 2x2x2 bricks: 7.10 ->
    // 5.40 ms per frame; the stitched maps and the image are the same).
    bool disjoint = true;
    for (int a = 0; a < nb && disjoint; ++a)
      for (int b = a + 1; b < nb && disjoint; ++b) {
        bool inside = true;
        for (int d = 0; d < 3; ++d)
          inside = inside && G[a].bmin[d] < G[b].bmax[d] && G[b].bmin[d] < G[a].bmax[d];
        disjoint = !inside;
      }
    // the outer cell layer marked: its corners are those vertices (one mask for
    // every brick, the map size is shared)
    const unsigned char* shell = nullptr;
    if (disjoint && nb > 1) {
      s = brick_shell_mask(r, G[0].pd);
      if (s != BEAMS_OK) return s;
      shell = r->d_shell_mask;
    }
    // the shell's vertices listed once (the bricks' maps share their size)
    const unsigned* shell_list = nullptr;
    r->shell_listed = shell != nullptr;
    if (shell) {
      s = ensure_buffer(r, (void**)&r->d_vlist, &r->vlist_cap, marked_list_bytes(G[0].pd),
                        "allocating the map vertex list");
      if (s != BEAMS_OK) return s;
      e = launch_list_marked_vertices(G[0], shell, nullptr, r->d_vlist, r->stream);
      if (e != cudaSuccess) return cuda_fail(r, e, "listing the shell vertices");
      launches += 2;  // the block pass and the list
      shell_list = r->d_vlist;
    }
    s = brick_lanes_fork(r);
    if (s != BEAMS_OK) return s;
    for (int b = 0; b < nb; ++b) {
      Brick& B = r->bricks[b];
      e = launch_light_march_f32(G[b], B.d_quads, B.d_tab, r->d_tf, B.d_map_local, r->d_brick_cnt + b, lane(b),
                                 nullptr, 0, -1, nullptr, nullptr, shell_list);
      if (e != cudaSuccess) return lane_fail(e, "brick light march");
      ++launches;
    }
    e = brick_lanes_join(r);
    if (e != cudaSuccess) return cuda_fail(r, e, "joining brick streams");
    // Phases 2-3: stitched maps (each reads every brick's Phase-1 map)
    // The lazy map: each brick's view rays (their limits and pixel window as in
    // Phase 4) mark the cells of its map they read, and the stitched march
    // builds only those cells' corners; a brick no pixel reaches needs none.
    bool reached[kMaxBricks];
    if (lazy) {
      s = prepare_ray_limits(r, G[0], launches);
      if (s != BEAMS_OK) return s;
      for (int b = 0; b < nb; ++b) {
        G[b].ray_max = G[0].ray_max;
        reached[b] = brick_window(G[b], G[b].win);
        Brick& B = r->bricks[b];
        const size_t ncell = (size_t)(G[b].pd[0] - 1) * (G[b].pd[1] - 1) * (G[b].pd[2] - 1);
        s = ensure_buffer(r, (void**)&B.d_cell_mask, &B.cell_mask_cap, ncell, "allocating a brick's cell mask");
        if (s == BEAMS_OK)
          s = ensure_buffer(r, (void**)&B.d_vlist, &B.vlist_cap, marked_list_bytes(G[b].pd),
                            "allocating a brick's vertex list");
        if (s != BEAMS_OK) return s;
      }
    }
    s = brick_lanes_fork(r);
    if (s != BEAMS_OK) return s;
    for (int b = 0; b < nb; ++b) {
      Brick& B = r->bricks[b];
      B.final_partial = lazy;
      const unsigned* list = nullptr;
      if (lazy) {
        if (!reached[b]) continue;
        // mode 2 keeps a brick's marks while its view's inputs are unchanged
        MarkKey key;
        mark_key(r, G[b], key);
        key.volume_version = B.version;
        if (!(r->keep_marks && B.marks_valid && std::memcmp(&key, &B.mark_key, sizeof(key)) == 0)) {
          B.marks_valid = false;
          const size_t ncell = (size_t)(G[b].pd[0] - 1) * (G[b].pd[1] - 1) * (G[b].pd[2] - 1);
          e = cudaMemsetAsync(B.d_cell_mask, 0, ncell, lane(b));
          if (e == cudaSuccess)
            e = launch_mark_view_cells(G[b], B.d_quads, B.d_tab, r->d_tf, B.d_cell_mask, r->d_brick_cnt + b,
                                       nullptr, nullptr, lane(b));
          if (e != cudaSuccess) return lane_fail(e, "brick map cell marking");
          ++launches;
          B.mark_key = key;
          B.marks_valid = r->keep_marks;
        }
        e = launch_list_marked_vertices(G[b], B.d_cell_mask, nullptr, B.d_vlist, lane(b));
        if (e != cudaSuccess) return lane_fail(e, "brick map vertex listing");
        launches += 2;  // the block pass and the list
        list = B.d_vlist;
      }
      e = launch_light_march_f32(G[b], B.d_quads, B.d_tab, r->d_tf, B.d_map_final, r->d_brick_cnt + b, lane(b),
                                 r->d_refs, nb, b, nullptr, nullptr, list);
      if (e != cudaSuccess) return lane_fail(e, "brick stitch march");
      ++launches;
    }
    e = brick_lanes_join(r);
    if (e != cudaSuccess) return cuda_fail(r, e, "joining brick streams");
  }
  cudaEventRecord(r->ev[1], r->stream);
  if (!lazy) {
    s = prepare_ray_limits(r, G[0], launches);  // one camera: the same limits for every brick
    if (s != BEAMS_OK) return s;
    for (int b = 1; b < nb; ++b) G[b].ray_max = G[0].ray_max;
  }
  // Phase 4: view marches
  s = brick_lanes_fork(r);
  if (s != BEAMS_OK) return s;
  for (int b = 0; b < nb; ++b) {
    Brick& B = r->bricks[b];
    float4* img = r->d_brick_imgs + (size_t)b * npix;
    // only the pixels whose rays can reach this brick are marched; the rest stay transparent
    const bool any = brick_window(G[b], G[b].win);
    if (!any || (size_t)G[b].win[2] * G[b].win[3] < npix) {
      e = cudaMemsetAsync(img, 0, npix * sizeof(float4), lane(b));
      if (e != cudaSuccess) return lane_fail(e, "clearing brick image");
      if (!any) continue;
    }
    e = launch_view_march_f32(G[b], (const float*)B.d_field, B.d_quads, B.d_tab, r->d_tf,
                              r->use_map ? B.d_map_final : nullptr, img, r->d_brick_cnt + b, lane(b));
    if (e != cudaSuccess) return lane_fail(e, "brick view march");
    ++launches;
  }
  e = brick_lanes_join(r);
  if (e != cudaSuccess) return cuda_fail(r, e, "joining brick streams");
  cudaEventRecord(r->ev[2], r->stream);
  // Depth order: |camera - block centre| in float (MapperLightedVolume.cxx:221-241).
  std::vector<std::pair<float, int>> order;
  const float cp[3] = {(float)cam->position[0], (float)cam->position[1], (float)cam->position[2]};
  for (int b = 0; b < nb; ++b) {
    float c3[3];
    for (int d = 0; d < 3; ++d) c3[d] = (float)((G[b].bmin[d] + G[b].bmax[d]) * 0.5);
    const float dx = cp[0] - c3[0], dy = cp[1] - c3[1], dz = cp[2] - c3[2];
    order.push_back({std::sqrt(dx * dx + dy * dy + dz * dz), b});
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<float, int>& l, const std::pair<float, int>& q) { return l.first < q.first; });
  int idx[kMaxBricks];
  for (int b = 0; b < nb; ++b) idx[b] = order[b].second;
  e = launch_composite(r->d_brick_imgs, nb, npix, idx, out, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "brick composite");
  ++launches;
  return BEAMS_OK;
}

// beams_render for a multi-block scene: output handling and timings around render_bricks.
beams_status render_bricks_frame(beams_renderer* r, const beams_camera* cam, float* rgba_out, int out_on_device,
                                 beams_timings* t, int& launches) {
  const size_t npix = (size_t)cam->width * cam->height;
  float4* dst = (float4*)rgba_out;
  const bool direct = out_on_device == BEAMS_OUT_DEVICE && (((uintptr_t)rgba_out & 15) == 0);
  beams_status s;
  if (!direct) {
    s = ensure_buffer(r, (void**)&r->d_rgba, &r->rgba_cap, npix * sizeof(float4), "allocating image");
    if (s != BEAMS_OK) return s;
    dst = r->d_rgba;
  }
  s = render_bricks(r, cam, dst, launches);
  if (s != BEAMS_OK) return s;
  s = blend_background(r, dst, npix, launches);
  if (s != BEAMS_OK) return s;
  cudaError_t e;
  if (!direct) {
    e = cudaMemcpyAsync(rgba_out, dst, npix * sizeof(float4),
                        out_on_device == BEAMS_OUT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "copying image out");
  }
  cudaEventRecord(r->ev[3], r->stream);
  if (t) {
    std::memset(t, 0, sizeof(*t));
    e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "render");
    // the frame's counters plus every brick's (the per-brick launches count into their own)
    std::vector<Counters> c(1 + r->bricks.size());
    e = cudaMemcpy(c.data(), r->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(c.data() + 1, r->d_brick_cnt, r->bricks.size() * sizeof(Counters), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(r, e, "reading counters");
    cudaEventElapsedTime(&t->map_build_ms, r->ev[0], r->ev[1]);
    cudaEventElapsedTime(&t->view_march_ms, r->ev[1], r->ev[2]);
    cudaEventElapsedTime(&t->composite_ms, r->ev[2], r->ev[3]);
    cudaEventElapsedTime(&t->total_ms, r->ev[0], r->ev[3]);
    for (const Counters& k : c) {
      t->light_samples += k.light_samples;
      t->lit_samples += k.lit_samples;
      t->rays_hit += k.rays_hit;
    }
    // the stitched maps' vertices (Phase 1 is not counted); under the lazy map
    // the listed ones: the masked builds count what they build, Phase 1's
    // shell list (its length in the list's first entry) included, so that is
    // taken off once per brick
    size_t nv = 0;
    if (r->lazy_map && r->use_map) {
      for (size_t b = 1; b < c.size(); ++b) nv += c[b].map_vertices;
      if (r->shell_listed) {
        unsigned shell_n = 0;
        e = cudaMemcpy(&shell_n, r->d_vlist, sizeof(unsigned), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(r, e, "reading the shell list length");
        nv -= (size_t)shell_n * r->bricks.size();
      }
    } else {
      for (auto& b : r->bricks) nv += r->use_map ? b.map_count : 0;
    }
    t->map_vertices = (int)nv;
    t->kernel_launches = launches;
  } else if (out_on_device == BEAMS_OUT_HOST) {
    e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "render");
  }
  return BEAMS_OK;
}

}  // namespace beams

using namespace beams;

// ---------------------------------------------------------------------------
extern "C" {

int beams_abi_version(void) { return BEAMS_ABI_VERSION; }

const char* beams_last_error(const beams_renderer* r) {
  return r ? r->err.c_str() : g_tls_error.c_str();
}

beams_status beams_create(beams_renderer** out, int device, void* stream) {
  if (!out) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "device index out of range");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
  beams_renderer* r = new beams_renderer();
  r->device = device;
  r->stream = (cudaStream_t)stream;
  for (int i = 0; i < 4; ++i) {
    e = cudaEventCreate(&r->ev[i]);
    if (e != cudaSuccess) {
      delete r;
      return cuda_fail(nullptr, e, "cudaEventCreate");
    }
  }
  e = cudaMalloc((void**)&r->d_cnt, 2 * sizeof(Counters));  // [1]: the learned form's fallback pass
  if (e != cudaSuccess) {
    delete r;
    return cuda_fail(nullptr, e, "allocating counters");
  }
  e = cudaMemset(r->d_cnt, 0, 2 * sizeof(Counters));
  if (e != cudaSuccess) {
    delete r;
    return cuda_fail(nullptr, e, "clearing counters");
  }
  *out = r;
  return BEAMS_OK;
}

beams_status beams_destroy(beams_renderer* r) {
  if (!r) return BEAMS_OK;
  cudaSetDevice(r->device);
  cudaStreamSynchronize(r->stream);
  delete r;
  return BEAMS_OK;
}

beams_status beams_set_volume(beams_renderer* r, const beams_volume* v) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!v || !v->data) return fail(r, BEAMS_ERR_INVALID_ARG, "volume or volume data is NULL");
  if (v->dtype != BEAMS_F32 && v->dtype != BEAMS_BF16 && v->dtype != BEAMS_F16)
    return fail(r, BEAMS_ERR_INVALID_ARG, "volume dtype must be F32, BF16 or F16");
  if (v->assoc != BEAMS_ASSOC_POINTS && v->assoc != BEAMS_ASSOC_CELLS)
    return fail(r, BEAMS_ERR_INVALID_ARG, "volume assoc must be POINTS or CELLS");
  for (int d = 0; d < 3; ++d) {
    if (v->dims[d] < 2 || v->dims[d] > 8192)
      return fail(r, BEAMS_ERR_INVALID_ARG, "volume dims must be in [2, 8192] (point dimensions)");
    if (!(v->spacing[d] > 0.0) || !std::isfinite(v->spacing[d]) || !std::isfinite(v->origin[d]))
      return fail(r, BEAMS_ERR_INVALID_ARG, "volume spacing must be positive and finite");
  }
  if (!std::isfinite(v->range[0]) || !std::isfinite(v->range[1]))
    return fail(r, BEAMS_ERR_INVALID_ARG, "volume range must be finite");
  cudaSetDevice(r->device);
  const size_t elem = (v->dtype == BEAMS_F32) ? 4 : 2;
  size_t count = (size_t)v->dims[0] * v->dims[1] * v->dims[2];
  if (v->assoc == BEAMS_ASSOC_CELLS) count = (size_t)(v->dims[0] - 1) * (v->dims[1] - 1) * (v->dims[2] - 1);
  const size_t bytes = count * elem;
  if (v->on_device) {
    r->d_field = v->data;
  } else {
    beams_status s = ensure_buffer(r, &r->d_field_owned, &r->field_cap, bytes, "allocating volume");
    if (s != BEAMS_OK) return s;
    cudaError_t e = cudaMemcpyAsync(r->d_field_owned, v->data, bytes, cudaMemcpyHostToDevice, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "copying volume to device");
    r->d_field = r->d_field_owned;
  }
  r->vol = *v;
  r->vol.data = r->d_field;
  r->vol.on_device = 1;
  r->field_bytes = bytes;
  r->has_volume = true;
  r->brick_mode = false;
  r->rect = false;  // a new volume is uniform until beams_set_volume_coordinates
  ++r->volume_version;
  return BEAMS_OK;
}

beams_status beams_set_volume_coordinates(beams_renderer* r, const float* x, const float* y, const float* z) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!x && !y && !z) {
    if (r->rect) ++r->volume_version;
    r->rect = false;
    return BEAMS_OK;
  }
  if (!x || !y || !z) return fail(r, BEAMS_ERR_INVALID_ARG, "volume coordinates: give all three axes or none");
  if (!r->has_volume) return fail(r, BEAMS_ERR_STATE, "volume coordinates: set a volume first (beams_set_volume)");
  const float* a[3] = {x, y, z};
  for (int d = 0; d < 3; ++d) {
    const int n = r->vol.dims[d];
    for (int i = 0; i < n; ++i)
      if (!std::isfinite(a[d][i]) || (i > 0 && !(a[d][i] > a[d][i - 1])))
        return fail(r, BEAMS_ERR_INVALID_ARG, "volume coordinates must be finite and strictly increasing");
  }
  for (int d = 0; d < 3; ++d) r->coords[d].assign(a[d], a[d] + r->vol.dims[d]);
  r->rect = true;
  ++r->volume_version;  // new cell tables, occupancy and map
  return BEAMS_OK;
}

beams_status beams_set_color_map(beams_renderer* r, const float* rgba, int n) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!rgba || n < 1 || n > 1024) return fail(r, BEAMS_ERR_INVALID_ARG, "colour map needs 1..1024 RGBA entries");
  for (int i = 0; i < 4 * n; ++i)
    if (!std::isfinite(rgba[i])) return fail(r, BEAMS_ERR_INVALID_ARG, "colour map has a non-finite entry");
  cudaSetDevice(r->device);
  r->tf.assign(rgba, rgba + 4 * n);
  beams_status s = ensure_buffer(r, (void**)&r->d_tf, &r->tf_cap, sizeof(float) * 4 * 1024, "allocating colour map");
  if (s != BEAMS_OK) return s;
  cudaError_t e = cudaMemcpyAsync(r->d_tf, r->tf.data(), sizeof(float) * 4 * n, cudaMemcpyHostToDevice, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "copying colour map");
  // -ln(1 - a_i) per entry for the precision form's optical depth, a_i = alpha /
  // max alpha in float32 as the light march forms it; a_i = 1 -> +inf (a cut).
  {
    float ma = 0.f;
    for (int i = 0; i < n; ++i) ma = (ma < rgba[4 * i + 3]) ? rgba[4 * i + 3] : ma;
    r->tau.assign(n, 0.f);
    for (int i = 0; i < n; ++i) {
      const float a = (ma > 0.f) ? rgba[4 * i + 3] / ma : 0.f;
      r->tau[i] = (a >= 1.f) ? INFINITY : (float)(-std::log1p(-(double)a));
    }
    s = ensure_buffer(r, (void**)&r->d_tau, &r->tau_cap, sizeof(float) * 1024, "allocating tau table");
    if (s != BEAMS_OK) return s;
    e = cudaMemcpyAsync(r->d_tau, r->tau.data(), sizeof(float) * n, cudaMemcpyHostToDevice, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "copying tau table");
  }
  r->tf_n = n;
  ++r->tf_version;
  return BEAMS_OK;
}

beams_status beams_set_shadow_map_size(beams_renderer* r, int mx, int my, int mz) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (mx < 1 || my < 1 || mz < 1 || mx > 2047 || my > 2047 || mz > 2047)
    return fail(r, BEAMS_ERR_INVALID_ARG, "shadow map size must be in [1, 2047] cells per axis");
  r->map_m[0] = mx;
  r->map_m[1] = my;
  r->map_m[2] = mz;
  return BEAMS_OK;
}

beams_status beams_set_use_shadow_map(beams_renderer* r, int enable) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->use_map = enable != 0;
  return BEAMS_OK;
}

beams_status beams_clear_lights(beams_renderer* r) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->lights.clear();
  return BEAMS_OK;
}

static beams_status add_light(beams_renderer* r, int kind, const double v[3], const float color[3], float intensity) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!v || !color || !finite3(v) || !std::isfinite(intensity) || !std::isfinite(color[0]) ||
      !std::isfinite(color[1]) || !std::isfinite(color[2]))
    return fail(r, BEAMS_ERR_INVALID_ARG, "light: non-finite or NULL argument");
  if (kind == 1 && v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0)
    return fail(r, BEAMS_ERR_INVALID_ARG, "directional light: zero direction");
  Light L;
  L.kind = kind;
  for (int d = 0; d < 3; ++d) {
    L.v[d] = v[d];
    L.color[d] = color[d];
  }
  L.intensity = intensity;
  r->lights.push_back(L);
  return BEAMS_OK;
}

beams_status beams_add_point_light(beams_renderer* r, const double pos[3], const float color[3], float intensity) {
  return add_light(r, 0, pos, color, intensity);
}

beams_status beams_add_directional_light(beams_renderer* r, const double dir[3], const float color[3],
                                         float intensity) {
  return add_light(r, 1, dir, color, intensity);
}

beams_status beams_set_sample_distance(beams_renderer* r, float d) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!(d > 0.f) || !std::isfinite(d)) return fail(r, BEAMS_ERR_INVALID_ARG, "Sample distance must be positive.");
  r->sample_distance = d;
  return BEAMS_OK;
}

beams_status beams_set_density_scale(beams_renderer* r, float scale) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->density_scale = scale;
  return BEAMS_OK;
}

beams_status beams_get_density_scale(const beams_renderer* r, float* scale) {
  if (!r || !scale) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "get_density_scale: NULL argument");
  *scale = r->density_scale;
  return BEAMS_OK;
}

beams_status beams_set_termination_alpha(beams_renderer* r, float a) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!(a > 0.f) || !std::isfinite(a)) return fail(r, BEAMS_ERR_INVALID_ARG, "termination alpha must be positive");
  r->cutoff = a;
  return BEAMS_OK;
}

beams_status beams_set_light_steps(beams_renderer* r, float steps) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!(steps >= 1.f && steps <= 65536.f)) return fail(r, BEAMS_ERR_INVALID_ARG, "light steps must be in [1, 65536]");
  r->light_steps = steps;
  return BEAMS_OK;
}

beams_status beams_set_slab_fp64(beams_renderer* r, int enable) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->slab_fp64 = enable != 0;
  return BEAMS_OK;
}

beams_status beams_set_multi_light(beams_renderer* r, int enable) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->multi_light = enable != 0;
  return BEAMS_OK;
}

beams_status beams_test_fail_allocation(int nth) {
  if (nth < 0) return BEAMS_ERR_INVALID_ARG;
  g_fail_alloc_in.store(nth);
  return BEAMS_OK;
}

beams_status beams_set_tuning(beams_renderer* r, const beams_tuning* t) {
  if (!r || !t) return fail(r, BEAMS_ERR_INVALID_ARG, "set_tuning: NULL argument");
  int lb = 0;
  switch (t->light_brick) {
    case 0: lb = 0; break;
    case 8: lb = 3; break;
    case 16: lb = 4; break;
    case 32: lb = 5; break;
    case 64: lb = 6; break;
    default: return fail(r, BEAMS_ERR_INVALID_ARG, "set_tuning: light_brick must be 0, 8, 16, 32 or 64");
  }
  r->light_brick_log2 = lb;
  r->empty_skip = t->no_empty_skip ? 0 : 1;
  r->view_skip = t->no_view_skip ? 0 : 1;
  return BEAMS_OK;
}

beams_status beams_get_tuning(beams_renderer* r, beams_tuning* t) {
  if (!r || !t) return fail(r, BEAMS_ERR_INVALID_ARG, "get_tuning: NULL argument");
  std::memset(t, 0, sizeof(*t));
  t->light_brick = r->light_brick_log2 ? 1 << r->light_brick_log2 : 0;
  t->no_empty_skip = r->empty_skip ? 0 : 1;
  t->no_view_skip = r->view_skip ? 0 : 1;
  return BEAMS_OK;
}

beams_status beams_set_reuse_shadow_map(beams_renderer* r, int enable) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->reuse_map = enable != 0;
  return BEAMS_OK;
}

beams_status beams_set_lazy_shadow_map(beams_renderer* r, int mode) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (mode < 0 || mode > 2) return fail(r, BEAMS_ERR_INVALID_ARG, "lazy shadow map mode must be 0, 1 or 2");
  r->lazy_map = mode != 0;
  r->keep_marks = mode == 2;  // kept marks stay valid only while their key matches
  return BEAMS_OK;
}

beams_status beams_set_background(beams_renderer* r, int enable, const float rgba[4]) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->bg = enable != 0;
  if (rgba)
    for (int i = 0; i < 4; ++i) r->bg_rgba[i] = rgba[i];
  return BEAMS_OK;
}

beams_status beams_set_form(beams_renderer* r, int form, const void* opts) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (form == BEAMS_FORM_EXACT) {
    r->form = form;
    return BEAMS_OK;
  }
  if (form == BEAMS_FORM_MLP) {
    beams_status s = mlp_set_render_options(r, (const beams_mlp_options*)opts);
    if (s != BEAMS_OK) return s;
    r->form = form;
    return BEAMS_OK;
  }
  if (form == BEAMS_FORM_PRECISION) {
    int dt = BEAMS_BF16;
    if (opts) dt = ((const beams_precision_options*)opts)->field_dtype;
    if (dt != BEAMS_BF16 && dt != BEAMS_F16)
      return fail(r, BEAMS_ERR_INVALID_ARG, "precision form: field_dtype must be BEAMS_BF16 or BEAMS_F16");
    r->form = form;
    r->prec_dtype = dt;
    return BEAMS_OK;
  }
  return fail(r, BEAMS_ERR_UNSUPPORTED, "form not available in this build");
}

beams_status beams_build_shadow_map(beams_renderer* r, beams_timings* t) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  beams_status s = check_ready(r);
  if (s != BEAMS_OK) return s;
  if (r->lights.empty()) return fail(r, BEAMS_ERR_STATE, "no light added");
  cudaSetDevice(r->device);
  ExactGeo g;
  s = make_geo(r, nullptr, g);
  if (s != BEAMS_OK) return s;
  cudaError_t e = cudaMemsetAsync(r->d_cnt, 0, sizeof(Counters), r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "clearing counters");
  cudaEventRecord(r->ev[0], r->stream);
  int launches = 0;
  bool built = false;
  s = prepare_layouts(r, g, launches);
  if (s != BEAMS_OK) return s;
  const bool keep = r->reuse_map;
  r->reuse_map = false;
  s = build_map(r, g, launches, built);
  r->reuse_map = keep;
  if (s != BEAMS_OK) return s;
  cudaEventRecord(r->ev[1], r->stream);
  if (t) {
    std::memset(t, 0, sizeof(*t));
    e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "light march");
    Counters c;
    e = cudaMemcpy(&c, r->d_cnt, sizeof(c), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(r, e, "reading counters");
    cudaEventElapsedTime(&t->map_build_ms, r->ev[0], r->ev[1]);
    t->total_ms = t->map_build_ms;
    t->light_samples = c.light_samples;
    t->map_vertices = built ? (int)r->map_count : 0;
    t->kernel_launches = launches;
  }
  return BEAMS_OK;
}

beams_status beams_autotune(beams_renderer* r, const beams_camera* cam, beams_tuning* best, float* best_map_ms,
                            float* best_view_ms) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  beams_status s = check_ready(r);
  if (s != BEAMS_OK) return s;
  if (r->lights.empty()) return fail(r, BEAMS_ERR_STATE, "no light added");
  if (r->brick_mode || r->vol.assoc != BEAMS_ASSOC_POINTS || r->form == BEAMS_FORM_MLP)
    return fail(r, BEAMS_ERR_UNSUPPORTED, "autotune: single point volume in the exact or precision form");
  cudaSetDevice(r->device);
  ExactGeo g;
  s = make_geo(r, nullptr, g);
  if (s != BEAMS_OK) return s;
  int launches = 0;
  s = prepare_layouts(r, g, launches);
  if (s != BEAMS_OK) return s;
  const int keep_lb = r->light_brick_log2, keep_skip = r->empty_skip;
  const bool keep_reuse = r->reuse_map;
  r->reuse_map = false;
  int best_lb = keep_lb, best_skip = keep_skip;
  float best_t = 3.4e38f;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  for (int lb : {0, 3, 4, 5, 6}) {
    for (int skip : {0, 1}) {
      r->light_brick_log2 = lb;
      r->empty_skip = skip;
      s = make_geo(r, nullptr, g);
      bool built = false;
      if (s == BEAMS_OK) s = build_map(r, g, launches, built);  // warm-up (and the occupancy grid)
      float tmin = 3.4e38f;
      for (int rep = 0; rep < 2 && s == BEAMS_OK; ++rep) {
        cudaEventRecord(a, r->stream);
        s = build_map(r, g, launches, built);
        cudaEventRecord(b, r->stream);
        cudaError_t e = cudaEventSynchronize(b);
        if (e != cudaSuccess) s = cuda_fail(r, e, "autotune");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        tmin = std::min(tmin, ms);
      }
      if (s != BEAMS_OK) break;
      if (tmin < best_t) {
        best_t = tmin;
        best_lb = lb;
        best_skip = skip;
      }
    }
    if (s != BEAMS_OK) break;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  r->reuse_map = keep_reuse;
  r->map_valid = false;
  if (s != BEAMS_OK) {
    r->light_brick_log2 = keep_lb;
    r->empty_skip = keep_skip;
    return s;
  }
  r->light_brick_log2 = best_lb;
  r->empty_skip = best_skip;
  float best_v = 0.f;
  if (cam) {
    // the view march with and without its skip, on the map just chosen
    const int keep_view = r->view_skip;
    const bool keep_reuse2 = r->reuse_map, keep_lazy = r->lazy_map;
    r->reuse_map = true;  // the first render of each choice builds the map; the timed ones reuse it
    r->lazy_map = false;  // (a lazy frame would mark and build again)
    float tv[2] = {3.4e38f, 3.4e38f};
    float4* img = nullptr;
    s = validate_camera(r, cam);
    if (s == BEAMS_OK) {
      const size_t npix = (size_t)cam->width * cam->height;
      s = ensure_buffer(r, (void**)&r->d_rgba, &r->rgba_cap, npix * sizeof(float4), "allocating image");
      img = r->d_rgba;
    }
    for (int vs = 0; vs < 2 && s == BEAMS_OK; ++vs) {
      r->view_skip = vs;
      for (int rep = 0; rep < 3 && s == BEAMS_OK; ++rep) {
        cudaEvent_t a2, b2;
        cudaEventCreate(&a2);
        cudaEventCreate(&b2);
        cudaEventRecord(a2, r->stream);
        s = beams_render(r, cam, (float*)img, 1, nullptr);
        cudaEventRecord(b2, r->stream);
        cudaError_t e = cudaEventSynchronize(b2);
        if (e != cudaSuccess && s == BEAMS_OK) s = cuda_fail(r, e, "autotune");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a2, b2);
        cudaEventDestroy(a2);
        cudaEventDestroy(b2);
        if (rep > 0) tv[vs] = std::min(tv[vs], ms);
      }
    }
    r->reuse_map = keep_reuse2;
    r->lazy_map = keep_lazy;
    if (s != BEAMS_OK) {
      r->view_skip = keep_view;
      return s;
    }
    r->view_skip = tv[1] < tv[0] ? 1 : 0;
    best_v = std::min(tv[0], tv[1]);
  }
  if (best) beams_get_tuning(r, best);
  if (best_map_ms) *best_map_ms = best_t;
  if (best_view_ms) *best_view_ms = best_v;
  return BEAMS_OK;
}

beams_status beams_get_shadow_map(beams_renderer* r, float* dst, size_t count, int dst_on_device) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!r->map_valid) return fail(r, BEAMS_ERR_STATE, "no map has been built");
  if (!dst || count < r->map_count) return fail(r, BEAMS_ERR_INVALID_ARG, "destination too small for the map");
  cudaSetDevice(r->device);
  if (r->map_is_half) {
    // precision form: binary16 transmittance, widened to float on the host
    if (dst_on_device) return fail(r, BEAMS_ERR_UNSUPPORTED, "precision-form maps are copied to the host only");
    std::vector<__half> h(r->map_count);
    cudaError_t e = cudaMemcpyAsync(h.data(), r->d_map, r->map_count * 2, cudaMemcpyDeviceToHost, r->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "copying map");
    for (size_t i = 0; i < r->map_count; ++i) dst[i] = __half2float(h[i]);
    return BEAMS_OK;
  }
  cudaError_t e = cudaMemcpyAsync(dst, r->d_map, r->map_count * sizeof(float),
                                  dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "copying map");
  return BEAMS_OK;
}

static beams_status render_frame(beams_renderer* r, const beams_camera* cam, float* rgba_out, int out_on_device,
                                 beams_timings* t);

beams_status beams_set_profiler(beams_renderer* r, beams_profile_fn fn, void* user) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  r->profile_fn = fn;
  r->profile_user = fn ? user : nullptr;
  return BEAMS_OK;
}

beams_status beams_render(beams_renderer* r, const beams_camera* cam, float* rgba_out, int out_on_device,
                          beams_timings* t) {
  if (!r || !r->profile_fn) return render_frame(r, cam, rgba_out, out_on_device, t);
  // a profiler needs the frame's event times: take the timings path
  beams_timings local{};
  beams_timings* tt = t ? t : &local;
  const beams_status s = render_frame(r, cam, rgba_out, out_on_device, tt);
  if (s != BEAMS_OK) return s;
  r->profile_fn(r->profile_user, "Render", 0, tt->total_ms);
  r->profile_fn(r->profile_user, r->brick_mode ? "Phases 1-3" : "Phase 1", 1, tt->map_build_ms);
  r->profile_fn(r->profile_user, "Phase 4", 1, tt->view_march_ms);
  r->profile_fn(r->profile_user, "Phase 5", 1, tt->composite_ms);
  return BEAMS_OK;
}

static beams_status render_frame(beams_renderer* r, const beams_camera* cam, float* rgba_out, int out_on_device,
                                 beams_timings* t) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  beams_status s = validate_camera(r, cam);
  if (s != BEAMS_OK) return s;
  if (!rgba_out) return fail(r, BEAMS_ERR_INVALID_ARG, "rgba_out is NULL");
  if (out_on_device < BEAMS_OUT_HOST || out_on_device > BEAMS_OUT_HOST_ASYNC)
    return fail(r, BEAMS_ERR_INVALID_ARG, "out_on_device must be BEAMS_OUT_HOST, _DEVICE or _HOST_ASYNC");
  s = check_ready(r);
  if (s != BEAMS_OK) return s;
  cudaSetDevice(r->device);
  ExactGeo g;
  s = make_geo_vol(r, r->brick_mode ? r->bricks[0].vol : r->vol, cam, g);
  if (s != BEAMS_OK) return s;
  int launches = 0;
  cudaError_t e = cudaMemsetAsync(r->d_cnt, 0, 2 * sizeof(Counters), r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "clearing counters");
  cudaEventRecord(r->ev[0], r->stream);
  bool built = false;
  if (r->brick_mode) return render_bricks_frame(r, cam, rgba_out, out_on_device, t, launches);
  s = prepare_layouts(r, g, launches);
  if (s != BEAMS_OK) return s;
  const bool use_mlp = r->form == BEAMS_FORM_MLP;
  const bool need_map = r->use_map && r->vol.assoc == BEAMS_ASSOC_POINTS && !use_mlp;
  const bool lazy = need_map && r->lazy_map && (r->form == BEAMS_FORM_EXACT || r->form == BEAMS_FORM_PRECISION);
  if (lazy) {
    // the marking pass clips rays to the canvas depth like the view march
    s = prepare_ray_limits(r, g, launches);
    if (s == BEAMS_OK) s = build_map_lazy(r, g, launches);
    if (s != BEAMS_OK) return s;
  } else if (need_map) {
    s = build_map(r, g, launches, built);
    if (s != BEAMS_OK) return s;
  }
  cudaEventRecord(r->ev[1], r->stream);
  const size_t npix = (size_t)cam->width * cam->height;
  float4* dst = (float4*)rgba_out;
  const bool direct = out_on_device == BEAMS_OUT_DEVICE && (((uintptr_t)rgba_out & 15) == 0);
  if (!direct) {
    s = ensure_buffer(r, (void**)&r->d_rgba, &r->rgba_cap, npix * sizeof(float4), "allocating image");
    if (s != BEAMS_OK) return s;
    dst = r->d_rgba;
  }
  if (!lazy) {
    s = prepare_ray_limits(r, g, launches);
    if (s != BEAMS_OK) return s;
  }
  if (use_mlp) {
    s = mlp_render_view(r, g, dst, launches);
    if (s != BEAMS_OK) return s;
    --launches;  // counted below with the other view marches
    e = cudaSuccess;
  } else {
    const unsigned char* occ = nullptr;
    if (r->view_skip && r->vol.assoc == BEAMS_ASSOC_POINTS && !g.rect) {
      s = prepare_occupancy(r, g, launches);
      if (s != BEAMS_OK) return s;
      occ = r->d_occ;
    }
    if (r->form == BEAMS_FORM_PRECISION && r->vol.assoc == BEAMS_ASSOC_POINTS)
      e = launch_view_march_prec(g, quad_dtype(r), r->d_quads, r->d_tab, r->d_tf,
                                 need_map ? (const __half*)r->d_map : nullptr, dst, r->d_cnt, r->stream, occ);
    else
      e = launch_view_march_f32(g, (const float*)r->d_field, (const float4*)r->d_quads, r->d_tab, r->d_tf,
                                need_map ? r->d_map : nullptr, dst, r->d_cnt, r->stream, occ);
  }
  if (e != cudaSuccess) return cuda_fail(r, e, "view_march launch");
  ++launches;
  cudaEventRecord(r->ev[2], r->stream);
  s = blend_background(r, dst, npix, launches);
  if (s != BEAMS_OK) return s;
  if (!direct) {
    e = cudaMemcpyAsync(rgba_out, dst, npix * sizeof(float4),
                        out_on_device == BEAMS_OUT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "copying image out");
  }
  cudaEventRecord(r->ev[3], r->stream);
  if (t) {
    std::memset(t, 0, sizeof(*t));
    e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "render");
    Counters c;
    e = cudaMemcpy(&c, r->d_cnt, sizeof(c), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(r, e, "reading counters");
    cudaEventElapsedTime(&t->map_build_ms, r->ev[0], r->ev[1]);
    cudaEventElapsedTime(&t->view_march_ms, r->ev[1], r->ev[2]);
    cudaEventElapsedTime(&t->composite_ms, r->ev[2], r->ev[3]);
    cudaEventElapsedTime(&t->total_ms, r->ev[0], r->ev[3]);
    t->light_samples = c.light_samples;
    t->lit_samples = c.lit_samples;
    t->rays_hit = c.rays_hit;
    t->mlp_samples = c.mlp_samples;
    t->mlp_rows = c.mlp_rows;
    t->fallback_tiles = (int)c.fallback_tiles;
    // the learned form's fallback and the lazy map build only the vertices their view rays read
    t->map_vertices = (use_mlp || lazy) ? (int)c.map_vertices : (built ? (int)r->map_count : 0);
    t->kernel_launches = launches;
  } else if (out_on_device == BEAMS_OUT_HOST) {
    // The caller reads rgba_out on return.
    e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "render");
  }
  return BEAMS_OK;
}

beams_status beams_synchronize(beams_renderer* r) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  cudaSetDevice(r->device);
  const cudaError_t e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "synchronize");
  return BEAMS_OK;
}

beams_status beams_set_bricks(beams_renderer* r, const beams_volume* bricks, int nbricks) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!bricks || nbricks < 1 || nbricks > kMaxBricks)
    return fail(r, BEAMS_ERR_INVALID_ARG, "bricks: need 1..32 volumes");
  for (int b = 0; b < nbricks; ++b) {
    const beams_volume& v = bricks[b];
    if (!v.data || v.dtype != BEAMS_F32 || v.assoc != BEAMS_ASSOC_POINTS)
      return fail(r, BEAMS_ERR_INVALID_ARG, "bricks: each brick must be a float32 point field");
    for (int d = 0; d < 3; ++d)
      if (v.dims[d] < 2 || v.dims[d] > 8192 || !(v.spacing[d] > 0.0) || !std::isfinite(v.spacing[d]) ||
          !std::isfinite(v.origin[d]))
        return fail(r, BEAMS_ERR_INVALID_ARG, "bricks: bad dims/origin/spacing");
    if (!std::isfinite(v.range[0]) || !std::isfinite(v.range[1]))
      return fail(r, BEAMS_ERR_INVALID_ARG, "bricks: range must be finite");
  }
  cudaSetDevice(r->device);
  cudaStreamSynchronize(r->stream);  // the previous frame's brick work (lanes join into r->stream) is done
  for (auto& b : r->bricks) b.release();
  r->bricks.assign(nbricks, Brick());
  for (int b = 0; b < nbricks; ++b) {
    Brick& B = r->bricks[b];
    const beams_volume& v = bricks[b];
    const size_t bytes = (size_t)v.dims[0] * v.dims[1] * v.dims[2] * sizeof(float);
    if (v.on_device) {
      B.d_field = v.data;
    } else {
      beams_status s = ensure_buffer(r, &B.d_field_owned, &B.field_cap, bytes, "allocating brick field");
      if (s != BEAMS_OK) return s;
      cudaError_t e = cudaMemcpyAsync(B.d_field_owned, v.data, bytes, cudaMemcpyHostToDevice, r->stream);
      if (e != cudaSuccess) return cuda_fail(r, e, "copying brick field");
      B.d_field = B.d_field_owned;
    }
    B.vol = v;
    B.vol.data = B.d_field;
    B.vol.on_device = 1;
    B.version = ++r->brick_counter;
  }
  r->brick_mode = true;
  r->map_valid = false;
  return BEAMS_OK;
}

beams_status beams_get_brick_map(beams_renderer* r, int brick, int stage, float* dst, size_t count,
                                 int dst_on_device) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!r->brick_mode || brick < 0 || brick >= (int)r->bricks.size())
    return fail(r, BEAMS_ERR_INVALID_ARG, "no such brick");
  Brick& B = r->bricks[brick];
  const float* src = stage ? B.d_map_final : B.d_map_local;
  if (!src || B.map_count == 0) return fail(r, BEAMS_ERR_STATE, "brick map not built yet");
  if (stage && B.final_partial)
    return fail(r, BEAMS_ERR_STATE, "the lazy map built only the stitched vertices the view reads");
  if (!dst || count < B.map_count) return fail(r, BEAMS_ERR_INVALID_ARG, "destination too small for the map");
  cudaSetDevice(r->device);
  cudaError_t e = cudaMemcpyAsync(dst, src, B.map_count * sizeof(float),
                                  dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "copying brick map");
  return BEAMS_OK;
}

beams_status beams_selftest_division(float origin, float spacing, int ncells, int samples,
                                     unsigned long long* checked, unsigned long long* mismatches) {
  if (ncells < 1 || samples < 4 || !checked || !mismatches || !(spacing > 0.f))
    return fail(nullptr, BEAMS_ERR_INVALID_ARG, "selftest_division: bad argument");
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc((void**)&d, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(d, 0, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = launch_selftest_division(origin, spacing, ncells, samples, d, nullptr);
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "selftest_division");
  *mismatches = h[0];
  *checked = h[1];
  return BEAMS_OK;
}

beams_status beams_generate_blobs(float* dev_out, const int n[3], const float* params, int nblobs, int normalise,
                                  void* stream) {
  if (!dev_out || !n || !params || nblobs < 1 || nblobs > 4096)
    return fail(nullptr, BEAMS_ERR_INVALID_ARG, "generate_blobs: bad argument");
  if (n[0] < 2 || n[1] < 2 || n[2] < 2) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "generate_blobs: dims < 2");
  cudaStream_t st = (cudaStream_t)stream;
  float* d_prm = nullptr;
  unsigned* d_mm = nullptr;
  cudaError_t e = cudaMalloc((void**)&d_prm, sizeof(float) * 5 * nblobs);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_mm, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_prm, params, sizeof(float) * 5 * nblobs, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_generate_blobs(dev_out, n, d_prm, nblobs, st);
  if (e == cudaSuccess && normalise)
    e = launch_normalise01(dev_out, (int64_t)n[0] * n[1] * n[2], d_mm, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_prm);
  cudaFree(d_mm);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "generate_blobs");
  return BEAMS_OK;
}

beams_status beams_generate_noise(float* dev_out, const int n[3], const unsigned char* perm, int octaves,
                                  float base_freq, float lacunarity, float gain, void* stream) {
  if (!dev_out || !n || !perm || octaves < 1 || octaves > 16)
    return fail(nullptr, BEAMS_ERR_INVALID_ARG, "generate_noise: bad argument");
  if (n[0] < 2 || n[1] < 2 || n[2] < 2) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "generate_noise: dims < 2");
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* d_perm = nullptr;
  unsigned* d_mm = nullptr;
  cudaError_t e = cudaMalloc((void**)&d_perm, 256);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_mm, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_perm, perm, 256, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_generate_noise(dev_out, n, d_perm, octaves, base_freq, lacunarity, gain, st);
  if (e == cudaSuccess) e = launch_normalise01(dev_out, (int64_t)n[0] * n[1] * n[2], d_mm, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_perm);
  cudaFree(d_mm);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "generate_noise");
  return BEAMS_OK;
}

}  // extern "C"
