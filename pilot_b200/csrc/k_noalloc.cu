// k_noalloc.cu — a render entry point that allocates no device memory.
//
// Who needs it: code that may not call cudaMalloc/cudaFree itself — a custom
// call or plugin running inside another framework that owns all device memory
// through its own allocator (an ML runtime, a visualization host application),
// or a real-time frame loop that must not stall, since cudaMalloc and cudaFree
// can synchronise the whole device. beams_render keeps per-renderer buffers
// (the map, a quad copy of the field, cell tables) that it allocates on first
// use; this entry point instead keeps its only scratch, the frame's
// transmittance map, in a fixed static device array below, and otherwise uses
// the caller's input and output buffers.
//
// The kernels here restate the same reference arithmetic as k_exact.cu on the
// plain field layout (eight scalar loads per cell, coordinates generated as
// origin + spacing*i, IEEE division), so the image equals beams_render's.
// Compiled with -fmad=false like every kernel file.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/beams_b200.h"
#include "exact_device.cuh"
#include "renderer.h"

namespace beams {
namespace {

constexpr int kMaxMapCells = BEAMS_NOALLOC_MAX_MAP_CELLS;
constexpr size_t kMaxMapVertices = (size_t)(kMaxMapCells + 1) * (kMaxMapCells + 1) * (kMaxMapCells + 1);
constexpr size_t kScratchFloats = (kMaxMapVertices + 63) / 64 * 64;
constexpr int kMaxTFn = 1024;

// The scratch: one frame's (M+1)^3 map, M <= BEAMS_NOALLOC_MAX_MAP_CELLS
// (129^3 floats, 8.6 MB). Every device that loads this library holds it until
// the process exits. In host code its name is only a host-side handle: the
// kernels get the device address from cudaGetSymbolAddress.
static __device__ __align__(256) float g_noalloc_map[kScratchFloats];

// Device address of the scratch in the current context, looked up on every
// call: it is cheap once the module is loaded, and it stays right when the
// context changes under this library (a cudaDeviceReset, or a host that runs
// the call under its own driver-API context on the device). With lazy module
// loading (CUDA_MODULE_LOADING=LAZY, the default) the first lookup on a device
// loads this file's module and so reserves the array; that first call must not
// run inside a stream capture.
cudaError_t scratch_address(float** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_map);
  if (e != cudaSuccess) return e;
  *out = (float*)p;
  return cudaSuccess;
}

// Errors go to the thread-local text that beams_last_error(NULL) returns.
beams_status nf(beams_status s, const char* msg) { return fail(nullptr, s, msg); }

// Reference-order TF staging: RGBA in shared memory plus alpha / max alpha
// (TransmittanceMap.h:329, GetMaxAlpha :515-525).
__device__ void stage_tf(const float4* __restrict__ tf, int n, float4* s_tf, float* s_a, float* s_max) {
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int i = 0; i < n; ++i) m = mx(m, tf[i].w);
    *s_max = m;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  const float m = *s_max;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_a[i] = (m > 0.f) ? s_tf[i].w / m : 0.f;
  __syncthreads();
}

// The view march reads the TF colours only (no alpha / max alpha pass).
__device__ void stage_tf_colors(const float4* __restrict__ tf, int n, float4* s_tf) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
}

// Smallest cell c with val <= coord(c+1) (RectilinearMeshOracle.h:154-176).
__device__ __forceinline__ int cell_bsearch_gen(const ExactGeo& g, int d, float val) {
  const int cmax = g.n[d] - 2;
  int c = (int)fminf(fmaxf((val - g.org[d]) * g.invh[d], 0.f), (float)cmax);
  while (c > 0 && val <= coord(g, d, c)) --c;
  while (c < cmax && val > coord(g, d, c + 1)) ++c;
  return c;
}

// Unique cell with coord(c) <= p < coord(c+1) (LightedVolumeRenderer.cxx:119-165).
__device__ __forceinline__ int cell_walk_gen(const ExactGeo& g, int d, float p) {
  const int cmax = g.n[d] - 2;
  int c = (int)fminf(fmaxf((p - g.org[d]) * g.invh[d], 0.f), (float)cmax);
  while (c > 0 && p < coord(g, d, c)) --c;
  while (c < cmax && p >= coord(g, d, c + 1)) ++c;
  return c;
}

__device__ __forceinline__ void cell_values(const float* __restrict__ f, const ExactGeo& g, int c0, int c1, int c2,
                                            float v[8]) {
  const unsigned nx = (unsigned)g.n[0], nxy = (unsigned)g.n[0] * (unsigned)g.n[1];
  const float* b = f + ((unsigned)c2 * nxy + (unsigned)c1 * nx + (unsigned)c0);
  v[0] = __ldg(b);
  v[1] = __ldg(b + 1);
  v[2] = __ldg(b + 1 + nx);
  v[3] = __ldg(b + nx);
  v[4] = __ldg(b + nxy);
  v[5] = __ldg(b + nxy + 1);
  v[6] = __ldg(b + nxy + 1 + nx);
  v[7] = __ldg(b + nxy + nx);
}

// Light march (TransmittanceMap.h:279-332) writing the scratch map.
__global__ void __launch_bounds__(256) k_noalloc_light_march(const ExactGeo g, const float* __restrict__ field,
                                                             const float4* __restrict__ tf,
                                                             float* __restrict__ map, int nvert) {
  __shared__ float4 s_tf[kMaxTFn];
  __shared__ float s_a[kMaxTFn];
  __shared__ float s_max;
  stage_tf(tf, g.tf_n, s_tf, s_a, &s_max);
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nvert) return;
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
  const int n1 = g.tf_n - 1;
  float o = 0.f;
  for (int b = g.light_budget; b > 0; --b) {
    const float q0 = s[0] - st[0], q1 = s[1] - st[1], q2 = s[2] - st[2];
    if (!(q0 * q0 + q1 * q1 + q2 * q2 <= len2)) break;
    s[0] = s[0] + g.step * dir[0];
    s[1] = s[1] + g.step * dir[1];
    s[2] = s[2] + g.step * dir[2];
    if (!inside_vol(g, s)) break;
    int c[3];
    float pc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      c[d] = cell_bsearch_gen(g, d, s[d]);
      const float lo = coord(g, d, c[d]), hi = coord(g, d, c[d] + 1);
      pc[d] = (s[d] - lo) / (hi - lo);
    }
    float vals[8];
    cell_values(field, g, c[0], c[1], c[2], vals);
    float scalar = hex_interp(vals, pc[0], pc[1], pc[2]);
    scalar = (scalar - g.min_scalar) * g.inv_delta;
    o = o + (1.f - o) * s_a[tf_index_clamped(scalar * (float)n1, n1)];
    if (o == 1.f) break;
  }
  map[id] = o;
}

__device__ __forceinline__ float map_opacity_gen(const ExactGeo& g, const float* __restrict__ map, const float p[3]) {
  int c[3];
  float pc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float t = (p[d] - g.morig[d]) * g.minv[d];
    if (t < 0.f) t = 0.f;
    if (t >= (float)(g.pd[d] - 1)) t = (float)(g.pd[d] - 2);
    c[d] = (int)t;
    const float lo = vtx_coord(g, d, c[d]), hi = vtx_coord(g, d, c[d] + 1);
    pc[d] = (p[d] - lo) / (hi - lo);
  }
  const unsigned px = (unsigned)g.pd[0], pxy = (unsigned)g.pd[0] * (unsigned)g.pd[1];
  const float* m = map + ((unsigned)c[2] * pxy + (unsigned)c[1] * px + (unsigned)c[0]);
  float v[8] = {m[0], m[1], m[1 + px], m[px], m[pxy], m[pxy + 1], m[pxy + 1 + px], m[pxy + px]};
  return hex_interp(v, pc[0], pc[1], pc[2]);
}

// View march (LightedVolumeRenderer.cxx:346-498) shading by the scratch map.
__global__ void __launch_bounds__(256) k_noalloc_view_march(const ExactGeo g, const float* __restrict__ field,
                                                            const float4* __restrict__ tf,
                                                            const float* __restrict__ map,
                                                            float4* __restrict__ out) {
  __shared__ float4 s_tf[kMaxTFn];
  stage_tf_colors(tf, g.tf_n, s_tf);
  const int tiles_x = (g.width + 15) >> 4;
  const int x = (blockIdx.x % tiles_x) * 16 + (threadIdx.x & 15);
  const int y = (blockIdx.x / tiles_x) * 16 + (threadIdx.x >> 4);
  if (x >= g.width || y >= g.height) return;
  float4 color = make_float4(0.f, 0.f, 0.f, 0.f);
  float o[3], d[3], minD, maxD;
  if (ray_setup(g, x, y, o, d, minD, maxD)) {
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
    float bl[3] = {0.f, 0.f, 0.f}, inv[3] = {0.f, 0.f, 0.f};
    bool newCell = true;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    float s0 = 0.f, s1m0 = 0.f, s2m3 = 0.f, s3 = 0.f, s4 = 0.f, s5m4 = 0.f, s6m7 = 0.f, s7 = 0.f;
    int c[3] = {0, 0, 0};
    const int n1 = g.tf_n - 1;
    while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
      const float mint = mn(tx, mn(ty, tz));
      const float maxt = mx(tx, mx(ty, tz));
      if (maxt > 1.f || mint < 0.f) newCell = true;
      if (newCell) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (p[k] == g.maxp[k]) {
            c[k] = g.n[k] - 2;  // the reference keeps invSpacing[k] here
          } else {
            c[k] = cell_walk_gen(g, k, p[k]);
            inv[k] = 1.f / (coord(g, k, c[k] + 1) - coord(g, k, c[k]));
          }
          bl[k] = coord(g, k, c[k]);
        }
        float v[8];
        cell_values(field, g, c[0], c[1], c[2], v);
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
        const float4 tfc = s_tf[(int)fi];
        const float sa = tfc.w * (1.f - color.w);
        const float tr = 1.f - map_opacity_gen(g, map, p);
        const float sc0 = clamp01(tfc.x * (tr * g.light_color[0]));
        const float sc1 = clamp01(tfc.y * (tr * g.light_color[1]));
        const float sc2 = clamp01(tfc.z * (tr * g.light_color[2]));
        color.x = color.x + sc0 * sa;
        color.y = color.y + sc1 * sa;
        color.z = color.z + sc2 * sa;
        color.w = sa + color.w;
      }
      dist += g.sd;
      p[0] = p[0] + g.sd * d[0];
      p[1] = p[1] + g.sd * d[1];
      p[2] = p[2] + g.sd * d[2];
      tx = (p[0] - bl[0]) * inv[0];
      ty = (p[1] - bl[1]) * inv[1];
      tz = (p[2] - bl[2]) * inv[2];
      if (color.w >= g.cutoff) break;
    }
  }
  out[(size_t)y * g.width + x] = color;
}

bool finite3(const double* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

}  // namespace
}  // namespace beams

using namespace beams;

extern "C" beams_status beams_render_noalloc(const beams_volume* vol, const float* tf_rgba_device, int tf_n,
                                             const double light_pos[3], const float light_color[3],
                                             float light_intensity, int map_cells, float sample_distance,
                                             float termination_alpha, const beams_camera* cam,
                                             float* rgba_out_device, void* cuda_stream) {
  if (!vol || !vol->data || !tf_rgba_device || !light_pos || !light_color || !cam || !rgba_out_device)
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: NULL argument");
  if (!vol->on_device || vol->dtype != BEAMS_F32 || vol->assoc != BEAMS_ASSOC_POINTS)
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: the volume must be a float32 point field in device memory");
  for (int d = 0; d < 3; ++d)
    if (vol->dims[d] < 2 || vol->dims[d] > 8192 || !(vol->spacing[d] > 0.0) || !std::isfinite(vol->spacing[d]) ||
        !std::isfinite(vol->origin[d]))
      return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: bad volume dims/origin/spacing");
  if ((double)vol->dims[0] * vol->dims[1] * vol->dims[2] >= 4294967296.0)
    return nf(BEAMS_ERR_UNSUPPORTED, "render_noalloc: volume too large for 32-bit indexing");
  if (tf_n < 1 || tf_n > kMaxTFn) return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: tf_n must be in [1, 1024]");
  if (map_cells < 1 || map_cells > kMaxMapCells)
    return nf(BEAMS_ERR_INVALID_ARG,
              "render_noalloc: map_cells must be in [1, BEAMS_NOALLOC_MAX_MAP_CELLS = 128]; the map lives in a "
              "fixed 129^3-float static scratch array");
  if (!finite3(light_pos) || !std::isfinite(light_intensity) || !(termination_alpha > 0.f) ||
      !std::isfinite(vol->range[0]) || !std::isfinite(vol->range[1]))
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: non-finite light, range or termination alpha");
  if (cam->width < 1 || cam->height < 1 || cam->width > 16384 || cam->height > 16384 ||
      !(cam->fov_y_deg > 0.0 && cam->fov_y_deg < 180.0) || !finite3(cam->position) || !finite3(cam->look_at) ||
      !finite3(cam->up))
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: bad camera");
  if (((uintptr_t)rgba_out_device & 15) != 0 || ((uintptr_t)tf_rgba_device & 15) != 0)
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: output and colour map must be 16-byte aligned");
  if (((uintptr_t)vol->data & 3) != 0)
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: the volume data must be 4-byte aligned");
  if (!std::isfinite(light_color[0]) || !std::isfinite(light_color[1]) || !std::isfinite(light_color[2]))
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: non-finite light colour");

  // Parameters, derived in the reference's float32 order (as beams_render does).
  ExactGeo g;
  std::memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) {
    g.n[d] = vol->dims[d];
    g.org[d] = (float)vol->origin[d];
    g.h[d] = (float)vol->spacing[d];
    g.invh[d] = 1.f / g.h[d];
    g.minp[d] = g.org[d] + g.h[d] * 0.f;
    g.maxp[d] = g.org[d] + g.h[d] * (float)(vol->dims[d] - 1);
    g.bmin[d] = (double)g.minp[d];
    g.bmax[d] = (double)g.maxp[d];
  }
  const float fmin = (float)vol->range[0], fmax = (float)vol->range[1];
  g.min_scalar = fmin;
  g.inv_delta = ((fmax - fmin) != 0.f) ? 1.f / (fmax - fmin) : fmin;
  g.tf_n = tf_n;
  float ext[3];
  for (int d = 0; d < 3; ++d) ext[d] = (float)(g.bmax[d] - g.bmin[d]);
  g.extent_mag = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]);
  for (int d = 0; d < 3; ++d) {
    g.pd[d] = map_cells + 1;
    g.morig[d] = (float)g.bmin[d];
    g.msp[d] = ext[d] / (float)map_cells;
    g.minv[d] = 1.f / g.msp[d];
    g.light_color[d] = light_color[d] * light_intensity;
    g.light[d] = (float)light_pos[d];
  }
  g.sd = (sample_distance > 0.f) ? sample_distance : g.extent_mag / 200.f;
  if (!(g.extent_mag / g.sd <= 1.0e6f))
    return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: sample distance below 1e-6 of the volume diagonal");
  g.mesh_eps = g.extent_mag * 0.0001f;
  g.step = g.extent_mag / 128.f;
  g.cutoff = termination_alpha;
  g.light_budget = (int)(g.extent_mag / g.step) + 8;
  g.dir_dist = 2.f * g.extent_mag;
  g.light_kind = 0;
  g.slab_fp64 = 1;
  g.use_map = 1;
  {
    double f[3], rr[3], u[3];
    for (int d = 0; d < 3; ++d) f[d] = cam->look_at[d] - cam->position[d];
    const double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (int d = 0; d < 3; ++d) f[d] /= fl;
    const double* up = cam->up;
    rr[0] = f[1] * up[2] - f[2] * up[1];
    rr[1] = f[2] * up[0] - f[0] * up[2];
    rr[2] = f[0] * up[1] - f[1] * up[0];
    const double rl = std::sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
    if (!(fl > 0) || !(rl > 0)) return nf(BEAMS_ERR_INVALID_ARG, "render_noalloc: degenerate camera");
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
  }

  float* map = nullptr;
  cudaError_t e = scratch_address(&map);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return nf(BEAMS_ERR_CUDA, "render_noalloc: cudaGetSymbolAddress of the scratch map failed");
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const int nvert = g.pd[0] * g.pd[1] * g.pd[2];
  // The light march writes every one of the nvert map entries before the view
  // march reads any, so the scratch needs no clearing between calls.
  k_noalloc_light_march<<<(nvert + 255) / 256, 256, 0, st>>>(g, (const float*)vol->data,
                                                            (const float4*)tf_rgba_device, map, nvert);
  const int tiles = ((g.width + 15) >> 4) * ((g.height + 15) >> 4);
  k_noalloc_view_march<<<tiles, 256, 0, st>>>(g, (const float*)vol->data, (const float4*)tf_rgba_device, map,
                                              (float4*)rgba_out_device);
  e = cudaGetLastError();
  if (e != cudaSuccess) return nf(BEAMS_ERR_CUDA, cudaGetErrorString(e));
  return BEAMS_OK;
}
