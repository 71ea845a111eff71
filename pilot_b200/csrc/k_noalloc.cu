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
// The kernels run the same march code as beams_render's K1 and K2
// (march_vertex, view_march_pixel) on the plain float32 field with the cell
// tables computed into shared memory, so the image equals beams_render's bit
// for bit.
// Compiled with -fmad=false like every kernel file.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/beams_b200.h"
#include "exact_device.cuh"
#include "light_march.cuh"
#include "renderer.h"
#include "view_march.cuh"

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

// The cell tables {lo, hi, hi - lo, RN(1/(hi - lo))} computed into shared
// memory from the generated coordinates (the entries beams_render builds once
// per volume into device memory), n entries from the start.
__device__ void stage_tables(const ExactGeo& g, int n, float4* s_tab) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_tab[i] = table_entry(g, i);
}

// K1: one thread per map vertex, the light march of k_light_march
// (march_vertex, TransmittanceMap.h:279-332) on the plain field, into the
// scratch map. Alpha / max alpha as GetMaxAlpha (TransmittanceMap.h:515-525).
__global__ void __launch_bounds__(256) k_noalloc_light_march(const ExactGeo g, const FieldF32* __restrict__ field,
                                                             const float4* __restrict__ tf,
                                                             float* __restrict__ map, int nvert) {
  extern __shared__ float4 s_dyn[];
  float4* s_tab = s_dyn;                              // field axes' entries
  float* s_a = reinterpret_cast<float*>(s_dyn + g.max_off[0]);
  __shared__ float s_max;
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int i = 0; i < g.tf_n; ++i) m = mx(m, tf[i].w);
    s_max = m;
  }
  stage_tables(g, g.max_off[0], s_tab);
  __syncthreads();
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_a[i] = (s_max > 0.f) ? tf[i].w / s_max : 0.f;
  __syncthreads();
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nvert) return;
  float V[3], L[3];
  map_vertex(g, id, V);
  light_origin(g, V, L);
  Accum<false> acc;
  unsigned ns = 0;
  march_vertex<FieldF32, false, false>(g, field, s_tab + g.ax_off[0], s_tab + g.ax_off[1], s_tab + g.ax_off[2], s_a,
                                       nullptr, nullptr, V, L, [](const float*) { return 0.f; }, acc, ns);
  map[id] = acc.o;
}

// K2: one thread per pixel in 16 x 16 blocks, the view march of k_view_march
// (view_march_pixel, LightedVolumeRenderer.cxx:346-498) shading by the scratch map.
__global__ void __launch_bounds__(256) k_noalloc_view_march(const ExactGeo g, const FieldF32* __restrict__ field,
                                                            const float4* __restrict__ tf,
                                                            const float* __restrict__ map,
                                                            float4* __restrict__ out) {
  extern __shared__ float4 s_dyn[];
  float4* s_tab = s_dyn;            // field and map axes' entries
  float4* s_tf = s_dyn + g.ntab;
  stage_tables(g, g.ntab, s_tab);
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  const int tiles_x = (g.width + 15) >> 4;
  const int x = (blockIdx.x % tiles_x) * 16 + (threadIdx.x & 15);
  const int y = (blockIdx.x / tiles_x) * 16 + (threadIdx.x >> 4);
  if (x >= g.width || y >= g.height) return;
  float4 color;
  unsigned lit = 0, hit = 0;
  view_march_pixel<FieldF32, true, float>(g, field, s_tab, s_tf, map, x, y, color, lit, hit);
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
  if ((size_t)(vol->dims[0] + vol->dims[1] + vol->dims[2] - 3 + 3 * (size_t)map_cells + kMaxTFn) * 16 > 200 * 1024)
    return nf(BEAMS_ERR_UNSUPPORTED, "render_noalloc: volume/map axes too long for the shared-memory cell tables");
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
  {
    int off = 0;
    for (int d = 0; d < 3; ++d) {
      g.ax_off[d] = off;
      off += g.n[d] - 1;
    }
    for (int d = 0; d < 3; ++d) {
      g.max_off[d] = off;
      off += map_cells;
    }
    g.ntab = off;
  }
  geo_loop_constants(g);
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
  const size_t smem1 = (size_t)g.max_off[0] * sizeof(float4) + (size_t)tf_n * sizeof(float);
  const size_t smem2 = ((size_t)g.ntab + (size_t)tf_n) * sizeof(float4);
  e = cudaFuncSetAttribute(k_noalloc_light_march, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_noalloc_view_march, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
  if (e != cudaSuccess) return nf(BEAMS_ERR_CUDA, cudaGetErrorString(e));
  // The light march writes every one of the nvert map entries before the view
  // march reads any, so the scratch needs no clearing between calls.
  const FieldF32* field = (const FieldF32*)vol->data;
  k_noalloc_light_march<<<(nvert + 255) / 256, 256, smem1, st>>>(g, field, (const float4*)tf_rgba_device, map, nvert);
  const int tiles = ((g.width + 15) >> 4) * ((g.height + 15) >> 4);
  k_noalloc_view_march<<<tiles, 256, smem2, st>>>(g, field, (const float4*)tf_rgba_device, map,
                                                  (float4*)rgba_out_device);
  e = cudaGetLastError();
  if (e != cudaSuccess) return nf(BEAMS_ERR_CUDA, cudaGetErrorString(e));
  return BEAMS_OK;
}
