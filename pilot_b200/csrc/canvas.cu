// canvas.cu — the canvas side of the mapper: depth clipping of the camera rays
// and the background blend.
//
// The reference mapper (beams/rendering/MapperLightedVolume.cxx:147-153) builds
// the camera rays, then RayOperations::MapCanvasToRays turns the canvas depth
// buffer into each ray's MaxDistance, which the slab test (CalcRayStart,
// LightedVolumeRenderer.cxx:644-718) narrows to the volume's exit; after the
// sort-last composite it blends the background when SetCompositeBackground is
// on (:185-188). Both routines are VTK-m's (not vendored), so this file states
// them in its own terms:
//   * the depth buffer holds, per pixel of the output image (row y at y * W,
//     row 0 at the bottom like the image), either the ray distance itself
//     (BEAMS_DEPTH_RAY_DISTANCE) or an OpenGL window depth d in [0, 1] under
//     the camera's perspective projection with the given near and far planes
//     (BEAMS_DEPTH_WINDOW). A window depth is unprojected at the pixel centre:
//     z_ndc = 2d - 1, view depth t = 2fn / ((f + n) - z_ndc (f - n)), and the
//     distance along the normalised ray through that pixel is t * |v|, v the
//     un-normalised camera ray (forward + sx right + sy up) of camera_ray —
//     the inverse of the standard perspective and look-at matrices applied to
//     (x_ndc, y_ndc, z_ndc, 1). d = 1 is the far plane, so a cleared buffer
//     clips at the far plane as a cleared canvas does;
//   * the background blend is Porter and Duff's "over" of the premultiplied
//     image over the background colour: a = bg.a (1 - C.a), C.rgb += bg.rgb a,
//     C.a += a (pixels with C.a >= 1 unchanged).
// Compiled with -fmad=false like every kernel file.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/beams_b200.h"
#include "exact_device.cuh"
#include "renderer.h"

namespace beams {

beams_status make_geo_vol(beams_renderer* r, const beams_volume& v, const beams_camera* cam, ExactGeo& g);
beams_status validate_camera(beams_renderer* r, const beams_camera* cam);

namespace {

struct DepthXform {
  int kind;
  float A, B, C;  // window depth: t = A / (B - z_ndc * C), A = 2fn, B = f + n, C = f - n
};

__global__ void k_ray_limits(const ExactGeo g, const float* __restrict__ depth, DepthXform X,
                             float* __restrict__ out) {
  const size_t n = (size_t)g.width * g.height;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = depth[i];
    float lim;
    if (X.kind == BEAMS_DEPTH_RAY_DISTANCE) {
      lim = (v == v) ? v : __int_as_float(0x7f800000);  // NaN: no limit
    } else {
      const int x = (int)(i % (size_t)g.width), y = (int)(i / (size_t)g.width);
      const float d = (v == v) ? fminf(fmaxf(v, 0.f), 1.f) : 1.f;
      const float z = 2.f * d - 1.f;
      const float t = X.A / (X.B - z * X.C);
      const float sx = ((float)x + 0.5f) * g.kx - g.cx;
      const float sy = ((float)y + 0.5f) * g.ky - g.cy;
      float w[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) w[k] = (g.cf[k] + sx * g.cr[k]) + sy * g.cu[k];
      lim = t * sqrtf(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    }
    out[i] = lim;
  }
}

__global__ void k_blend_background(float4* __restrict__ img, size_t n, float4 bg) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float4 c = img[i];
    if (c.w >= 1.f) continue;
    const float a = bg.w * (1.f - c.w);
    c.x = c.x + bg.x * a;
    c.y = c.y + bg.y * a;
    c.z = c.z + bg.z * a;
    c.w = a + c.w;
    img[i] = c;
  }
}

int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

}  // namespace

// Fills r->d_raymax for the camera in g and points g.ray_max at it (nothing
// when no depth buffer is set).
beams_status prepare_ray_limits(beams_renderer* r, ExactGeo& g, int& launches) {
  g.ray_max = nullptr;
  if (!r->depth_set) return BEAMS_OK;
  if (g.width != r->depth_w || g.height != r->depth_h)
    return fail(r, BEAMS_ERR_INVALID_ARG, "depth buffer size differs from the camera's image size");
  const size_t n = (size_t)g.width * g.height;
  beams_status s = ensure_buffer(r, (void**)&r->d_raymax, &r->raymax_cap, n * sizeof(float),
                                 "allocating ray limits");
  if (s != BEAMS_OK) return s;
  DepthXform X{r->depth_kind, 0.f, 0.f, 0.f};
  const double f = r->depth_far, nn = r->depth_near;
  X.A = (float)(2.0 * f * nn);
  X.B = (float)(f + nn);
  X.C = (float)(f - nn);
  k_ray_limits<<<grid_for(n), 256, 0, r->stream>>>(g, r->d_depth, X, r->d_raymax);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(r, e, "ray limits launch");
  ++launches;
  g.ray_max = r->d_raymax;
  return BEAMS_OK;
}

// The background blend of the finished image, when enabled.
beams_status blend_background(beams_renderer* r, float4* img, size_t npix, int& launches) {
  if (!r->bg) return BEAMS_OK;
  const float4 bg = make_float4(r->bg_rgba[0], r->bg_rgba[1], r->bg_rgba[2], r->bg_rgba[3]);
  k_blend_background<<<grid_for(npix), 256, 0, r->stream>>>(img, npix, bg);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(r, e, "background blend launch");
  ++launches;
  return BEAMS_OK;
}

}  // namespace beams

using namespace beams;

extern "C" beams_status beams_set_depth_buffer(beams_renderer* r, const float* depth, int width, int height,
                                               int kind, double near_plane, double far_plane, int on_device) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  ++r->depth_version;  // every call may change the ray limits
  if (!depth) {
    r->depth_set = false;
    return BEAMS_OK;
  }
  if (width < 1 || height < 1 || width > 16384 || height > 16384)
    return fail(r, BEAMS_ERR_INVALID_ARG, "depth buffer: width and height must be in [1, 16384]");
  if (kind != BEAMS_DEPTH_RAY_DISTANCE && kind != BEAMS_DEPTH_WINDOW)
    return fail(r, BEAMS_ERR_INVALID_ARG, "depth buffer: kind must be BEAMS_DEPTH_RAY_DISTANCE or BEAMS_DEPTH_WINDOW");
  if (kind == BEAMS_DEPTH_WINDOW &&
      !(near_plane > 0.0 && far_plane > near_plane && std::isfinite(far_plane)))
    return fail(r, BEAMS_ERR_INVALID_ARG, "depth buffer: window depth needs 0 < near < far < inf");
  cudaSetDevice(r->device);
  const size_t n = (size_t)width * height;
  beams_status s = ensure_buffer(r, (void**)&r->d_depth, &r->depth_cap, n * sizeof(float), "allocating depth buffer");
  if (s != BEAMS_OK) return s;
  cudaError_t e = cudaMemcpyAsync(r->d_depth, depth, n * sizeof(float),
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(r->stream);  // the caller may reuse its buffer
  if (e != cudaSuccess) return cuda_fail(r, e, "copying depth buffer");
  r->depth_set = true;
  r->depth_w = width;
  r->depth_h = height;
  r->depth_kind = kind;
  r->depth_near = near_plane;
  r->depth_far = far_plane;
  return BEAMS_OK;
}

extern "C" beams_status beams_get_ray_limits(beams_renderer* r, const beams_camera* cam, float* dst,
                                             int dst_on_device) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!cam || !dst) return fail(r, BEAMS_ERR_INVALID_ARG, "ray limits: NULL camera or destination");
  if (!r->depth_set) return fail(r, BEAMS_ERR_STATE, "ray limits: no depth buffer set");
  if (!r->has_volume && r->bricks.empty()) return fail(r, BEAMS_ERR_STATE, "ray limits: no volume set");
  beams_status s = validate_camera(r, cam);
  if (s != BEAMS_OK) return s;
  cudaSetDevice(r->device);
  ExactGeo g;
  s = make_geo_vol(r, r->brick_mode ? r->bricks[0].vol : r->vol, cam, g);
  if (s != BEAMS_OK) return s;
  int launches = 0;
  s = prepare_ray_limits(r, g, launches);
  if (s != BEAMS_OK) return s;
  const size_t n = (size_t)cam->width * cam->height;
  cudaError_t e = cudaMemcpyAsync(dst, r->d_raymax, n * sizeof(float),
                                  dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "copying ray limits");
  return BEAMS_OK;
}
