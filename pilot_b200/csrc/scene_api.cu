// scene_api.cu — scenes from a parsed stage description: the reference's sphere
// dataset on the device, its colour table, camera and light, and the light orbit
// of its driver loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/beams_b200.h"
#include "kernels.h"
#include "renderer.h"

namespace beams {

beams_status ensure_buffer(beams_renderer* r, void** buf, size_t* cap, size_t bytes, const char* what);

namespace {

// SphereFieldGenerator::operator() (beams/sources/Spheres.cxx:36-91): e = {cx, cy,
// cz, rx, ry, rz, min, max} per ellipsoid. vtkm::Lerp(a, b, t) is taken as
// a + t * (b - a) (VTK-m is not vendored here; with min == max, as in the
// reference's scenes, every form of the lerp gives the value itself).
__global__ void k_spheres(float* __restrict__ out, int nx, int ny, int nz, float ox, float oy, float oz, float hx,
                          float hy, float hz, const float* __restrict__ e, int ne, float def, int has_floor,
                          float floor_y, float floor_v) {
  const long long total = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    const float p[3] = {ox + hx * (float)x, oy + hy * (float)y, oz + hz * (float)z};
    float sum = 0.f, cnt = 0.f;
    for (int k = 0; k < ne; ++k) {
      const float* s = e + 8 * k;
      const float d0 = s[0] - p[0], d1 = s[1] - p[1], d2 = s[2] - p[2];
      float a = ((d0 * d0) / (s[3] * s[3])) + ((d1 * d1) / (s[4] * s[4]));
      a = a + ((d2 * d2) / (s[5] * s[5]));
      a = sqrtf(a);
      if (a <= 1.f) {
        sum = sum + (s[6] + a * (s[7] - s[6]));
        cnt = cnt + 1.f;
      }
    }
    float v = cnt > 0.f ? sum / cnt : def;
    if (has_floor && p[1] < floor_y) v = floor_v;
    out[i] = v;
  }
}

// ---- colour tables --------------------------------------------------------------
// "cool to warm": K. Moreland, "Diverging Color Maps for Scientific Visualization"
// (ISVC 2009): interpolation in Msh space (polar CIELAB) between the endpoints
// (0.230, 0.299, 0.754) and (0.706, 0.016, 0.150), through an unsaturated white
// midpoint when the endpoints' hues differ by more than pi/3.
struct Msh {
  double M, s, h;
};
double srgb_to_lin(double c) { return c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4); }
double lin_to_srgb(double c) { return c <= 0.0031308 ? 12.92 * c : 1.055 * std::pow(c, 1.0 / 2.4) - 0.055; }
const double kWhite[3] = {0.95047, 1.0, 1.08883};  // D65
double lab_f(double t) { return t > 0.008856 ? std::cbrt(t) : 7.787 * t + 16.0 / 116.0; }
double lab_finv(double t) { return t > 0.206893 ? t * t * t : (t - 16.0 / 116.0) / 7.787; }

Msh rgb_to_msh(const double rgb[3]) {
  double l[3];
  for (int i = 0; i < 3; ++i) l[i] = srgb_to_lin(rgb[i]);
  const double X = 0.4124564 * l[0] + 0.3575761 * l[1] + 0.1804375 * l[2];
  const double Y = 0.2126729 * l[0] + 0.7151522 * l[1] + 0.0721750 * l[2];
  const double Z = 0.0193339 * l[0] + 0.1191920 * l[1] + 0.9503041 * l[2];
  const double fx = lab_f(X / kWhite[0]), fy = lab_f(Y / kWhite[1]), fz = lab_f(Z / kWhite[2]);
  const double L = 116.0 * fy - 16.0, a = 500.0 * (fx - fy), b = 200.0 * (fy - fz);
  const double M = std::sqrt(L * L + a * a + b * b);
  return {M, M > 0 ? std::acos(L / M) : 0.0, std::atan2(b, a)};
}

void msh_to_rgb(const Msh& m, double rgb[3]) {
  const double L = m.M * std::cos(m.s), a = m.M * std::sin(m.s) * std::cos(m.h), b = m.M * std::sin(m.s) * std::sin(m.h);
  const double fy = (L + 16.0) / 116.0, fx = fy + a / 500.0, fz = fy - b / 200.0;
  const double X = kWhite[0] * lab_finv(fx), Y = kWhite[1] * lab_finv(fy), Z = kWhite[2] * lab_finv(fz);
  const double l[3] = {3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z, -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z,
                       0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z};
  for (int i = 0; i < 3; ++i) rgb[i] = std::min(1.0, std::max(0.0, lin_to_srgb(std::min(1.0, std::max(0.0, l[i])))));
}

double adjust_hue(const Msh& sat, double m_unsat) {
  if (sat.M >= m_unsat) return sat.h;
  const double spin = sat.s * std::sqrt(m_unsat * m_unsat - sat.M * sat.M) / (sat.M * std::sin(sat.s));
  return sat.h > -M_PI / 3.0 ? sat.h + spin : sat.h - spin;
}

void diverging(double t, double rgb[3]) {
  const double c1[3] = {0.230, 0.299, 0.754}, c2[3] = {0.706, 0.016, 0.150};
  Msh a = rgb_to_msh(c1), b = rgb_to_msh(c2);
  if (a.s > 0.05 && b.s > 0.05 && std::fabs(a.h - b.h) > M_PI / 3.0) {
    const double mid = std::max(std::max(a.M, b.M), 88.0);
    if (t < 0.5) {
      b = {mid, 0.0, 0.0};
      t = 2.0 * t;
    } else {
      a = {mid, 0.0, 0.0};
      t = 2.0 * t - 1.0;
    }
  }
  if (a.s < 0.05 && b.s > 0.05) a.h = adjust_hue(b, a.M);
  else if (b.s < 0.05 && a.s > 0.05) b.h = adjust_hue(a, b.M);
  const Msh m = {(1 - t) * a.M + t * b.M, (1 - t) * a.s + t * b.s, (1 - t) * a.h + t * b.h};
  msh_to_rgb(m, rgb);
}

// Alpha through the points, linear in between and clamped at the ends; the
// points are in data units and map to the table over [range.min, range.max].
void build_table(const beams_scene_desc& d, std::vector<float>& rgba) {
  const int n = d.tf_size;
  rgba.assign((size_t)4 * n, 0.f);
  const double lo = d.tf_range[0], hi = d.tf_range[1], span = (hi != lo) ? hi - lo : 1.0;
  for (int i = 0; i < n; ++i) {
    const double v = (double)i / (n - 1);
    double c[3];
    if (std::strcmp(d.tf_preset, "ramp") == 0) {
      const double a0[3] = {0.23, 0.30, 0.75}, a1[3] = {0.95, 0.55, 0.10};
      for (int k = 0; k < 3; ++k) c[k] = a0[k] * (1 - v) + a1[k] * v;
    } else {
      diverging(v, c);
    }
    double a;
    const int np = d.tf_points;
    const double x0 = (d.tf_x[0] - lo) / span, xn = (d.tf_x[np - 1] - lo) / span;
    if (v <= x0) {
      a = d.tf_alpha[0];
    } else if (v >= xn) {
      a = d.tf_alpha[np - 1];
    } else {
      a = d.tf_alpha[np - 1];
      for (int k = 0; k + 1 < np; ++k) {
        const double xa = (d.tf_x[k] - lo) / span, xb = (d.tf_x[k + 1] - lo) / span;
        if (v >= xa && v <= xb) {
          a = xb > xa ? d.tf_alpha[k] + (v - xa) / (xb - xa) * (d.tf_alpha[k + 1] - d.tf_alpha[k]) : d.tf_alpha[k + 1];
          break;
        }
      }
    }
    for (int k = 0; k < 3; ++k) rgba[4 * i + k] = (float)c[k];
    rgba[4 * i + 3] = (float)a;
  }
}

// The orbit camera: looks at the bounds' centre from distance |diag| / 2 /
// tan(fov/2) (the bounding sphere fills the vertical field of view), azimuth
// about +y from +z, elevation above the xz plane. (The reference's
// vtkm::rendering::Camera::ResetToBounds + Azimuth + Elevation are not
// vendored here; this is this build's definition of those two angles.)
void orbit_camera(const beams_scene_desc& d, const double lo[3], const double hi[3], beams_camera& c) {
  double ctr[3], diag = 0;
  for (int k = 0; k < 3; ++k) {
    ctr[k] = 0.5 * (lo[k] + hi[k]);
    diag += (hi[k] - lo[k]) * (hi[k] - lo[k]);
  }
  diag = std::sqrt(diag);
  const double fov = d.fov_y_deg * M_PI / 180.0;
  const double dist = 0.5 * diag / std::tan(0.5 * fov);
  const double az = d.azimuth * M_PI / 180.0, el = d.elevation * M_PI / 180.0;
  const double dir[3] = {std::cos(el) * std::sin(az), std::sin(el), std::cos(el) * std::cos(az)};
  const double up[3] = {-std::sin(el) * std::sin(az), std::cos(el), -std::sin(el) * std::cos(az)};
  for (int k = 0; k < 3; ++k) {
    c.position[k] = ctr[k] + dist * dir[k];
    c.look_at[k] = ctr[k];
    c.up[k] = up[k];
  }
  c.fov_y_deg = d.fov_y_deg;
  c.width = d.width;
  c.height = d.height;
}

}  // namespace
}  // namespace beams

using namespace beams;

extern "C" {

beams_status beams_generate_spheres(float* dev_out, const int n[3], const double origin[3], const double spacing[3],
                                    const float* ellipsoids, int n_ellipsoids, float default_value, int has_floor,
                                    float floor_height, float floor_value, void* cuda_stream) {
  if (!dev_out || !n || !origin || !spacing || n_ellipsoids < 0 || n_ellipsoids > 4096 ||
      (n_ellipsoids > 0 && !ellipsoids))
    return fail(nullptr, BEAMS_ERR_INVALID_ARG, "generate_spheres: bad arguments");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  float* d_e = nullptr;
  cudaError_t e = cudaSuccess;
  if (n_ellipsoids > 0) {
    e = cudaMalloc((void**)&d_e, (size_t)n_ellipsoids * 8 * sizeof(float));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_e, ellipsoids, (size_t)n_ellipsoids * 8 * sizeof(float), cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) {
    const long long total = (long long)n[0] * n[1] * n[2];
    const unsigned blocks = (unsigned)std::min<long long>((total + 255) / 256, 148 * 32);
    k_spheres<<<blocks, 256, 0, st>>>(dev_out, n[0], n[1], n[2], (float)origin[0], (float)origin[1], (float)origin[2],
                                      (float)spacing[0], (float)spacing[1], (float)spacing[2], d_e, n_ellipsoids,
                                      default_value, has_floor, (float)origin[1] + floor_height, floor_value);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (d_e) cudaFree(d_e);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "generate_spheres");
  return BEAMS_OK;
}

// The "vtk_file" provider: a legacy VTK volume from disk (the reference's
// FileDescriptor scenes, read through pilot/io/DataSetUtils.cxx:13-42).
static beams_status load_vtk_scene(beams_renderer* r, const beams_scene_desc* d, int cells[3], double org[3],
                                   double hi[3]) {
  if (!d->file_name[0]) return fail(r, BEAMS_ERR_CONFIG, "apply_scene: vtk_file provider without file_name");
  beams_vtk_field f;
  beams_status s = beams_vtk_read(d->file_name, &f);
  if (s != BEAMS_OK) return fail(r, s, std::string("apply_scene: ") + beams_last_error(nullptr));
  beams_volume v;
  std::memset(&v, 0, sizeof(v));
  v.data = f.data;
  v.dtype = BEAMS_F32;
  v.assoc = f.assoc;
  v.on_device = 0;
  for (int k = 0; k < 3; ++k) {
    v.dims[k] = f.dims[k];
    v.origin[k] = f.origin[k];
    v.spacing[k] = f.spacing[k];
    cells[k] = f.dims[k] - 1;
  }
  v.range[0] = f.range[0];
  v.range[1] = f.range[1];
  s = beams_set_volume(r, &v);
  if (s == BEAMS_OK) {
    const cudaError_t e = cudaStreamSynchronize(r->stream);  // the host copy is freed below
    if (e != cudaSuccess) s = cuda_fail(r, e, "apply_scene: volume upload");
  }
  if (s == BEAMS_OK && f.coords[0]) s = beams_set_volume_coordinates(r, f.coords[0], f.coords[1], f.coords[2]);
  for (int k = 0; k < 3; ++k) {
    org[k] = f.coords[k] ? (double)f.coords[k][0] : (double)(float)f.origin[k];
    hi[k] = f.coords[k] ? (double)f.coords[k][f.dims[k] - 1]
                        : (double)((float)f.origin[k] + (float)f.spacing[k] * (float)(f.dims[k] - 1));
  }
  beams_vtk_free(&f);
  return s;
}

// The generated providers (SceneFactory / DataSetFactory): the field on
// [0,1]^3 with cell_dims + 1 points per axis, generated on the device.
static beams_status generate_scene(beams_renderer* r, const beams_scene_desc* d, double org[3], double hi[3]) {
  int pts[3];
  double sp[3];
  for (int k = 0; k < 3; ++k) {
    pts[k] = d->cell_dims[k] + 1;
    if (d->cell_dims[k] < 1) return fail(r, BEAMS_ERR_CONFIG, "apply_scene: cell_dims must be positive");
    sp[k] = 1.0 / d->cell_dims[k];  // the reference's spacing 1 / size (SubdividedSpheresScene.cxx)
    hi[k] = (double)((float)org[k] + (float)sp[k] * (float)d->cell_dims[k]);
  }
  const size_t count = (size_t)pts[0] * pts[1] * pts[2];
  // the generated field is owned by the renderer
  beams_status s = ensure_buffer(r, &r->d_field_owned, &r->field_cap, count * sizeof(float), "allocating volume");
  if (s != BEAMS_OK) return s;
  float* f = (float*)r->d_field_owned;
  const std::string type = d->provider_type;
  if (type == "subdivided_spheres" || type == "spheres") {
    std::vector<float> e;
    float def = 0.1f;
    int floor = 0;
    if (type == "subdivided_spheres") {
      e = {0.5f, 0.5f, 0.5f, 0.45f, 0.45f, 0.45f, 1.f, 1.f};  // SubdividedSpheresScene.cxx
    } else {
      e = {0.5f, 0.5f, 0.5f, 0.1f, 0.1f, 0.1f, 1.f, 1.f};  // SpheresScene.cxx: centre sphere and floor
      floor = 1;
    }
    s = beams_generate_spheres(f, pts, org, sp, e.data(), 1, def, floor, -0.01f, 0.7f, r->stream);
  } else if (type == "blobs") {
    // 8 seeded blobs as in the 128^3 blob workload (centres U[0.2,0.8], sigma U[0.05,0.15], amplitude U[0.5,1])
    std::vector<float> prm;
    unsigned x = d->seed * 2654435761u + 12345u;
    auto u01 = [&]() {
      x ^= x << 13;
      x ^= x >> 17;
      x ^= x << 5;
      return (float)(x >> 8) * (1.f / 16777216.f);
    };
    for (int b = 0; b < 8; ++b) {
      prm.push_back(0.2f + 0.6f * u01());
      prm.push_back(0.2f + 0.6f * u01());
      prm.push_back(0.2f + 0.6f * u01());
      prm.push_back(0.05f + 0.1f * u01());
      prm.push_back(0.5f + 0.5f * u01());
    }
    s = beams_generate_blobs(f, pts, prm.data(), 8, 1, r->stream);
  } else if (type == "noise") {
    unsigned char perm[256];
    for (int i = 0; i < 256; ++i) perm[i] = (unsigned char)i;
    unsigned x = d->seed * 2654435761u + 777u;
    for (int i = 255; i > 0; --i) {
      x ^= x << 13;
      x ^= x >> 17;
      x ^= x << 5;
      const int j = (int)(x % (unsigned)(i + 1));
      std::swap(perm[i], perm[j]);
    }
    s = beams_generate_noise(f, pts, perm, d->octaves, d->base_freq, 2.f, 0.5f, r->stream);
  } else {
    return fail(r, BEAMS_ERR_CONFIG, "apply_scene: unknown dataset provider type");
  }
  if (s != BEAMS_OK) return fail(r, s, std::string("apply_scene: dataset: ") + beams_last_error(nullptr));
  beams_volume v;
  std::memset(&v, 0, sizeof(v));
  v.data = f;
  v.dtype = BEAMS_F32;
  for (int k = 0; k < 3; ++k) {
    v.dims[k] = pts[k];
    v.origin[k] = org[k];
    v.spacing[k] = sp[k];
  }
  v.range[0] = 0.0;
  v.range[1] = 1.0;
  v.assoc = BEAMS_ASSOC_POINTS;
  v.on_device = 1;
  s = beams_set_volume(r, &v);
  if (s != BEAMS_OK) return s;
  return BEAMS_OK;
}

beams_status beams_apply_scene(beams_renderer* r, const beams_scene_desc* d, beams_camera* camera_out) {
  if (!r || !d) return fail(r, BEAMS_ERR_INVALID_ARG, "apply_scene: NULL argument");
  cudaSetDevice(r->device);
  int cells[3];
  double org[3] = {0, 0, 0}, hi[3];
  beams_status s;
  if (std::string(d->provider_type) == "vtk_file") {
    s = load_vtk_scene(r, d, cells, org, hi);
  } else {
    s = generate_scene(r, d, org, hi);
    for (int k = 0; k < 3; ++k) cells[k] = d->cell_dims[k];
  }
  if (s != BEAMS_OK) return s;
  std::vector<float> tf;
  build_table(*d, tf);
  s = beams_set_color_map(r, tf.data(), d->tf_size);
  if (s != BEAMS_OK) return s;
  int m[3];
  for (int k = 0; k < 3; ++k) {
    if (d->shadow_size[k] > 0) m[k] = d->shadow_size[k];
    else if (d->shadow_size_ratio > 0.f) m[k] = std::max(1, (int)((float)cells[k] * d->shadow_size_ratio));
    else m[k] = 16;  // LightedVolumeRenderer.cxx:752-759
  }
  s = beams_set_shadow_map_size(r, m[0], m[1], m[2]);
  if (s == BEAMS_OK) s = beams_set_use_shadow_map(r, d->shadow_enabled);
  if (s == BEAMS_OK) s = beams_set_light_steps(r, d->light_steps);
  if (s == BEAMS_OK) s = beams_clear_lights(r);
  if (s != BEAMS_OK) return s;
  if (d->n_lights > 0) {
    const beams_config_light& L = d->lights[0];  // the reference uses Locations[0] only
    s = L.kind == 1 ? beams_add_directional_light(r, L.position, L.color, L.intensity)
                    : beams_add_point_light(r, L.position, L.color, L.intensity);
  } else {
    const double pos[3] = {0.5, 5.0, 0.5};  // SubdividedSpheresScene::Ready
    const float col[3] = {1.f, 1.f, 1.f};
    s = beams_add_point_light(r, pos, col, 2.f);
  }
  if (s != BEAMS_OK) return s;
  if (d->sample_distance > 0.f) s = beams_set_sample_distance(r, d->sample_distance);
  if (s == BEAMS_OK) s = beams_set_termination_alpha(r, d->termination_alpha);
  if (s == BEAMS_OK) s = beams_set_background(r, d->composite_background, d->background);
  if (s != BEAMS_OK) return s;
  if (d->form == BEAMS_FORM_PRECISION) {
    beams_precision_options po{d->field_dtype};
    s = beams_set_form(r, BEAMS_FORM_PRECISION, &po);
  } else if (d->form == BEAMS_FORM_MLP) {
    beams_mlp_options o;
    std::memset(&o, 0, sizeof(o));
    o.samples_log2 = d->mlp_samples_log2;
    o.n_lights = d->mlp_lights;
    o.epochs = 4;
    o.batch = 16384;
    o.lr = 2e-3f;
    o.seed = d->seed;
    o.fallback_tol = d->mlp_fallback_tol;
    o.probe_fraction = d->mlp_probe_fraction;
    o.knot = d->mlp_knot;
    o.focus = 0.875f;
    s = beams_set_form(r, BEAMS_FORM_EXACT, nullptr);
    if (s == BEAMS_OK) s = beams_mlp_train(r, &o, nullptr);
    if (s == BEAMS_OK) s = beams_set_form(r, BEAMS_FORM_MLP, &o);
  } else {
    s = beams_set_form(r, BEAMS_FORM_EXACT, nullptr);
  }
  if (s != BEAMS_OK) return s;
  if (camera_out) {
    beams_camera c;
    std::memset(&c, 0, sizeof(c));
    if (d->camera_explicit) {
      for (int k = 0; k < 3; ++k) {
        c.position[k] = d->position[k];
        c.look_at[k] = d->look_at[k];
        c.up[k] = d->up[k];
      }
      c.fov_y_deg = d->fov_y_deg;
      c.width = d->width;
      c.height = d->height;
    } else {
      orbit_camera(*d, org, hi, c);
    }
    *camera_out = c;
  }
  return BEAMS_OK;
}

beams_status beams_scene_color_table(const beams_scene_desc* d, float* rgba, int n) {
  if (!d || !rgba || n != d->tf_size || d->tf_points < 1) return BEAMS_ERR_INVALID_ARG;
  std::vector<float> tf;
  build_table(*d, tf);
  std::memcpy(rgba, tf.data(), tf.size() * sizeof(float));
  return BEAMS_OK;
}

beams_status beams_orbit_light(beams_renderer* r, const beams_scene_desc* d, int frame) {
  if (!r || !d) return fail(r, BEAMS_ERR_INVALID_ARG, "orbit_light: NULL argument");
  const double phi = (double)frame * 5.0 * M_PI / 180.0;
  const double pos[3] = {0.5 + 0.5 * std::cos(phi), 0.5 + 0.5 * std::sin(phi), 0.5};
  float col[3] = {1.f, 1.f, 1.f};
  float inten = 2.f;
  if (d->n_lights > 0) {
    for (int k = 0; k < 3; ++k) col[k] = d->lights[0].color[k];
    inten = d->lights[0].intensity;
  }
  beams_status s = beams_clear_lights(r);
  if (s == BEAMS_OK) s = beams_add_point_light(r, pos, col, inten);
  return s;
}

}  // extern "C"
