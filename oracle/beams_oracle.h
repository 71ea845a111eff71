/*
 * beams_oracle.h — CPU oracle for the Beams lighted volume renderer hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker: a plain C++ restatement of the
 * reference worklets, used by the tests, by smoke() and as the CPU baseline.
 * Nothing in the product library links, loads or calls it.
 *
 * Parity is UNPINNED: the reference ships no tests, golden images or fixtures,
 * and it cannot be built here (VTK-m 1.9, MPI, fmt and toml++ are absent and its
 * driver's Run() body is commented out). The restatement follows the reference
 * source line by line; the few VTK-m internals it relies on are restated from
 * their published definitions (see beams_oracle.cpp).
 *
 * Two modes share one template: "f32" repeats the reference's float32 arithmetic
 * (no FMA contraction, IEEE division and sqrt), "f64" is the same algorithm in
 * double precision and is the accuracy yardstick.
 */
#ifndef BEAMS_ORACLE_H
#define BEAMS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene {
  const float* field;   /* point field, x fastest */
  int dims[3];          /* point dims */
  double origin[3];
  double spacing[3];
  double range[2];
  const float* tf;      /* tf_n x RGBA */
  int tf_n;
  int light_kind;       /* 0 point, 1 directional */
  double light[3];      /* position, or travel direction */
  float light_color[3];
  float light_intensity;
  int map_m[3];         /* cells per axis of the map */
  int use_map;
  float sample_distance;/* <= 0: |extent| / 200 (LightedVolumeRenderer.cxx:815-819) */
  float alpha_cutoff;   /* reference: 1.0 */
  float light_steps;    /* reference: 128 */
  int slab_fp64;        /* 1: slab test in double, rounded to float (f32 mode) */
  double cam_pos[3];
  double cam_look[3];
  double cam_up[3];
  double fov_y_deg;
  int width;
  int height;
  /* 0: the reference algorithm. 1: the precision form — optical depth
   * tau = sum -ln(1 - a_i) accumulated in float with Kahan compensation (a_i = 1
   * cuts the ray), the map stores transmittance T = exp(-tau) rounded to IEEE
   * binary16, and the view march shades by the interpolated T. */
  int precision;
  /* Canvas depth clipping: width x height per-pixel limits on the camera ray's
   * distance (row y at y * width), the slab test's initial MaxDistance; NULL:
   * no limit (MapperLightedVolume.cxx:151-152, LightedVolumeRenderer.cxx:644-718). */
  const float* ray_max;
  /* Explicit rectilinear coordinates: dims[d] float32 values per axis (the
   * reference's ArrayHandleCartesianProduct); NULL: origin + spacing * i. */
  const float* coords[3];
} oracle_scene;

/* Light march over every map vertex ((M+1)^3, x fastest). */
int oracle_light_march_f32(const oracle_scene* s, float* map_out, int threads, uint64_t* samples);
int oracle_light_march_f64(const oracle_scene* s, double* map_out, int threads, uint64_t* samples);
/* Light march over a list of flat vertex ids only (bounded CPU samples). */
int oracle_light_march_ids_f32(const oracle_scene* s, const int64_t* ids, int64_t n, float* out,
                               int threads, uint64_t* samples);
int oracle_light_march_ids_f64(const oracle_scene* s, const int64_t* ids, int64_t n, double* out,
                               int threads, uint64_t* samples);
/* Transmittance 1 - o at arbitrary points (march from the light to each point). */
int oracle_light_march_points_f64(const oracle_scene* s, const double* pts, int64_t n,
                                  const double* light_pos, double* opacity_out, int threads);
int oracle_light_march_points_f32(const oracle_scene* s, const float* pts, int64_t n, const float* light_pos,
                                  float* out, int threads);

/* View march over the pixel window [x0,x0+w) x [y0,y0+h); rgba_out is w*h*4.
 * map may be NULL when use_map == 0. lazy != 0: ignore map and compute the map
 * vertices a lookup needs on demand (memoised). */
int oracle_view_march_f32(const oracle_scene* s, const float* map, int x0, int y0, int w, int h,
                          float* rgba_out, int threads, uint64_t* lit_samples);
int oracle_view_march_f64(const oracle_scene* s, const double* map, int x0, int y0, int w, int h,
                          double* rgba_out, int threads, uint64_t* lit_samples);
/* Cell-associated field (SamplerCellAssoc): s->field holds (dims-1)^3 cell
 * values, x fastest; unlit, use_map is ignored. rgba_out is w*h*4. */
int oracle_view_march_cells_f32(const oracle_scene* s, int x0, int y0, int w, int h, float* rgba_out, int threads,
                                uint64_t* lit_samples);
int oracle_view_march_cells_f64(const oracle_scene* s, int x0, int y0, int w, int h, double* rgba_out, int threads,
                                uint64_t* lit_samples);
/* Per-pixel ray limits of a window-depth buffer (OpenGL depth in [0, 1] under
 * the camera's perspective with near/far planes, unprojected at the pixel
 * centre: t = 2fn / ((f + n) - (2d - 1)(f - n)) times the length of the
 * un-normalised camera ray), in double. */
int oracle_window_depth_to_distance(const oracle_scene* s, const float* depth, double near_plane,
                                    double far_plane, double* out);
/* Multi-light extension: n_lights exact-form maps stacked in light order, shaded
 * with sum_l (1 - opacity_l) * light_colors[l] (colour * intensity, float32). */
int oracle_view_march_multi_f32(const oracle_scene* s, const float* maps, int n_lights, const float* light_colors,
                                int x0, int y0, int w, int h, float* rgba_out, int threads, uint64_t* lit_samples);
int oracle_view_march_lazy_f64(const oracle_scene* s, int x0, int y0, int w, int h, int stride,
                               double* rgba_out, int threads, uint64_t* lit_samples);

/* Lit samples of a pixel window in march order (x, y, z, r, g, b, sa per sample). */
int oracle_record_samples_f32(const oracle_scene* s, int x0, int y0, int w, int h, float* rec, int64_t cap,
                              int* counts);

/* Per-pixel slab test (t_enter, t_exit; miss -> t_enter = -1). */
int oracle_ray_setup_f32(const oracle_scene* s, int x, int y, float out[8]);

/* Multi-block render: scenes[b] describes block b (its own field, dims, origin,
 * spacing; camera, light, TF, map size shared). Outputs (each optional except
 * rgba): per-block Phase-1 maps and stitched final maps concatenated in block
 * order, per-block images (nbricks*W*H*4), the depth-ordered composite. */
int oracle_render_bricks_f32(const oracle_scene* scenes, int nbricks, float* maps_local, float* maps_final,
                             float* brick_images, float* rgba, int threads, uint64_t* lit);
int oracle_render_bricks_f64(const oracle_scene* scenes, int nbricks, double* maps_local, double* maps_final,
                             double* brick_images, double* rgba, int threads, uint64_t* lit);

/* Gradient-noise field (x fastest), remapped to [0,1]; the reference arm's input. */
int oracle_generate_noise(float* out, int nx, int ny, int nz, const unsigned char* perm, int octaves,
                          float f0, float lac, float gain, int threads);

/* The sphere / ellipsoid field of sources::Spheres (beams/sources/Spheres.cxx:36-91)
 * on the float32 grid origin + spacing * i: e = n x {cx, cy, cz, rx, ry, rz, min, max}. */
int oracle_generate_spheres(float* out, int nx, int ny, int nz, const float origin[3], const float spacing[3],
                            const float* e, int ne, float def, int has_floor, float floor_y, float floor_v);

/* Sort-last "over" of B premultiplied RGBA images in the given order
 * (MapperLightedVolume.cxx:284-297). */
int oracle_composite_f32(const float* images, int nimages, int npix, const int* order,
                         float* out);

#ifdef __cplusplus
}
#endif
#endif
