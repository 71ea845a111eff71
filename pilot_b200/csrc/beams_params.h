// beams_params.h — kernel parameter blocks, derived on the host from the scene
// exactly as the reference derives them (float32 arithmetic, no contraction).
#pragma once
#include <stdint.h>

namespace beams {

// Everything the exact light and view marches need, passed by value.
struct ExactGeo {
  // Field grid. Rectilinear coordinates are generated, not stored:
  // coord(d, i) = org[d] + h[d] * float(i), the float32 ArrayHandleCounting the
  // reference scenes build (beams/sources/Spheres.cxx:144-156).
  int n[3];
  float org[3], h[3], invh[3];  // invh only seeds the cell search
  float minp[3], maxp[3];       // coord(d,0), coord(d,n-1)
  double bmin[3], bmax[3];      // vtkm::Bounds of the coordinates (double)
  float min_scalar, inv_delta;  // LightedVolumeRenderer.cxx:331-334
  // Transfer function (RGBA table in global memory, staged to shared memory).
  int tf_n;
  float max_alpha;              // TransmittanceMap.h:515-525
  // Map grid: (M+1)^3 vertices over the field bounds (TransmittanceMap.h:550-563).
  int pd[3];
  float morig[3], msp[3], minv[3];
  float light_color[3];         // Color * Intensity (LightedVolumeRenderer.cxx:840)
  float extent_mag;             // BoundsMagnitude (beams/Math.h:13-21)
  float sd;                     // view sample distance
  float mesh_eps;               // |extent| * 1e-4 (LightedVolumeRenderer.cxx:1261)
  float step;                   // light step |extent| / steps (TransmittanceMap.h:584-585)
  float cutoff;                 // early-termination alpha
  int light_kind;               // 0 point, 1 directional
  float light[3];               // position, or normalised travel direction
  float dir_dist;               // directional light: per-vertex origin distance
  int light_budget;             // iteration cap of one light ray
  // Camera (pinhole, pixel centres).
  float cam_pos[3], cf[3], cr[3], cu[3];
  float kx, cx, ky, cy;
  int width, height;
  int slab_fp64;
  int use_map;
  int assoc_cells;
  // Cell tables: per axis, one float4 {lo, hi, RN(1/(hi-lo)), 0} per cell, field
  // axes first (n-1 cells each), then map axes (M cells each).
  int ax_off[3];   // offset of field axis d in the table
  int max_off[3];  // offset of map axis d in the table
  int ntab;        // total table entries
  // K1 vertex order: 0 = x-fastest rows of the vertex grid; b > 0 = cubic
  // bricks of 2^b vertices per edge in brick order (rays in flight stay in a
  // narrow cone towards the light, so the field they read stays in L2).
  int light_brick_log2;
  // Brick order that follows the light: bricks are visited in pencils along
  // bo_axis[0] (the axis the light travels most along, in map-vertex units),
  // the two other brick coordinates (bo_axis[1], bo_axis[2]) sheared by
  // floor(w * bo_shear / 65536) modulo their brick counts, so that a pencil
  // tracks the light rays through the brick grid; pencils in raster order.
  // The bricks in flight then sit in a few adjacent pencils and their light
  // rays cross one narrow region of the field. Any order gives the same map.
  int bo_axis[3];
  int bo_shear[2];
  // Occupancy of 8^3-cell macro-cells (empty-space skipping): counts per axis.
  int occ_n[3];
  // The multi-light extension: n_lights maps, map l at map + l * (M+1)^3, the
  // view march shading by sum_l T_l * light_colors[l] (n_lights <= 1: light 0 only).
  int n_lights;
  float light_colors[8][3];
  // Explicit rectilinear coordinates (beams_set_volume_coordinates): the field
  // axes' cell tables hold the given coordinates and cells are found by
  // search instead of from the uniform spacing; org/h/invh then only describe
  // the average spacing. 0: coord(d, i) = org[d] + h[d] * float(i).
  int rect;
  // Loop constants the exact light march takes from the kernel's parameter
  // space (the constant bank) instead of holding them in registers (set by
  // geo_loop_constants): per field axis the cell guess's upper clamp n - 2 as
  // a float, the quad strides (n0 - 1) and (n0 - 1)(n1 - 1), and the TF's last
  // index as a float. The 257^3-vertex map of a 512^3 noise field: 2.59 ->
  // 2.38 ms against the same values derived in the kernel.
  float cmaxf[3];
  unsigned qxs, qzs;
  float n1f;
  // Pixel window {x0, y0, w, h} the (non-listed) view march covers; the whole
  // image unless a brick's projection is known to lie inside a smaller one
  // (every pixel outside it misses the volume).
  int win[4];
  // Canvas depth clipping: per-pixel limit on each camera ray's distance
  // (width * height floats, row y at y * width), the MaxDistance that
  // MapCanvasToRays hands the slab test (MapperLightedVolume.cxx:151-152).
  // Null: no limit.
  const float* ray_max;
};

constexpr int kMaxMultiLights = 8;

constexpr int kMacroLog2 = 3;  // macro-cell edge = 8 field cells

// What the stitch kernel needs of every other brick (multi-block scenes): its
// bounds (for SegmentAABB) and its Phase-1 map with that map's geometry.
struct BrickRef {
  double bmin[3], bmax[3];
  float morig[3], msp[3], minv[3];
  int pd[3];
  const float* map;
};

constexpr int kMaxBricks = 32;
// Learned form: pixel tile that falls back to the exact map as a unit.
constexpr int kFallbackTile = 32;

// Counters written by the kernels (one atomic per warp).
struct Counters {
  unsigned long long light_samples;
  unsigned long long lit_samples;
  unsigned long long rays_hit;
  unsigned long long mlp_samples;
  unsigned long long fallback_tiles;
  unsigned long long errors;
  unsigned int tiles_light;   // persistent-block work counters (zeroed per frame)
  unsigned int tiles_view;
  unsigned long long mlp_rows;  // network rows computed (idle lanes included)
  unsigned long long map_vertices;  // vertices a masked (lazy) light march built
  unsigned int tiles_mark;  // the map-cell marking pass's tile counter (zeroed by its launcher)
  unsigned int reserved;
};

// Derives ExactGeo's loop constants from n[] and tf_n.
inline void geo_loop_constants(ExactGeo& g) {
  for (int d = 0; d < 3; ++d) g.cmaxf[d] = (float)(g.n[d] - 2);
  g.qxs = (unsigned)(g.n[0] - 1);
  g.qzs = g.qxs * (unsigned)(g.n[1] - 1);
  g.n1f = (float)(g.tf_n - 1);
}

}  // namespace beams
