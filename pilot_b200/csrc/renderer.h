// renderer.h — the opaque beams_renderer behind the C ABI.
//
// Mirrors the state of MapperLightedVolume::InternalsType
// (beams/rendering/MapperLightedVolume.cxx:27-45) and LightedVolumeRenderer
// (beams/rendering/LightedVolumeRenderer.h:231-261), with device buffers.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/beams_b200.h"
#include "beams_params.h"

namespace beams {

struct MlpState;    // learned form (mlp_api.cu)
struct BatchState;  // batched form (batch_api.cu)

struct Light {
  int kind = 0;  // 0 point, 1 directional
  double v[3] = {0, 0, 0};
  float color[3] = {1, 1, 1};
  float intensity = 1.f;
};

// One block of a multi-block scene: its own field and derived buffers (the
// reference holds one block per MPI rank; here all blocks share one GPU).
// What the lazy map's cell marks depend on: the view rays and their samples
// (volume, colour map, canvas depth, camera, window, sample distance,
// termination, slab mode, value range, and the form with its field's type,
// whose rounding moves the samples' values) and the map grid; not the light.
struct MarkKey {
  unsigned long long volume_version, tf_version, depth_version;
  float cam[12], k[4], sd, mesh_eps, cutoff, min_scalar, inv_delta, morig[3], minv[3];
  int size[2], win[4], slab_fp64, pd[3], form, quad_dtype;
};

struct Brick {
  beams_volume vol{};
  void* d_field_owned = nullptr;
  size_t field_cap = 0;
  const void* d_field = nullptr;
  unsigned long long version = 0;
  float4* d_quads = nullptr;
  size_t quads_cap = 0;
  unsigned long long quads_version = 0;
  float4* d_tab = nullptr;
  size_t tab_cap = 0;
  unsigned long long tab_key[4] = {0, 0, 0, 0};
  float* d_map_local = nullptr;
  size_t local_cap = 0;
  float* d_map_final = nullptr;
  size_t final_cap = 0;
  size_t map_count = 0;
  // the lazy map (beams_set_lazy_shadow_map): the cells this brick's view rays
  // read and their corner vertices; the stitched map is then partial
  unsigned char* d_cell_mask = nullptr;
  size_t cell_mask_cap = 0;
  unsigned* d_vlist = nullptr;
  size_t vlist_cap = 0;
  bool final_partial = false;
  bool marks_valid = false;  // mode 2: this brick's marks kept while mark_key matches
  MarkKey mark_key{};
  void release() {
    if (d_field_owned) cudaFree(d_field_owned);
    if (d_quads) cudaFree(d_quads);
    if (d_tab) cudaFree(d_tab);
    if (d_map_local) cudaFree(d_map_local);
    if (d_map_final) cudaFree(d_map_final);
    if (d_cell_mask) cudaFree(d_cell_mask);
    if (d_vlist) cudaFree(d_vlist);
    d_cell_mask = nullptr;
    d_vlist = nullptr;
    cell_mask_cap = vlist_cap = 0;
    d_field_owned = d_quads = nullptr;
    d_quads = nullptr;
    d_tab = nullptr;
    d_map_local = d_map_final = nullptr;
  }
};

struct MapKey {
  unsigned long long volume_version;
  unsigned long long tf_version;
  int m[3];
  float steps;
  int form;
  int light_kind;
  double light[3];
  int n_lights;          // the multi-light extension: lights 1.. below
  int extra_kind[8];
  double extra[8][3];
};

}  // namespace beams

struct beams_renderer {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;

  // volume (SetData)
  bool has_volume = false;
  beams_volume vol{};
  void* d_field_owned = nullptr;
  size_t field_cap = 0;
  const void* d_field = nullptr;
  size_t field_bytes = 0;
  unsigned long long volume_version = 0;

  // colour map (SetColorMap)
  std::vector<float> tf;
  float4* d_tf = nullptr;
  size_t tf_cap = 0;
  int tf_n = 0;
  unsigned long long tf_version = 0;

  // lights, map and march settings; defaults are the reference's
  // (LightedVolumeRenderer.cxx:752-759: shadow map on, 16^3, sample distance -1).
  std::vector<beams::Light> lights;
  int map_m[3] = {16, 16, 16};
  bool use_map = true;
  float sample_distance = -1.f;
  float cutoff = 1.f;
  float density_scale = 1.f;  // SetDensityScale: stored, never read (as in the reference)
  float light_steps = 128.f;
  int slab_fp64 = 1;
  int light_brick_log2 = 3;  // beams_set_tuning (8^3-vertex bricks)
  bool reuse_map = false;
  // beams_set_lazy_shadow_map: the exact form builds only the map vertices
  // that the frame's view rays read (d_cell_mask marks their cells)
  bool lazy_map = false;
  bool keep_marks = false;    // mode 2: marks kept while mark_key matches
  bool marks_valid = false;
  beams::MarkKey mark_key{};
  unsigned char* d_cell_mask = nullptr;
  size_t cell_mask_cap = 0;
  // the masked map builds' vertex list ((M+1)^3 + 1 entries: count, then ids),
  // shared by the lazy map, the learned form's fallback and the bricks' Phase 1
  unsigned* d_vlist = nullptr;
  size_t vlist_cap = 0;
  bool bg = false;
  float bg_rgba[4] = {1.f, 1.f, 1.f, 1.f};
  // explicit rectilinear coordinates of the volume's point axes (beams_set_volume_coordinates)
  bool rect = false;
  std::vector<float> coords[3];
  // canvas depth buffer (beams_set_depth_buffer) and the per-pixel ray limits derived from it
  bool depth_set = false;
  unsigned long long depth_version = 0;  // bumped by every beams_set_depth_buffer
  int depth_w = 0, depth_h = 0, depth_kind = 0;
  double depth_near = 0.0, depth_far = 0.0;
  float* d_depth = nullptr;
  size_t depth_cap = 0;
  float* d_raymax = nullptr;
  size_t raymax_cap = 0;
  int form = BEAMS_FORM_EXACT;
  beams_profile_fn profile_fn = nullptr;  // beams_set_profiler
  void* profile_user = nullptr;

  // transmittance map
  float* d_map = nullptr;
  size_t map_cap = 0;
  size_t map_count = 0;
  bool map_valid = false;
  beams::MapKey map_key{};
  bool map_is_half = false;  // precision form: binary16 transmittance

  // precision form
  int prec_dtype = BEAMS_BF16;
  std::vector<float> tau;     // -ln(1 - a_i) per TF entry
  float* d_tau = nullptr;
  size_t tau_cap = 0;

  // derived layouts: 4-corner quads of the field, per-axis cell tables
  void* d_quads = nullptr;                // float4 (exact) or 8-byte 16-bit quads (precision)
  size_t quads_cap = 0;
  unsigned long long quads_version = 0;  // volume_version * 4 + quad dtype the quads were built from
  float4* d_tab = nullptr;
  size_t tab_cap = 0;
  unsigned long long tab_key[4] = {0, 0, 0, 0};  // volume_version, map m[3] packed
  // empty-space occupancy of 8^3-cell macro-cells (light-march skip)
  unsigned char* d_occ = nullptr;
  size_t occ_cap = 0;
  unsigned long long occ_key[2] = {~0ull, ~0ull};  // quads key, tf_version
  int empty_skip = 1;  // map build skips empty macro-cells
  int view_skip = 1;   // view march skips empty macro-cells
  int multi_light = 0; // beams_set_multi_light: shade by every light (one map each)

  // multi-block scene (beams_set_bricks)
  std::vector<beams::Brick> bricks;
  bool brick_mode = false;
  beams::BrickRef* d_refs = nullptr;
  size_t refs_cap = 0;
  float4* d_brick_imgs = nullptr;
  size_t brick_imgs_cap = 0;
  unsigned long long brick_counter = 0;
  // Per-brick launches run on kBrickLanes side streams (fork/join by events),
  // so one brick's launch fills the SMs that the previous one's tail leaves
  // idle; each brick has its own work counters (d_brick_cnt[b]).
  static constexpr int kBrickLanes = 4;
  cudaStream_t brick_lane[kBrickLanes] = {nullptr, nullptr, nullptr, nullptr};
  unsigned char* d_shell_mask = nullptr;  // Phase 1's outer-cell-layer mask
  bool shell_listed = false;              // this frame's Phase 1 ran over the shell's list (d_vlist)
  size_t shell_cap = 0;
  int shell_pd[3] = {0, 0, 0};
  cudaEvent_t brick_fork = nullptr;
  cudaEvent_t brick_join[kBrickLanes] = {nullptr, nullptr, nullptr, nullptr};
  beams::Counters* d_brick_cnt = nullptr;  // kMaxBricks entries

  // learned form: parameters, optimiser state, inference weights
  beams::MlpState* mlp = nullptr;
  beams::BatchState* batch = nullptr;

  // image + counters + timing
  float4* d_rgba = nullptr;
  size_t rgba_cap = 0;
  beams::Counters* d_cnt = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  ~beams_renderer();
  void release_buffers() {
    if (d_field_owned) cudaFree(d_field_owned);
    if (d_tf) cudaFree(d_tf);
    if (d_map) cudaFree(d_map);
    if (d_quads) cudaFree(d_quads);
    if (d_tab) cudaFree(d_tab);
    if (d_occ) cudaFree(d_occ);
    if (d_tau) cudaFree(d_tau);
    if (d_rgba) cudaFree(d_rgba);
    if (d_depth) cudaFree(d_depth);
    if (d_raymax) cudaFree(d_raymax);
    for (auto& b : bricks) b.release();
    if (d_refs) cudaFree(d_refs);
    if (d_brick_imgs) cudaFree(d_brick_imgs);
    if (d_brick_cnt) cudaFree(d_brick_cnt);
    if (d_shell_mask) cudaFree(d_shell_mask);
    if (d_cell_mask) cudaFree(d_cell_mask);
    if (d_vlist) cudaFree(d_vlist);
    for (auto& s : brick_lane)
      if (s) cudaStreamDestroy(s);
    for (auto& e : brick_join)
      if (e) cudaEventDestroy(e);
    if (brick_fork) cudaEventDestroy(brick_fork);
    if (d_cnt) cudaFree(d_cnt);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

namespace beams {
void mlp_release(beams_renderer* r);
void batch_release(beams_renderer* r);
beams_status fail(beams_renderer* r, beams_status s, const std::string& msg);
beams_status cuda_fail(beams_renderer* r, cudaError_t e, const char* what);
beams_status ensure_buffer(beams_renderer* r, void** buf, size_t* cap, size_t bytes, const char* what);
// The map of a masked build: the vertices it does not build are still read by
// samples of premultiplied alpha 0 (which add 0 times their shading, exactly 0
// for any finite value), so a newly allocated buffer is zeroed on st, and so
// is a reused one when clear is set (its data came in another format).
beams_status ensure_masked_map(beams_renderer* r, float** buf, size_t* cap, size_t bytes, cudaStream_t st,
                               bool clear);
beams_status prepare_ray_limits(beams_renderer* r, ExactGeo& g, int& launches);
beams_status blend_background(beams_renderer* r, float4* img, size_t npix, int& launches);
}  // namespace beams

inline beams_renderer::~beams_renderer() {
  beams::mlp_release(this);
  beams::batch_release(this);
  release_buffers();
}
