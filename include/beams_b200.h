/*
 * beams_b200.h — C ABI of the B200-native Beams lighted volume renderer.
 *
 * The library replaces the hot path behind beams::rendering::MapperLightedVolume
 * (beams/rendering/MapperLightedVolume.h:16-62) and LightedVolumeRenderer
 * (beams/rendering/LightedVolumeRenderer.h:20-101): the light-space march that
 * builds the (M+1)^3 transmittance ("opacity") map and the view-ray march that
 * samples the field, applies the transfer function, shades by the map and
 * composites front to back.
 *
 * Conventions
 *  - Every entry point returns a beams_status; no C++ exception crosses the ABI.
 *    The reference throws vtkm::cont::ErrorBadValue at the matching places.
 *  - Caller-owned inputs are copied unless the struct says on_device=1, in which
 *    case the device pointer is borrowed until the next set_* call or destroy.
 *  - One renderer per host thread. All GPU work is ordered on the stream given
 *    to beams_create (NULL = the legacy default stream); multi-brick frames
 *    fork their per-brick launches onto the renderer's own side streams and
 *    join them back onto it before the call returns.
 *  - Pixel (x, y) is stored at rgba[4*(y*width + x)], y = 0 is the bottom row.
 */
#ifndef BEAMS_B200_H
#define BEAMS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEAMS_ABI_VERSION 1

typedef enum beams_status {
  BEAMS_OK = 0,
  BEAMS_ERR_INVALID_ARG = 1,
  BEAMS_ERR_UNSUPPORTED = 2,
  BEAMS_ERR_CUDA = 3,
  BEAMS_ERR_OOM = 4,
  BEAMS_ERR_TIMEOUT = 5,
  BEAMS_ERR_CONFIG = 6,
  BEAMS_ERR_INTERNAL = 7,
  BEAMS_ERR_STATE = 8
} beams_status;

typedef enum beams_dtype { BEAMS_F32 = 0, BEAMS_BF16 = 1, BEAMS_F16 = 2 } beams_dtype;
typedef enum beams_assoc { BEAMS_ASSOC_POINTS = 0, BEAMS_ASSOC_CELLS = 1 } beams_assoc;

/* Render forms. EXACT is the reference algorithm in FP32. PRECISION stores the
 * field (BF16/F16, chosen by the volume dtype) and the map (F16) in 16 bits and
 * accumulates optical depth in FP32 with Kahan compensation. MLP replaces the
 * map build and lookup by a trained transmittance network. */
typedef enum beams_form { BEAMS_FORM_EXACT = 0, BEAMS_FORM_PRECISION = 1, BEAMS_FORM_MLP = 2 } beams_form;

/* Options of BEAMS_FORM_PRECISION: the dtype the field is stored and read in
 * (BEAMS_BF16 or BEAMS_F16) when the volume is given in float32; a 16-bit
 * volume is used as given. The map is binary16 transmittance exp(-tau). */
typedef struct beams_precision_options {
  int field_dtype;
} beams_precision_options;

/* A structured scalar volume on a uniform grid. The renderer builds the same
 * float32 rectilinear coordinate arrays the reference scenes build
 * (origin + i*spacing, beams/sources/Spheres.cxx:144-156). */
typedef struct beams_volume {
  const void* data;     /* dims[0]*dims[1]*dims[2] values, x fastest */
  int dtype;            /* beams_dtype */
  int dims[3];          /* point dimensions */
  double origin[3];
  double spacing[3];
  double range[2];      /* scalar range used to normalise (SetData's scalarRange) */
  int assoc;            /* beams_assoc */
  int on_device;        /* 1: data is a device pointer on the renderer's device */
} beams_volume;

/* Pinhole camera; rays through pixel centres. */
typedef struct beams_camera {
  double position[3];
  double look_at[3];
  double up[3];
  double fov_y_deg;
  int width;
  int height;
} beams_camera;

/* Filled by beams_render when a non-NULL pointer is given (the call then
 * synchronises the stream). Times are CUDA-event times on the renderer stream. */
typedef struct beams_timings {
  float map_build_ms;          /* light march (Phase 1 in the reference) */
  float view_march_ms;         /* slab + view march (Phase 4) */
  float composite_ms;          /* brick composite / copy-out (Phase 5) */
  float total_ms;
  unsigned long long light_samples;  /* light-march samples evaluated */
  unsigned long long lit_samples;    /* view samples composited */
  unsigned long long rays_hit;       /* view rays that entered the volume */
  unsigned long long mlp_samples;    /* view samples shaded by the MLP */
  int map_vertices;                  /* map vertices built this frame ((M+1)^3 per light, 0 if reused;
                                        fewer under the lazy map and the learned form's fallback) */
  int fallback_tiles;                /* MLP form: tiles that used the exact map */
  int kernel_launches;               /* kernels this call launched */
  unsigned long long mlp_rows;       /* learned form: network rows computed, idle lanes included */
} beams_timings;

typedef struct beams_renderer beams_renderer;

/* ---- lifetime ------------------------------------------------------------ */
/* Replaces MapperLightedVolume::MapperLightedVolume() (MapperLightedVolume.cxx:47-50)
 * and its InternalsType (MapperLightedVolume.cxx:27-45). */
beams_status beams_create(beams_renderer** out, int device, void* cuda_stream);
/* Replaces MapperLightedVolume::~MapperLightedVolume() (MapperLightedVolume.cxx:52). */
beams_status beams_destroy(beams_renderer* r);
/* Last error text of this renderer (thread-local text when r is NULL). */
const char* beams_last_error(const beams_renderer* r);
int beams_abi_version(void);

/* ---- scene setters --------------------------------------------------------- */
/* Replaces LightedVolumeRenderer::SetData (LightedVolumeRenderer.cxx:766-779),
 * called from MapperLightedVolume::RenderCells (MapperLightedVolume.cxx:160-161). */
beams_status beams_set_volume(beams_renderer* r, const beams_volume* v);
/* Replaces LightedVolumeRenderer::SetColorMap (LightedVolumeRenderer.cxx:761-764):
 * n RGBA entries, already sampled from the colour table. */
beams_status beams_set_color_map(beams_renderer* r, const float* rgba, int n);
/* Replaces MapperLightedVolume::SetShadowMapSize (MapperLightedVolume.cxx:101-104). */
beams_status beams_set_shadow_map_size(beams_renderer* r, int mx, int my, int mz);
/* Replaces MapperLightedVolume::SetUseShadowMap (MapperLightedVolume.cxx:96-99). */
beams_status beams_set_use_shadow_map(beams_renderer* r, int enable);
/* Replaces MapperLightedVolume::ClearLights (MapperLightedVolume.cxx:81-84). */
beams_status beams_clear_lights(beams_renderer* r);
/* Replaces MapperLightedVolume::AddLight with a PointLight (MapperLightedVolume.cxx:76-79,
 * LightedVolumeRenderer.cxx:835-841): light colour = color * intensity. Only the
 * first light shades, as in the reference (TransmittanceMap.h:591-592). */
beams_status beams_add_point_light(beams_renderer* r, const double pos[3], const float color[3],
                                   float intensity);
/* Extension (no reference counterpart; the reference has point lights only,
 * beams/rendering/PointLight.h:16-30): a directional light travelling along dir. */
beams_status beams_add_directional_light(beams_renderer* r, const double dir[3], const float color[3],
                                         float intensity);
/* Replaces MapperLightedVolume::SetSampleDistance (MapperLightedVolume.cxx:316-319) and
 * LightedVolumeRenderer::SetSampleDistance (LightedVolumeRenderer.cxx:1374-1379).
 * d <= 0 returns BEAMS_ERR_INVALID_ARG, where the reference throws. */
beams_status beams_set_sample_distance(beams_renderer* r, float d);
/* Replaces MapperLightedVolume::SetDensityScale (MapperLightedVolume.h:51,
 * MapperLightedVolume.cxx:86-89), which stores the value in the renderer
 * (LightedVolumeRenderer.h:71) where nothing reads it: stored here the same way,
 * with no effect on the image; beams_get_density_scale reads it back. */
beams_status beams_set_density_scale(beams_renderer* r, float scale);
beams_status beams_get_density_scale(const beams_renderer* r, float* scale);
/* Early-termination threshold on accumulated alpha. The reference breaks at
 * alpha >= 1.0 (LightedVolumeRenderer.cxx:491-492); 1.0 is the default. */
beams_status beams_set_termination_alpha(beams_renderer* r, float alpha);
/* Light-march step count over the volume diagonal; the reference fixes 128
 * (TransmittanceMap.h:584-585), which is the default. */
beams_status beams_set_light_steps(beams_renderer* r, float steps);
/* Slab test precision for view rays: 1 (default) = FP64 t_enter/t_exit,
 * 0 = the reference's FP32 rcp_safe form (LightedVolumeRenderer.cxx:644-718). */
beams_status beams_set_slab_fp64(beams_renderer* r, int enable);
/* Keep the last map when its inputs (volume, colour map, light, map size) did not
 * change. Off by default: the reference rebuilds the map every frame. */
beams_status beams_set_reuse_shadow_map(beams_renderer* r, int enable);
/* Extension (no reference counterpart; the reference builds every vertex,
 * TransmittanceMap.h:565-621): the exact form builds only the map vertices that
 * the frame's view rays read. A view march without shading (the samples and
 * their order do not depend on the map: early termination reads only the
 * colour map's alpha) marks the map cells the shading will interpolate at
 * samples of alpha above 0 (the others add 0 times their shading), then the
 * light march builds the corners of the marked cells. The image is the
 * full map's bit for bit; the map is partial, so beams_get_shadow_map returns
 * BEAMS_ERR_STATE after such a frame and the map is never reused.
 * beams_timings.map_vertices reports the vertices built. In a multi-block
 * scene each brick's view rays mark the cells of its stitched map (Phases 2-3)
 * and only their corners are stitched (beams_get_brick_map's stitched stage
 * then returns BEAMS_ERR_STATE; Phase 1 is unchanged). The precision form
 * builds its binary16 map the same way, marking over its 16-bit field. Off by
 * default; the learned form ignores it (its fallback is lazy already).
 * mode: 0 off, 1 on (the cells are marked every frame), 2 on and the marks are
 * kept while everything they depend on is unchanged: volume, colour map,
 * canvas depth, camera, sample distance, termination alpha, slab mode, form and
 * field type, and map size (not the light: a light orbit around a fixed camera
 * marks once). Other
 * values return BEAMS_ERR_INVALID_ARG. In a multi-block scene each brick
 * keeps its own marks the same way. */
beams_status beams_set_lazy_shadow_map(beams_renderer* r, int mode);
/* ---- legacy VTK files ---------------------------------------------------------
 * Replaces the reference's dataset read (pilot/io/DataSetUtils.cxx:13-42, VTK-m's
 * legacy reader) for structured volumes: DATASET STRUCTURED_POINTS or
 * RECTILINEAR_GRID, ASCII or BINARY, with POINT_DATA or CELL_DATA and one
 * one-component SCALARS array of any numeric type, read as float32 (x fastest).
 * coords[d] is NULL for STRUCTURED_POINTS; for RECTILINEAR_GRID it holds the
 * dims[d] axis coordinates (then origin/spacing give the first value and the
 * average spacing). Host memory, freed by beams_vtk_free. Host code only. */
typedef struct beams_vtk_field {
  int dims[3];        /* point dimensions */
  int assoc;          /* beams_assoc */
  double origin[3];
  double spacing[3];
  float* coords[3];
  float* data;
  double range[2];    /* min / max of the scalars */
  char name[64];
} beams_vtk_field;
beams_status beams_vtk_read(const char* path, beams_vtk_field* out);
void beams_vtk_free(beams_vtk_field* f);

/* Explicit rectilinear coordinates for the current volume, point or cell field
 * (after beams_set_volume): x, y, z hold dims[0], dims[1], dims[2] strictly increasing
 * float32 coordinates, the arrays of the ArrayHandleCartesianProduct coordinate
 * system that RenderCells receives (MapperLightedVolume.cxx:114-119) and that the
 * reference's RectilinearLocator and RectilinearMeshOracle search
 * (LightedVolumeRenderer.cxx:45-186, RectilinearMeshOracle.h:140-176). The
 * volume's origin/spacing are then ignored; the map grid spans the coordinates'
 * bounds. All three NULL return to uniform spacing; beams_set_volume also does.
 * Exact and precision forms of a single volume with one light (a cell field:
 * the exact form's unlit march); empty-space skipping is off for such a volume. */
beams_status beams_set_volume_coordinates(beams_renderer* r, const float* x, const float* y, const float* z);

/* Replaces MapperLightedVolume::SetCompositeBackground (MapperLightedVolume.cxx:321-324)
 * and the Canvas::BlendBackground call it enables (:185-188): after the image is
 * complete (composite included), the premultiplied image is placed over the
 * background colour (Porter-Duff over: a = bg.a (1 - C.a), C.rgb += bg.rgb a,
 * C.a += a; pixels with C.a >= 1 unchanged), on the device. Off by default. */
beams_status beams_set_background(beams_renderer* r, int enable, const float rgba[4]);

/* Canvas depth clipping. Replaces the canvas depth buffer that
 * RayOperations::MapCanvasToRays turns into each camera ray's MaxDistance before
 * the slab test narrows it (MapperLightedVolume.cxx:151-152,
 * LightedVolumeRenderer.cxx:644-718). depth holds width x height floats in the
 * image's pixel order (row y at y * width, row 0 at the bottom):
 *   BEAMS_DEPTH_RAY_DISTANCE  the limit itself, a distance along the normalised
 *                             ray from the camera (NaN or +inf: no limit);
 *   BEAMS_DEPTH_WINDOW        OpenGL window depth in [0, 1] under the camera's
 *                             perspective with near_plane / far_plane, unprojected
 *                             at the pixel centre (1 = far plane; NaN reads as 1).
 * Every render whose camera has this width and height is clipped (others fail
 * with BEAMS_ERR_INVALID_ARG) until the buffer is cleared with depth = NULL.
 * The buffer is copied; on_device says where depth lives. */
#define BEAMS_DEPTH_RAY_DISTANCE 0
#define BEAMS_DEPTH_WINDOW 1
beams_status beams_set_depth_buffer(beams_renderer* r, const float* depth, int width, int height, int kind,
                                    double near_plane, double far_plane, int on_device);
/* The per-pixel ray limits the current depth buffer gives for camera cam
 * (width x height floats). Synchronises. */
beams_status beams_get_ray_limits(beams_renderer* r, const beams_camera* cam, float* dst, int dst_on_device);
/* The multi-light extension (the reference's notes.txt:4 "use multiple lights";
 * its renderer uses Locations[0] only, TransmittanceMap.h:591-592, which stays the
 * default): with enable != 0 and more than one light, the exact form builds one
 * map per light and the view march shades by sum_l (1 - opacity_l) * color_l *
 * intensity_l (light order) in place of the single term. Up to 8 lights; exact
 * form, single point volume. beams_get_shadow_map returns the maps one after the
 * other. */
beams_status beams_set_multi_light(beams_renderer* r, int enable);
/* Launch tuning (no reference counterpart; results do not depend on it).
 * light_brick: the order in which the map build takes its vertices: 0 = rows
 * (x fastest), or cubic bricks of 8 (default), 16, 32 or 64 vertices per edge.
 * no_empty_skip: 1 turns off the map build's skipping of 8^3-cell macro-cells
 * whose values all map to colour-map alpha 0 (such samples change nothing).
 * no_view_skip: the same for the view march (skipped samples still count as lit). */
typedef struct beams_tuning {
  int light_brick;
  int no_empty_skip;
  int no_view_skip;
  int reserved;
} beams_tuning;
beams_status beams_set_tuning(beams_renderer* r, const beams_tuning* t);
beams_status beams_get_tuning(beams_renderer* r, beams_tuning* t);
/* Times the map build under every vertex order x empty-skip choice on the
 * current volume, colour map, light and form and, given a camera, the view
 * march with and without its skip; keeps the fastest (results are identical
 * under all of them) and reports it. Synchronises. */
beams_status beams_autotune(beams_renderer* r, const beams_camera* cam, beams_tuning* best, float* best_map_ms,
                            float* best_view_ms);
/* Selects the render form (beams_form). opts: NULL, or for BEAMS_FORM_MLP a
 * const beams_mlp_options*. */
beams_status beams_set_form(beams_renderer* r, int form, const void* opts);

/* ---- multi-block scenes (sort-last on one GPU) ------------------------------- */
/* Replaces the reference's one-block-per-rank decomposition: SetData of each
 * rank's block plus the BoundsMap of all blocks (BoundsMap.cxx:93-127). After this
 * call beams_render runs the reference's five phases on the device: Phase 1 local
 * maps, Phases 2-3 cross-block shadow stitching (LightedVolumeRenderer.cxx:968-1256,
 * TransmittanceMap.h:342-513: each other block's map opacity at the light
 * segment's exit point, over-composited in exit order, then the local march
 * re-run from that prefix), Phase 4 a view march per block clipped to its
 * bounds, and Phase 5 the depth-ordered over composite of the block images
 * (MapperLightedVolume.cxx:215-303). Blocks are float32 point fields; neighbours
 * share their face plane. Up to 32 blocks. beams_set_volume leaves this mode. */
beams_status beams_set_bricks(beams_renderer* r, const beams_volume* bricks, int nbricks);
/* Copies brick `brick`'s map after the last render: stage 0 = Phase 1 (local),
 * stage 1 = stitched. When no two bricks overlap, Phase 1 builds only the
 * vertices within one layer of a brick face (the only ones the stitch reads);
 * the other stage-0 entries are then unspecified. For tests and tools. */
beams_status beams_get_brick_map(beams_renderer* r, int brick, int stage, float* dst, size_t count,
                                 int dst_on_device);

/* ---- batched form (serving) ---------------------------------------------------- */
/* No reference counterpart: the reference renders one camera per RenderCells call
 * (MapperLightedVolume.cxx:114-193). Here volumes stay resident and a batch of
 * requests, each with its own volume, camera, light, map size and sample
 * distance, runs as ONE persistent kernel launch (map builds first, view tiles
 * after, a view tile waiting with a bounded wait for its request's map), or
 * split into a map-build launch and a view launch (beams_batch_options.split),
 * captured once into a CUDA graph and replayed while the batch's shapes stay
 * the same. The colour map is the renderer's. Results equal beams_render's
 * exact form for the same settings. */
beams_status beams_batch_set_volumes(beams_renderer* r, const beams_volume* vols, int n);  /* float32 points */
typedef struct beams_request {
  int volume;               /* index into the beams_batch_set_volumes list */
  beams_camera camera;
  int light_kind;           /* 0 point (light = position), 1 directional (light = travel direction) */
  double light[3];
  float light_color[3];
  float light_intensity;
  int map_cells;            /* M: the map has (M+1)^3 vertices */
  float sample_distance;    /* <= 0: |extent| / 200 */
  float termination_alpha;  /* (0, 1]; 1 is the reference's */
  float* rgba_out;          /* width * height RGBA */
  int out_on_device;
} beams_request;
typedef struct beams_batch_options {
  int tile_w, tile_h;       /* view work item in pixels (default 32 x 32): tile_w a multiple of 8, tile_h of 4,
                               at most 16384 pixels; warps take its 8 x 4 sub-tiles */
  int light_brick;          /* map-build vertex order: 0 rows, 8/16/32/64 bricks */
  int use_graph;            /* 1: capture once, replay (default) */
  int no_skip;              /* 1: no empty-space skipping (default 0: both marches skip empty macro-cells) */
  int split;                /* 1: two launches, every request's map build and then every view march, each
                               kernel at its own occupancy; 0: one launch whose view tiles wait for their map
                               (default) */
  int reserved;             /* 0; 0x7e57 makes the map items withhold their completion (tests of the bounded
                               wait of the one-launch plan: the call then returns BEAMS_ERR_TIMEOUT after
                               about 2 s) */
} beams_batch_options;
beams_status beams_set_batch_options(beams_renderer* r, const beams_batch_options* o);
/* Timings: total_ms = the batch (launch to last image copied), view_march_ms = the
 * persistent kernel(s) and their staging copies, lit_samples and rays_hit summed,
 * kernel_launches 1 or 2 (split). */
beams_status beams_render_batch(beams_renderer* r, const beams_request* reqs, int n, beams_timings* t);
/* Tunes the batch options on these requests: for each launch plan (one launch,
 * or map builds then view marches) a coordinate descent over the empty-space
 * skip, the vertex order {rows, 8, 16, 32, 64 bricks} and the view tile {8x8,
 * 16x16, 32x8, 8x32, 32x32, 64x32, 64x64}, repeated until a round changes
 * nothing (three rounds at most); keeps the fastest (images are identical under
 * all of them) and reports it. */
beams_status beams_batch_autotune(beams_renderer* r, const beams_request* reqs, int n, beams_batch_options* best,
                                  float* best_ms);
/* The autotuner's results cache: beams_batch_autotune keeps its result per batch
 * shape (each request's volume dimensions, map size and image size; cameras and
 * lights may differ) and returns it without timing when the same shape comes
 * again. A serving process saves the cache to a text file and loads it at
 * start-up (after beams_batch_set_volumes) to skip the tuning runs. */
beams_status beams_batch_tuning_save(beams_renderer* r, const char* path);
beams_status beams_batch_tuning_load(beams_renderer* r, const char* path);
beams_status beams_batch_tuning_clear(beams_renderer* r);

/* ---- profiling ---------------------------------------------------------------- */
/* Replaces MapperLightedVolume::SetProfiler (MapperLightedVolume.h:57,
 * MapperLightedVolume.cxx:305-309), whose beams::Profiler (beams/Profiler.h)
 * records named, nested frames ("Phase 1" and its sub-frames,
 * LightedVolumeRenderer.cxx:914-966). With a profiler set, every beams_render
 * reports its frames after it completes (the call then synchronises the stream,
 * as with timings): ("Render", depth 0, total) and at depth 1 "Phase 1" (layouts
 * and map build; "Phases 1-3" for bricks: local maps and stitch), "Phase 4"
 * (view march) and "Phase 5" (composite and copy-out), each its CUDA-event time
 * in ms on the renderer's stream. fn = NULL removes the profiler. */
typedef void (*beams_profile_fn)(void* user, const char* frame, int depth, double ms);
beams_status beams_set_profiler(beams_renderer* r, beams_profile_fn fn, void* user);

/* ---- learned form ------------------------------------------------------------ */
/* No reference counterpart: a transmittance network (encoded position and light
 * direction -> 4 x 64 ReLU -> sigmoid) that replaces the map build and lookup
 * in BEAMS_FORM_MLP. Trained on the device on samples of the exact light march. */
typedef struct beams_mlp_options {
  int samples_log2;      /* training samples 2^k (default 24) */
  int n_lights;          /* light directions on a Fibonacci sphere (default 32) */
  int epochs;            /* default 4 */
  int batch;             /* rows per step (default 16384) */
  float lr;              /* Adam learning rate, cosine-decayed (default 2e-3) */
  unsigned seed;
  float fallback_tol;    /* render: |MLP - exact| on the probe set that sends a tile to the exact map (0.01) */
  float probe_fraction;  /* render: fraction of pixels probed (0.01) */
  int knot;              /* render: MLP evaluated every `knot` lit samples (1..64), linear in between (1 = every sample) */
  int scene_light;       /* train: 1 = the renderer's current light is training light 0 (a directional light
                            stands in as a point at 1e4 x the diagonal); the rest on the Fibonacci sphere */
  float focus;           /* train: fraction of positions drawn where the colour map's alpha is non-zero
                            (rejection sampling, 16 tries); the rest uniform in the volume. 0 = all uniform */
} beams_mlp_options;

typedef struct beams_mlp_report {
  float datagen_ms;
  float train_ms;
  float holdout_rmse;   /* trained network on held-out samples */
  float initial_rmse;   /* the initial network on the same samples */
  float unlit_rmse;     /* the method without a shadow model: T = 1 */
  float mean_rmse;      /* the best constant T */
  int steps;
  int samples;
} beams_mlp_report;

/* Trains the network on the current volume and colour map. */
beams_status beams_mlp_train(beams_renderer* r, const beams_mlp_options* opts, beams_mlp_report* report);
int beams_mlp_param_count(void);
beams_status beams_mlp_get_params(beams_renderer* r, float* dst, int n);
beams_status beams_mlp_set_params(beams_renderer* r, const float* src, int n);
/* The training kernels' loss (mean squared error) and gradient for features
 * (n x 112 floats, rounded to bfloat16) and targets; T gets the predictions. */
beams_status beams_mlp_loss_grad(beams_renderer* r, const float* features, const float* target, int n,
                                 float* loss, float* grad, float* T);
/* Per-probe max |dRGBA| between the network's pixel and the pixel composited
 * with the exact light march's transmittance, for the last BEAMS_FORM_MLP frame
 * (row-major over the probe grid: probe (i, j) is pixel (i*P + P/2, j*P + P/2),
 * P = round(1/sqrt(probe_fraction))); +inf marks a probe past the sample cap.
 * n must be the probe count; for tests and tools. */
beams_status beams_mlp_probe_errors(beams_renderer* r, float* dst, int n);
/* The network's forward pass on the tcgen05 tensor cores for n rows of
 * features (n x 112 floats, rounded to bfloat16): T receives the predictions.
 * For tests and tools (the training loop and the dense render path call the
 * same kernel directly). */
beams_status beams_mlp_forward_tc(beams_renderer* r, const float* features, int n, float* T);
/* The same on device memory: features_bf16 = n x 112 bfloat16 rows, T = n floats;
 * asynchronous on the renderer's stream, allocates nothing once a network exists. */
beams_status beams_mlp_forward_tc_device(beams_renderer* r, const void* features_bf16, int n, float* T);
/* 1 (default): training and beams_mlp_loss_grad run the hidden layers on the
 * tcgen05 tensor cores; 0: on the CUDA cores (the reference path for tests). */
beams_status beams_mlp_set_tensor_cores(beams_renderer* r, int enable);
/* Order of a BEAMS_FORM_MLP frame. 0: the network shades every pixel (recording
 * the probe pixels), the probe check follows, and the failing tiles are
 * rendered again from the exact map. 1: the network shades the probe pixels
 * first, the check runs, and the network then shades only the tiles that
 * passed. The images are the same; 1 is faster when many tiles fail. -1
 * (default): 1 when more than 1/8 of the tiles failed in the last learned frame
 * whose count has reached the host (read without waiting), else 0. */
beams_status beams_mlp_set_probe_first(beams_renderer* r, int mode);
/* The network's input encoding of n world positions under n light features. */
beams_status beams_mlp_encode(beams_renderer* r, const float* pos, const float* lfeat, int n, float* out);
/* Versioned checkpoint of parameters and Adam moments (FNV-1a checksummed). */
beams_status beams_mlp_save(beams_renderer* r, const char* path);
beams_status beams_mlp_load(beams_renderer* r, const char* path);

/* ---- render --------------------------------------------------------------- */
/* Replaces MapperLightedVolume::RenderCells (MapperLightedVolume.cxx:114-193):
 * map build (Phase 1/3) + view march (Phase 4) + copy-out (Phase 5).
 * rgba_out holds width*height*4 floats, premultiplied RGBA. out_on_device:
 *   BEAMS_OUT_HOST        host memory; the call returns once the image is there;
 *   BEAMS_OUT_DEVICE      device memory; the call returns once the work is queued;
 *   BEAMS_OUT_HOST_ASYNC  pinned host memory; the copy is queued on the renderer's
 *                         stream and the call returns at once: read the image
 *                         after beams_synchronize (lets a caller upload the next
 *                         volume while this frame renders).
 * t may be NULL; a non-NULL t synchronises. */
#define BEAMS_OUT_HOST 0
#define BEAMS_OUT_DEVICE 1
#define BEAMS_OUT_HOST_ASYNC 2
beams_status beams_render(beams_renderer* r, const beams_camera* cam, float* rgba_out,
                          int out_on_device, beams_timings* t);
/* Waits for everything queued on the renderer's stream; reports an asynchronous
 * CUDA error of that work. */
beams_status beams_synchronize(beams_renderer* r);

/* Map access for tests and tools: copies the current (M+1)^3 float32 map
 * (x fastest) to dst (host or device). Returns BEAMS_ERR_STATE before a build. */
beams_status beams_get_shadow_map(beams_renderer* r, float* dst, size_t count, int dst_on_device);
/* Builds the map only (Phase 1), without a view march. */
beams_status beams_build_shadow_map(beams_renderer* r, beams_timings* t);

/* ---- render without device allocation ---------------------------------------- */
/* No counterpart in the reference: an addition for callers that may not
 * allocate device memory themselves (a plugin or custom call inside another
 * framework that owns all GPU memory through its own allocator, or a frame loop
 * that must not stall on cudaMalloc/cudaFree, which can synchronise the device).
 * Renders one frame like beams_create + set_* + beams_render with a point light,
 * the reference's 128 light steps and the FP64 slab, into rgba_out_device
 * (width*height*4 floats, 16-byte aligned), asynchronously on cuda_stream.
 * Inputs stay the caller's: vol must be a float32 point field with on_device = 1,
 * tf_rgba_device holds tf_n (<= 1024) RGBA entries on the device, 16-byte aligned.
 * It calls no cudaMalloc or cudaFree: its only scratch, the frame's
 * (map_cells+1)^3 transmittance map, lives in one static device array sized for
 * map_cells <= BEAMS_NOALLOC_MAX_MAP_CELLS (129^3 floats, 8.6 MB), which every
 * device that loads the library holds until exit; larger map_cells is rejected
 * with BEAMS_ERR_INVALID_ARG. Every call looks up that array's device address
 * in the current context (cudaGetSymbolAddress). With lazy module loading
 * (CUDA_MODULE_LOADING=LAZY, the CUDA default) the first call on a device is
 * what loads the module, and so where the 8.6 MB and the kernels' code are
 * taken: make that first call (a warm-up frame) before the host framework claims
 * its memory, and outside any stream capture. The volume data must be 4-byte
 * aligned. The marches are beams_render's own, on the plain field with the cell
 * tables in shared memory (so the image equals beams_render's bit for bit); the
 * tables limit the axes: (nx + ny + nz - 3 + 3 map_cells + 1024) * 16 bytes must
 * stay within 200 KiB, else BEAMS_ERR_UNSUPPORTED. All calls share the one array: calls that
 * overlap on the GPU (other streams, other threads) race and corrupt each
 * other's maps; serialise them. Each call rewrites every map entry it reads, so
 * no clearing is needed between calls. Errors: beams_last_error(NULL). */
#define BEAMS_NOALLOC_MAX_MAP_CELLS 128
beams_status beams_render_noalloc(const beams_volume* vol, const float* tf_rgba_device, int tf_n,
                                  const double light_pos[3], const float light_color[3], float light_intensity,
                                  int map_cells, float sample_distance, float termination_alpha,
                                  const beams_camera* cam, float* rgba_out_device, void* cuda_stream);

/* ---- diagnostics ------------------------------------------------------------ */
/* Fault injection for tests (no reference counterpart): the nth following device
 * buffer allocation of any renderer fails with BEAMS_ERR_OOM (0 disarms). */
beams_status beams_test_fail_allocation(int nth);
/* Checks, on the device, the kernels' correctly rounded division (Markstein's
 * correction on a tabulated reciprocal) against IEEE division for every cell
 * width of the counting coordinates origin + i*spacing (ncells cells) and
 * `samples` numerators per width. No reference counterpart (test support). */
beams_status beams_selftest_division(float origin, float spacing, int ncells, int samples,
                                     unsigned long long* checked, unsigned long long* mismatches);

/* ---- scene generation (synthetic inputs; device-side) ----------------------- */
/* Fills a float32 field (x fastest, n[0]*n[1]*n[2] values) on the device with a sum
 * of Gaussian blobs: params = nblobs x {cx, cy, cz, sigma, amplitude} in domain
 * units [0,1]^3; the result is normalised to [0,1] when normalise != 0. */
beams_status beams_generate_blobs(float* dev_out, const int n[3], const float* params, int nblobs,
                                  int normalise, void* cuda_stream);
/* Gradient (Perlin-style) noise, octaves summed with lacunarity and gain, then
 * remapped to [0,1]. perm: 256 bytes (a permutation of 0..255). */
beams_status beams_generate_noise(float* dev_out, const int n[3], const unsigned char* perm,
                                  int octaves, float base_freq, float lacunarity, float gain,
                                  void* cuda_stream);

/* Sphere / ellipsoid field of the reference's sources::Spheres
 * (beams/sources/Spheres.cxx:19-96, :172-199): at each point of the grid
 * origin + spacing * i (float32, the rectilinear coordinates it builds), the
 * mean over the ellipsoids containing the point of lerp(min, max, d), d the
 * ellipsoid distance sqrt(sum((c - p)^2 / r^2)) <= 1, else default_value; with
 * a floor (floor_height >= 0 is not required: has_floor != 0) points below
 * origin.y + floor_height take floor_value. ellipsoids: n x {cx, cy, cz, rx, ry,
 * rz, min, max}. */
beams_status beams_generate_spheres(float* dev_out, const int n[3], const double origin[3],
                                    const double spacing[3], const float* ellipsoids, int n_ellipsoids,
                                    float default_value, int has_floor, float floor_height, float floor_value,
                                    void* cuda_stream);

/* ---- configuration (stage TOML) -------------------------------------------- */
/* The reference reads `<base-dir>/stage.toml` (pilot/staging/Stage.cxx:25-49):
 * [dataset_providers.<name>] with `type` and `cell_dims` (an integer or
 * [x, y, z], SubdividedSpheresDescriptor.cxx:22-44); its render knobs lived in
 * the (now commented) JSON presets of beams/Config.cxx:140-247. This reader
 * takes that file plus tables named after those preset keys:
 *   [render]            width, height, sample_distance, termination_alpha,
 *                       form = "exact" | "precision" | "mlp", field_dtype = "bf16" | "f16",
 *                       composite_background, background = [r, g, b, a]
 *   [shadow_map]        enabled, size = N | [x, y, z] | size_ratio = f, num_steps
 *   [camera]            azimuth, elevation, fov_y (an orbit around the bounds), or
 *                       position / look_at / up
 *   [[light]]           type = "point" | "directional", position, color, intensity
 *   [transfer_function] preset = "cool to warm" | "ramp", points, alphas, range, size
 *   [form]              knot, probe_fraction, fallback_tol, samples_log2, lights
 * Providers: "subdivided_spheres" (the reference's scene: one sphere of radius
 * 0.45 at the centre, value 1, default 0.1, SubdividedSpheresScene.cxx),
 * "spheres" (that scene's centre sphere, radius 0.1, and floor), "blobs" and
 * "noise" (seeded, `seed`). Parsed by a TOML-subset reader (tables, arrays of
 * tables, strings, numbers, booleans, arrays; comments); unknown keys are
 * errors. No reference counterpart for the reader itself (the reference uses
 * toml++, which is absent here). */
#define BEAMS_MAX_CONFIG_LIGHTS 8
#define BEAMS_MAX_TF_POINTS 64
typedef struct beams_config_light {
  int kind;                 /* 0 point, 1 directional */
  double position[3];       /* point: position; directional: travel direction */
  float color[3];
  float intensity;
} beams_config_light;

typedef struct beams_scene_desc {
  char provider_name[64];
  char provider_type[32];
  int cell_dims[3];         /* the field has cell_dims + 1 points per axis on [0,1]^3 */
  unsigned seed;
  int octaves;
  float base_freq;
  int width, height;
  float sample_distance;
  float termination_alpha;
  int form;
  int field_dtype;
  int composite_background;
  float background[4];
  int shadow_enabled;
  int shadow_size[3];       /* 0: from shadow_size_ratio x cell_dims (OpacityMapOptions::CalculateSize) */
  float shadow_size_ratio;
  float light_steps;        /* num_steps */
  int camera_explicit;
  float azimuth, elevation, fov_y_deg;
  double position[3], look_at[3], up[3];
  int n_lights;
  beams_config_light lights[BEAMS_MAX_CONFIG_LIGHTS];
  char tf_preset[32];
  int tf_points;
  double tf_x[BEAMS_MAX_TF_POINTS];
  float tf_alpha[BEAMS_MAX_TF_POINTS];
  float tf_range[2];
  int tf_size;
  int mlp_knot;
  float mlp_probe_fraction, mlp_fallback_tol;
  int mlp_samples_log2, mlp_lights;
  char file_name[256];      /* provider type "vtk_file": the legacy VTK volume (relative paths
                               are taken from the stage file's directory by beams_load_config_toml) */
} beams_scene_desc;

/* Parses TOML text / a TOML file into *out (defaults for absent keys). On a
 * syntax or schema error returns BEAMS_ERR_CONFIG and writes "line N: ..." to err. */
beams_status beams_parse_config_toml(const char* text, beams_scene_desc* out, char* err, int errlen);
beams_status beams_load_config_toml(const char* path, beams_scene_desc* out, char* err, int errlen);
/* Scene::Ready + SceneFactory for a parsed description: generates the dataset
 * on the device (owned by the renderer), sets the colour map (preset RGB,
 * piecewise-linear alpha through the points over `range`), map size, light steps,
 * the first light (the reference uses Locations[0] only), sample distance,
 * termination alpha, background and form (the learned form trains here when no
 * network is loaded), and returns the camera. */
beams_status beams_apply_scene(beams_renderer* r, const beams_scene_desc* d, beams_camera* camera_out);
/* The colour table beams_apply_scene sets (d->tf_size RGBA entries into rgba; n = tf_size). */
beams_status beams_scene_color_table(const beams_scene_desc* d, float* rgba, int n);
/* The light orbit of the reference's Beams::Run (Beams.cxx:239-288): frame k
 * puts a point light at (0.5, 0.5, 0.5) + 0.5 (cos k*5deg, sin k*5deg, 0),
 * keeping the first configured light's colour and intensity. */
beams_status beams_orbit_light(beams_renderer* r, const beams_scene_desc* d, int frame);

#ifdef __cplusplus
}
#endif
#endif /* BEAMS_B200_H */
