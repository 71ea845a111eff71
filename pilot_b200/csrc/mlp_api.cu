// mlp_api.cu — C ABI of the learned form: training, parameter access, the
// gradient entry the tests check against the float64 oracle, checkpoints.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/beams_b200.h"
#include "kernels.h"
#include "mlp_common.cuh"
#include "mlp_host.h"
#include "renderer.h"

namespace beams {
using namespace mlp;

beams_status make_geo(beams_renderer* r, const beams_camera* cam, ExactGeo& g);
beams_status ensure_buffer(beams_renderer* r, void** buf, size_t* cap, size_t bytes, const char* what);
beams_status prepare_layouts(beams_renderer* r, const ExactGeo& g, int& launches);
beams_status check_ready(beams_renderer* r);

// Device state of the learned form (owned by the renderer).
struct MlpState {
  float* P = nullptr;  // float32 masters
  float* G = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  int step = 0;
  bool ready = false;
  TrainWS ws{};
  int ws_rows = 0;
  void* ws_mem = nullptr;
  float4* lights = nullptr;  // training light positions (xyz)
  float4* lfeat = nullptr;   // their direction features
  int nlights = 0;
  void* packed = nullptr;    // inference weights: B fragments + biases
  void* probe_mem = nullptr; // probe records, counts, tile flags, fallback list
  size_t probe_bytes = 0;
  float* probe_err = nullptr;  // per-probe max |dRGBA| of the last frame (tests)
  int probe_err_n = 0;
  unsigned char* vmask = nullptr;  // lazy fallback: map cells the failing tiles read
  size_t vmask_bytes = 0;
  beams_mlp_options render_opts{};
  bool use_tc = true;            // training forward on the tcgen05 tensor cores
  unsigned* err_slot = nullptr;  // their timeout flag in the workspace
  // Frame order: -1 chosen from the last frame's fallback fraction, 0 network
  // march first, 1 probe pixels first (the images are the same).
  int probe_first = -1;
  // Host-mapped, written by the fallback's first kernel: the failing-tile count
  // of the last learned frame that has got that far, and that frame's tile count.
  volatile unsigned* h_fallback = nullptr;
  int fb_tiles = 0;
  ~MlpState() {
    for (void* p : {(void*)P, (void*)G, (void*)m, (void*)v, ws_mem, (void*)lights, (void*)lfeat, packed, probe_mem,
                    (void*)probe_err, (void*)vmask})
      if (p) cudaFree(p);
    if (h_fallback) cudaFreeHost((void*)h_fallback);
  }
};

MlpState* mlp_state(beams_renderer* r) {
  if (!r->mlp) r->mlp = new MlpState();
  return r->mlp;
}
void mlp_release(beams_renderer* r) {
  delete r->mlp;
  r->mlp = nullptr;
}

Encoding mlp_encoding(const ExactGeo& g) {
  Encoding e;
  for (int d = 0; d < 3; ++d) {
    e.bmin[d] = g.minp[d];
    e.inv_ext[d] = 1.f / (g.maxp[d] - g.minp[d]);
  }
  return e;
}

// The light feature of the renderer's first light: unit vector from the
// volume centre towards the light (point) or against the travel direction.
void mlp_light_feature(const beams_renderer* r, const ExactGeo& g, float out[3]) {
  double v[3] = {0, 0, 1};
  if (!r->lights.empty()) {
    const Light& L = r->lights[0];
    for (int d = 0; d < 3; ++d)
      v[d] = (L.kind == 0) ? L.v[d] - 0.5 * ((double)g.minp[d] + (double)g.maxp[d]) : -L.v[d];
  }
  const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int d = 0; d < 3; ++d) out[d] = (float)(n > 0 ? v[d] / n : 0.0);
}

static beams_status alloc_params(beams_renderer* r, MlpState* s) {
  if (s->P) return BEAMS_OK;
  for (float** p : {&s->P, &s->G, &s->m, &s->v}) {
    cudaError_t e = cudaMalloc((void**)p, kParams * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(r, e, "allocating MLP parameters");
    cudaMemsetAsync(*p, 0, kParams * sizeof(float), r->stream);
  }
  return BEAMS_OK;
}

static beams_status ensure_ws(beams_renderer* r, MlpState* s, int rows) {
  if (s->ws_rows >= rows) return BEAMS_OK;
  if (s->ws_mem) cudaFree(s->ws_mem);
  s->ws_mem = nullptr;
  s->ws_rows = 0;
  const size_t nH = (size_t)rows * kHid;
  const size_t bytes = 4 * nH * sizeof(__nv_bfloat16) + (size_t)rows * kIn * 4 + nH * 4 + (size_t)rows * 8 + 256;
  cudaError_t e = cudaMalloc(&s->ws_mem, bytes);
  if (e != cudaSuccess) return cuda_fail(r, e, "allocating MLP workspace");
  char* p = (char*)s->ws_mem;
  for (int l = 0; l < 4; ++l) {
    s->ws.H[l] = (__nv_bfloat16*)p;
    p += nH * sizeof(__nv_bfloat16);
  }
  s->ws.dA = (float*)p;
  p += (size_t)rows * kIn * 4;
  s->ws.dB = (float*)p;
  p += nH * 4;
  s->ws.dz = (float*)p;
  p += (size_t)rows * 4;
  s->ws.T = (float*)p;
  p += (size_t)rows * 4;
  s->ws.loss = (float*)p;
  s->err_slot = (unsigned*)(p + 64);
  s->ws.err = s->use_tc ? s->err_slot : nullptr;  // the forward runs on the tcgen05 tensor cores
  e = cudaMemsetAsync(s->err_slot, 0, sizeof(unsigned), r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "clearing the MLP workspace");
  s->ws_rows = rows;
  return BEAMS_OK;
}

static void init_params(std::vector<float>& h, unsigned seed) {
  std::mt19937 rng(seed);
  h.assign(kParams, 0.f);
  auto fill = [&](int off, int fan_in, int count, float gain) {
    const float a = gain * std::sqrt(6.f / (float)fan_in);
    std::uniform_real_distribution<float> U(-a, a);
    for (int i = 0; i < count; ++i) h[off + i] = U(rng);
  };
  fill(oW1, kUsed, kIn * kHid, 1.f);
  for (int i = kUsed * kHid; i < kIn * kHid; ++i) h[oW1 + i] = 0.f;  // padding rows
  fill(oW2, kHid, kHid * kHid, 1.f);
  fill(oW3, kHid, kHid * kHid, 1.f);
  fill(oW4, kHid, kHid * kHid, 1.f);
  fill(oW5, kHid, kHid, 0.5f);
  h[oB5] = 2.f;  // sigmoid(2) = 0.88: most of the volume is lit
}

cudaError_t launch_view_march_mlp(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                  const uint2* W, const float* aux, const Encoding& enc, const float lf[3], int knot,
                                  float4* out, Counters* cnt, const MlpProbe& probe, const MlpPass& pass,
                                  cudaStream_t st);

bool mlp_ready(const beams_renderer* r) { return r->mlp && r->mlp->ready; }

beams_status mlp_set_render_options(beams_renderer* r, const beams_mlp_options* o) {
  MlpState* st = mlp_state(r);
  beams_mlp_options d;
  std::memset(&d, 0, sizeof(d));
  d.fallback_tol = 0.01f;
  d.probe_fraction = 0.01f;
  d.knot = 4;
  if (o) {
    if (o->knot < 1 || o->knot > 64) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp form: knot must be in [1, 64]");
    if (!(o->probe_fraction >= 0.f && o->probe_fraction <= 1.f) || !(o->fallback_tol >= 0.f))
      return fail(r, BEAMS_ERR_INVALID_ARG, "mlp form: bad probe fraction or tolerance");
    d.knot = o->knot;
    d.fallback_tol = o->fallback_tol;
    d.probe_fraction = o->probe_fraction;
  }
  st->render_opts = d;
  return BEAMS_OK;
}

struct ProbeBuffers {
  ProbeLayout L{};
  float4* rec = nullptr;
  int* count = nullptr;
  unsigned* flags = nullptr;
  unsigned* fcount = nullptr;
  unsigned* flist = nullptr;
};

// Lays out this frame's probe buffers (none when the probe fraction is 0).
static beams_status probe_buffers(beams_renderer* r, const ExactGeo& g, ProbeBuffers& pb) {
  MlpState* st = r->mlp;
  pb.L = probe_layout(g.width, g.height, st->render_opts.probe_fraction);
  const ProbeLayout& L = pb.L;
  if (L.stride == 0) return BEAMS_OK;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_rec = al((size_t)L.nprobe * L.cap * 2 * sizeof(float4));
  const size_t b_cnt = al((size_t)L.nprobe * sizeof(int) + 4);
  const size_t b_flags = al(((size_t)L.ntiles + 1) * sizeof(unsigned));
  const size_t b_list = al((size_t)L.ntiles * sizeof(unsigned) + 4);
  beams_status s = ensure_buffer(r, &st->probe_mem, &st->probe_bytes, b_rec + b_cnt + b_flags + b_list,
                                 "allocating the probe buffers");
  if (s != BEAMS_OK) return s;
  char* base = (char*)st->probe_mem;
  pb.rec = (float4*)base;
  pb.count = (int*)(base + b_rec);
  pb.flags = (unsigned*)(base + b_rec + b_cnt);
  pb.fcount = pb.flags + L.ntiles;
  pb.flist = (unsigned*)(base + b_rec + b_cnt + b_flags);
  if (st->probe_err_n < L.nprobe) {
    if (st->probe_err) cudaFree(st->probe_err);
    st->probe_err = nullptr;
    st->probe_err_n = 0;
    cudaError_t e = cudaMalloc((void**)&st->probe_err, (size_t)std::max(L.nprobe, 1) * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(r, e, "allocating probe errors");
    st->probe_err_n = std::max(L.nprobe, 1);
  }
  return BEAMS_OK;
}

// Probe pixels against the exact light march: the tiles that fail are flagged
// and listed. A network view march has already shaded the probe pixels and
// recorded their samples.
static beams_status mlp_probe_check(beams_renderer* r, const ExactGeo& g, const ProbeBuffers& pb, float4* out,
                                    int& launches) {
  MlpState* st = r->mlp;
  const ProbeLayout& L = pb.L;
  cudaError_t e = cudaMemsetAsync(pb.flags, 0, ((size_t)L.ntiles + 1) * sizeof(unsigned), r->stream);
  if (e == cudaSuccess)
    e = launch_mlp_probe(g, L, (const float4*)r->d_quads, r->d_tab, r->d_tf, out, st->render_opts.fallback_tol, pb.rec,
                         pb.count, pb.flags, pb.flist, pb.fcount, st->probe_err, r->d_cnt, r->stream, true);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp probe launch");
  ++launches;
  return BEAMS_OK;
}

// The exact map path over the listed tiles, built lazily: the map cells the
// listed tiles' view rays read are marked, K1 marches only their vertices (both gated on
// a non-empty list), K2 re-renders the listed tiles. Nothing here waits on the
// host; the first kernel writes the list's length to host-mapped memory for the
// next frame's choice of order.
static beams_status mlp_fallback(beams_renderer* r, const ExactGeo& g, const ProbeBuffers& pb, float4* out,
                                 int& launches) {
  MlpState* st = r->mlp;
  const ProbeLayout& L = pb.L;
  cudaError_t e;
  const size_t nvert = (size_t)g.pd[0] * g.pd[1] * g.pd[2];
  beams_status s = ensure_masked_map(r, &r->d_map, &r->map_cap, nvert * sizeof(float), r->stream, r->map_is_half);
  if (s != BEAMS_OK) return s;
  r->map_valid = false;  // a partial map, built (or not) on the device's decision
  r->map_is_half = false;
  const size_t ncell = (size_t)(g.pd[0] - 1) * (g.pd[1] - 1) * (g.pd[2] - 1);
  const size_t mask_bytes = (ncell + 15) & ~(size_t)15;
  s = ensure_buffer(r, (void**)&st->vmask, &st->vmask_bytes, mask_bytes, "allocating the fallback cell mask");
  if (s != BEAMS_OK) return s;
  if (!st->h_fallback) {
    unsigned* h = nullptr;
    e = cudaHostAlloc((void**)&h, sizeof(unsigned), cudaHostAllocMapped);
    if (e != cudaSuccess) return cuda_fail(r, e, "allocating the fallback count");
    *h = 0u;
    st->h_fallback = h;
  }
  s = ensure_buffer(r, (void**)&r->d_vlist, &r->vlist_cap, marked_list_bytes(g.pd),
                    "allocating the map vertex list");
  if (s != BEAMS_OK) return s;
  st->fb_tiles = L.ntiles;
  e = launch_mark_fallback_vertices(g, (const float4*)r->d_quads, r->d_tab, r->d_tf, pb.flist, pb.fcount, st->vmask,
                                    mask_bytes, (unsigned*)st->h_fallback, r->d_cnt, r->stream);
  if (e == cudaSuccess) e = launch_list_marked_vertices(g, st->vmask, pb.fcount, r->d_vlist, r->stream);
  if (e == cudaSuccess)
    e = launch_light_march_f32(g, (const float4*)r->d_quads, r->d_tab, r->d_tf, r->d_map, r->d_cnt, r->stream,
                               nullptr, 0, -1, pb.fcount, nullptr, r->d_vlist);
  if (e == cudaSuccess)
    e = launch_view_march_tiles(g, (const float4*)r->d_quads, r->d_tab, r->d_tf, r->d_map, out, r->d_cnt + 1,
                                pb.flist, pb.fcount, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp fallback launch");
  launches += 6;  // mask clear, marks, block pass, list, light march, view march
  return BEAMS_OK;
}

// Probe pixels first pays when many tiles fall back: the network then shades
// only the tiles that passed. Chosen from the last learned frame whose count
// has reached the host (read without waiting); the first frame marches the
// network first.
constexpr float kProbeFirstFraction = 0.125f;

static bool choose_probe_first(const MlpState* st) {
  if (st->probe_first >= 0) return st->probe_first == 1;
  if (!st->h_fallback || st->fb_tiles <= 0) return false;
  return (float)*st->h_fallback > kProbeFirstFraction * (float)st->fb_tiles;
}

// The view march shaded by the network (no map is built).
beams_status mlp_render_view(beams_renderer* r, const ExactGeo& g, float4* out, int& launches) {
  MlpState* st = r->mlp;
  if (!st || !st->ready) return fail(r, BEAMS_ERR_STATE, "mlp form: no trained or loaded network");
  if (!st->packed) {
    cudaError_t e = cudaMalloc(&st->packed, mlp_packed_bytes());
    if (e != cudaSuccess) return cuda_fail(r, e, "allocating packed MLP weights");
  }
  uint2* W = (uint2*)st->packed;
  float* aux = (float*)((char*)st->packed + (7 * 8 * 32 + 3 * 4 * 8 * 32) * sizeof(uint2));
  cudaError_t e = launch_pack_weights(st->P, W, aux, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "packing MLP weights");
  ++launches;
  float lf[3];
  mlp_light_feature(r, g, lf);
  ProbeBuffers pb;
  beams_status s = probe_buffers(r, g, pb);
  if (s != BEAMS_OK) return s;
  const MlpProbe none{0, 0, 0, 0, 0, nullptr, nullptr};
  MlpProbe probe = none;
  if (pb.L.stride > 0 && pb.L.nprobe > 0)
    probe = MlpProbe{pb.L.stride, pb.L.offset, pb.L.nqx, pb.L.nqy, pb.L.cap, pb.rec, pb.count};
  const Encoding enc = mlp_encoding(g);
  const int knot = st->render_opts.knot;
  const float4* quads = (const float4*)r->d_quads;
  if (probe.P > 0 && choose_probe_first(st)) {
    // probe pixels, their check, then the network over the tiles that passed
    e = launch_view_march_mlp(g, quads, r->d_tab, r->d_tf, W, aux, enc, lf, knot, out, r->d_cnt, probe,
                              MlpPass{nullptr, 0, 1}, r->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(&r->d_cnt->tiles_view, 0, sizeof(unsigned), r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "mlp probe march launch");
    ++launches;
    s = mlp_probe_check(r, g, pb, out, launches);
    if (s != BEAMS_OK) return s;
    // the network over the tiles that passed (a side stream beside the exact
    // path over the failing tiles measured no faster)
    const int ftx = (g.width + kFallbackTile - 1) / kFallbackTile;
    e = launch_view_march_mlp(g, quads, r->d_tab, r->d_tf, W, aux, enc, lf, knot, out, r->d_cnt, none,
                              MlpPass{pb.flags, ftx, 0}, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "mlp view march launch");
    ++launches;
    return mlp_fallback(r, g, pb, out, launches);
  }
  e = launch_view_march_mlp(g, quads, r->d_tab, r->d_tf, W, aux, enc, lf, knot, out, r->d_cnt, probe,
                            MlpPass{nullptr, 0, 0}, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp view march launch");
  ++launches;
  if (pb.L.stride == 0) return BEAMS_OK;  // probe fraction 0: the network's image stands
  s = mlp_probe_check(r, g, pb, out, launches);
  if (s != BEAMS_OK) return s;
  return mlp_fallback(r, g, pb, out, launches);
}

}  // namespace beams

using namespace beams;

extern "C" {

beams_status beams_mlp_forward_tc_device(beams_renderer* r, const void* features_bf16, int n, float* T) {
  if (!r || !features_bf16 || !T || n < 1) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_forward_tc_device: bad arguments");
  MlpState* st = r->mlp;
  if (!st || !st->P) return fail(r, BEAMS_ERR_STATE, "mlp_forward_tc_device: no network");
  if (!st->err_slot) {
    beams_status s = ensure_ws(r, st, 256);
    if (s != BEAMS_OK) return s;
  }
  cudaSetDevice(r->device);
  cudaError_t e = mlp_forward_tc_features((const __nv_bfloat16*)features_bf16, n, st->P, T, st->err_slot,
                                          r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_forward_tc_device");
  return BEAMS_OK;
}

beams_status beams_mlp_set_tensor_cores(beams_renderer* r, int enable) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  MlpState* st = mlp_state(r);
  st->use_tc = enable != 0;
  st->ws.err = (st->use_tc && st->err_slot) ? st->err_slot : nullptr;
  return BEAMS_OK;
}

beams_status beams_mlp_set_probe_first(beams_renderer* r, int mode) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (mode < -1 || mode > 1) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_set_probe_first: mode must be -1, 0 or 1");
  mlp_state(r)->probe_first = mode;
  return BEAMS_OK;
}

beams_status beams_mlp_forward_tc(beams_renderer* r, const float* features, int n, float* T) {
  if (!r || !features || !T || n < 1 || n > (1 << 24)) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_forward_tc: bad arguments");
  MlpState* st = r->mlp;
  if (!st || !st->P) return fail(r, BEAMS_ERR_STATE, "mlp_forward_tc: no network");
  cudaSetDevice(r->device);
  std::vector<__nv_bfloat16> hx((size_t)n * kIn);
  for (size_t i = 0; i < hx.size(); ++i) hx[i] = __float2bfloat16_rn(features[i]);
  __nv_bfloat16* dx = nullptr;
  float* dt = nullptr;
  unsigned* derr = nullptr;
  cudaError_t e = cudaMalloc((void**)&dx, hx.size() * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dt, (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&derr, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(unsigned), r->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dx, hx.data(), hx.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = mlp_forward_tc_features(dx, n, st->P, dt, derr, r->stream);
  unsigned herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(T, dt, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  cudaFree(dx);
  cudaFree(dt);
  cudaFree(derr);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_forward_tc");
  if (herr) return fail(r, BEAMS_ERR_TIMEOUT, "mlp_forward_tc: a tensor-core wait timed out");
  return BEAMS_OK;
}

beams_status beams_mlp_probe_errors(beams_renderer* r, float* dst, int n) {
  if (!r || !dst) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_probe_errors: NULL argument");
  MlpState* st = r->mlp;
  if (!st || !st->probe_err || n < 1 || n > st->probe_err_n)
    return fail(r, BEAMS_ERR_STATE, "mlp_probe_errors: no probed frame of that size");
  cudaSetDevice(r->device);
  cudaError_t e = cudaStreamSynchronize(r->stream);
  if (e == cudaSuccess) e = cudaMemcpy(dst, st->probe_err, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_probe_errors");
  return BEAMS_OK;
}

beams_status beams_mlp_train(beams_renderer* r, const beams_mlp_options* opt, beams_mlp_report* rep) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  beams_mlp_options o;
  std::memset(&o, 0, sizeof(o));
  o.samples_log2 = 24;
  o.n_lights = 32;
  o.epochs = 4;
  o.batch = 16384;
  o.lr = 2e-3f;
  o.seed = 1;
  o.focus = 0.875f;
  if (opt) o = *opt;
  if (o.samples_log2 < 10 || o.samples_log2 > 26 || o.n_lights < 1 || o.n_lights > kMaxLights || o.epochs < 1 ||
      o.batch < 256 || o.batch > (1 << 20) || !(o.lr > 0.f) || !(o.focus >= 0.f && o.focus <= 1.f))
    return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_train: options out of range");
  const int saved_form = r->form;
  r->form = BEAMS_FORM_EXACT;  // data come from the exact light march
  beams_status s = check_ready(r);
  if (s != BEAMS_OK) {
    r->form = saved_form;
    return s;
  }
  if (r->brick_mode || r->vol.assoc != BEAMS_ASSOC_POINTS || r->rect) {
    r->form = saved_form;
    return fail(r, BEAMS_ERR_UNSUPPORTED, "mlp_train: needs a single float32 point volume with uniform spacing");
  }
  cudaSetDevice(r->device);
  ExactGeo g;
  int launches = 0;
  s = make_geo(r, nullptr, g);
  if (s == BEAMS_OK) s = prepare_layouts(r, g, launches);
  r->form = saved_form;
  if (s != BEAMS_OK) return s;
  MlpState* st = mlp_state(r);
  s = alloc_params(r, st);
  if (s != BEAMS_OK) return s;

  // Training lights: Fibonacci sphere, point lights at 2x the diagonal from the centre.
  std::vector<float4> lp(o.n_lights), lf(o.n_lights);
  const double c[3] = {0.5 * ((double)g.minp[0] + g.maxp[0]), 0.5 * ((double)g.minp[1] + g.maxp[1]),
                       0.5 * ((double)g.minp[2] + g.maxp[2])};
  const double R = 2.0 * (double)g.extent_mag;
  const double ga = M_PI * (3.0 - std::sqrt(5.0));
  const int j0 = (o.scene_light && !r->lights.empty()) ? 1 : 0;
  const int nfib = o.n_lights - j0;
  for (int j = 0; j < nfib; ++j) {
    const double z = nfib > 0 ? 1.0 - (2.0 * j + 1.0) / nfib : 0.0;
    const double rr = std::sqrt(std::max(0.0, 1.0 - z * z));
    const double d[3] = {rr * std::cos(ga * j), rr * std::sin(ga * j), z};
    lp[j0 + j] = make_float4((float)(c[0] + R * d[0]), (float)(c[1] + R * d[1]), (float)(c[2] + R * d[2]), 0.f);
    lf[j0 + j] = make_float4((float)d[0], (float)d[1], (float)d[2], 0.f);
  }
  if (j0) {
    // the renderer's light: its own position (a directional light as a far point)
    const Light& L = r->lights[0];
    float f[3];
    mlp_light_feature(r, g, f);
    const double far = 1e4 * (double)g.extent_mag;
    for (int d = 0; d < 3; ++d) {
      const double p = (L.kind == 0) ? L.v[d] : c[d] + far * (double)f[d];
      (&lp[0].x)[d] = (float)p;
      (&lf[0].x)[d] = f[d];
    }
    lp[0].w = lf[0].w = 0.f;
  }
  cudaError_t e = cudaSuccess;
  if (!st->lights) e = cudaMalloc((void**)&st->lights, kMaxLights * sizeof(float4));
  if (e == cudaSuccess && !st->lfeat) e = cudaMalloc((void**)&st->lfeat, kMaxLights * sizeof(float4));
  if (e == cudaSuccess) e = cudaMemcpyAsync(st->lights, lp.data(), o.n_lights * sizeof(float4), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st->lfeat, lf.data(), o.n_lights * sizeof(float4), cudaMemcpyHostToDevice, r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_train: lights");
  st->nlights = o.n_lights;

  const int n = 1 << o.samples_log2;
  float4* d_samples = nullptr;
  float* d_target = nullptr;
  __nv_bfloat16* d_X = nullptr;
  cudaEvent_t t0, t1, t2;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventCreate(&t2);
  e = cudaMalloc((void**)&d_samples, (size_t)n * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_target, (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_X, (size_t)n * kIn * sizeof(__nv_bfloat16));
  if (e != cudaSuccess) {
    cudaFree(d_samples);
    cudaFree(d_target);
    cudaFree(d_X);
    return cuda_fail(r, e, "mlp_train: allocating the training set");
  }
  cudaEventRecord(t0, r->stream);
  e = mlp_gen_data(g, (const float4*)r->d_quads, r->d_tab, r->d_tf, st->lights, o.n_lights, o.seed, o.focus, d_samples,
                   d_target, n, r->stream);
  const Encoding enc = mlp_encoding(g);
  if (e == cudaSuccess) e = mlp_features(d_samples, st->lfeat, enc, d_X, n, r->stream);
  cudaEventRecord(t1, r->stream);

  std::vector<float> h;
  init_params(h, o.seed);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st->P, h.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, r->stream);
  for (float* p : {st->G, st->m, st->v})
    if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, kParams * sizeof(float), r->stream);
  st->step = 0;
  beams_status bs = ensure_ws(r, st, std::max(o.batch, std::min(n / 16, 65536)));
  if (bs != BEAMS_OK) {
    cudaFree(d_samples);
    cudaFree(d_target);
    cudaFree(d_X);
    return bs;
  }
  const int holdout = std::min(n / 16, 65536);
  const int ntrain = n - holdout;
  // Baselines on the held-out samples: the initial network, no shadow model
  // (T = 1) and the best constant.
  float init_loss = 0.f;
  std::vector<float> ht(holdout);
  if (e == cudaSuccess) e = cudaMemsetAsync(st->ws.loss, 0, sizeof(float), r->stream);
  if (e == cudaSuccess)
    e = mlp_fwd_bwd(st->P, nullptr, d_X + (size_t)ntrain * kIn, d_target + ntrain, holdout, st->ws, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&init_loss, st->ws.loss, sizeof(float), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ht.data(), d_target + ntrain, holdout * sizeof(float), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  double s1 = 0, s2 = 0, su = 0;
  for (float t : ht) {
    s1 += t;
    s2 += (double)t * t;
    su += (1.0 - t) * (1.0 - t);
  }
  const double mean_t = s1 / holdout;
  const int steps_per_epoch = std::max(1, ntrain / o.batch);
  const int total = steps_per_epoch * o.epochs;
  bool timed_out = false;
  for (int ep = 0; ep < o.epochs && e == cudaSuccess && !timed_out; ++ep) {
    const int rot = (int)(((unsigned)ep * 2654435761u) % (unsigned)std::max(1, ntrain - o.batch));
    for (int k = 0; k < steps_per_epoch && e == cudaSuccess && !timed_out; ++k) {
      int off = (rot + k * o.batch) % std::max(1, ntrain - o.batch + 1);
      const float prog = (float)st->step / (float)total;
      const float lr = o.lr * (0.05f + 0.95f * 0.5f * (1.f + std::cos((float)M_PI * prog)));
      e = mlp_fwd_bwd(st->P, st->G, d_X + (size_t)off * kIn, d_target + off, o.batch, st->ws, r->stream);
      if (e == cudaSuccess) e = mlp_adam(st->P, st->G, st->m, st->v, lr, ++st->step, r->stream);
      // a tensor-core wait that gave up ends the training early (checked every 256 steps)
      if (e == cudaSuccess && st->ws.err && (st->step & 255) == 0) {
        unsigned f = 0;
        e = cudaMemcpyAsync(&f, st->ws.err, sizeof(unsigned), cudaMemcpyDeviceToHost, r->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
        timed_out = f != 0;
      }
    }
  }
  cudaEventRecord(t2, r->stream);
  // held-out loss
  float hl = -1.f;
  if (e == cudaSuccess) e = cudaMemsetAsync(st->ws.loss, 0, sizeof(float), r->stream);
  if (e == cudaSuccess)
    e = mlp_fwd_bwd(st->P, nullptr, d_X + (size_t)ntrain * kIn, d_target + ntrain, holdout, st->ws, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hl, st->ws.loss, sizeof(float), cudaMemcpyDeviceToHost, r->stream);
  unsigned tc_err = 0;
  if (e == cudaSuccess && st->ws.err)
    e = cudaMemcpyAsync(&tc_err, st->ws.err, sizeof(unsigned), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e == cudaSuccess && tc_err) {
    cudaFree(d_samples);
    cudaFree(d_target);
    cudaFree(d_X);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaEventDestroy(t2);
    return fail(r, BEAMS_ERR_TIMEOUT, "mlp_train: a tensor-core wait timed out");
  }
  if (rep && e == cudaSuccess) {
    std::memset(rep, 0, sizeof(*rep));
    cudaEventElapsedTime(&rep->datagen_ms, t0, t1);
    cudaEventElapsedTime(&rep->train_ms, t1, t2);
    rep->holdout_rmse = std::sqrt(hl / (float)holdout);
    rep->initial_rmse = std::sqrt(init_loss / (float)holdout);
    rep->unlit_rmse = (float)std::sqrt(su / holdout);
    rep->mean_rmse = (float)std::sqrt(std::max(0.0, s2 / holdout - mean_t * mean_t));
    rep->steps = st->step;
    rep->samples = n;
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(t2);
  cudaFree(d_samples);
  cudaFree(d_target);
  cudaFree(d_X);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_train");
  st->ready = true;
  return BEAMS_OK;
}

beams_status beams_mlp_get_params(beams_renderer* r, float* dst, int n) {
  if (!r || !dst || n < kParams) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_get_params: need kParams floats");
  if (!r->mlp || !r->mlp->P) return fail(r, BEAMS_ERR_STATE, "no MLP parameters");
  cudaSetDevice(r->device);
  cudaError_t e = cudaMemcpyAsync(dst, r->mlp->P, kParams * sizeof(float), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_get_params");
  return BEAMS_OK;
}

beams_status beams_mlp_set_params(beams_renderer* r, const float* src, int n) {
  if (!r || !src || n != kParams) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_set_params: need kParams floats");
  cudaSetDevice(r->device);
  MlpState* st = mlp_state(r);
  beams_status s = alloc_params(r, st);
  if (s != BEAMS_OK) return s;
  cudaError_t e = cudaMemcpyAsync(st->P, src, kParams * sizeof(float), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_set_params");
  st->ready = true;
  return BEAMS_OK;
}

int beams_mlp_param_count(void) { return kParams; }

// Loss and gradients for given features (n x 112, float, rounded to bfloat16
// here) and targets, with the current parameters: the training kernels' own
// forward and backward. G is zeroed first; loss = mean (T - target)^2.
beams_status beams_mlp_loss_grad(beams_renderer* r, const float* features, const float* target, int n,
                                 float* loss, float* grad, float* T) {
  if (!r || !features || !target || n < 1 || n > (1 << 20))
    return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_loss_grad: bad arguments");
  if (!r->mlp || !r->mlp->P) return fail(r, BEAMS_ERR_STATE, "no MLP parameters");
  cudaSetDevice(r->device);
  MlpState* st = r->mlp;
  beams_status s = ensure_ws(r, st, n);
  if (s != BEAMS_OK) return s;
  std::vector<__nv_bfloat16> xb((size_t)n * kIn);
  for (size_t i = 0; i < xb.size(); ++i) xb[i] = __float2bfloat16_rn(features[i]);
  __nv_bfloat16* dX = nullptr;
  float* dt = nullptr;
  cudaError_t e = cudaMalloc((void**)&dX, xb.size() * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dt, (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dX, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dt, target, (size_t)n * 4, cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st->G, 0, kParams * sizeof(float), r->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st->ws.loss, 0, sizeof(float), r->stream);
  if (e == cudaSuccess) e = mlp_fwd_bwd(st->P, st->G, dX, dt, n, st->ws, r->stream);
  float l = 0.f;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&l, st->ws.loss, 4, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess && grad) e = cudaMemcpyAsync(grad, st->G, kParams * 4, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess && T) e = cudaMemcpyAsync(T, st->ws.T, (size_t)n * 4, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st->G, 0, kParams * sizeof(float), r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  cudaFree(dX);
  cudaFree(dt);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_loss_grad");
  if (loss) *loss = l / (float)n;
  return BEAMS_OK;
}

// Encoding of n positions (world, n x 3) under light features (n x 3) into
// n x 112 floats, for tests and tools.
beams_status beams_mlp_encode(beams_renderer* r, const float* pos, const float* lfeat, int n, float* out) {
  if (!r || !pos || !lfeat || !out || n < 1 || n > (1 << 20))
    return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_encode: bad arguments");
  beams_status s = check_ready(r);
  if (s != BEAMS_OK) return s;
  cudaSetDevice(r->device);
  ExactGeo g;
  s = make_geo(r, nullptr, g);
  if (s != BEAMS_OK) return s;
  std::vector<float4> smp(n), lf(n);
  for (int i = 0; i < n; ++i) {
    smp[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], (float)i);
    lf[i] = make_float4(lfeat[3 * i], lfeat[3 * i + 1], lfeat[3 * i + 2], 0.f);
  }
  float4 *ds = nullptr, *dl = nullptr;
  __nv_bfloat16* dX = nullptr;
  cudaError_t e = cudaMalloc((void**)&ds, n * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dl, n * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dX, (size_t)n * kIn * 2);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ds, smp.data(), n * sizeof(float4), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dl, lf.data(), n * sizeof(float4), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = mlp_features(ds, dl, mlp_encoding(g), dX, n, r->stream);
  std::vector<__nv_bfloat16> xb((size_t)n * kIn);
  if (e == cudaSuccess) e = cudaMemcpyAsync(xb.data(), dX, xb.size() * 2, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  cudaFree(ds);
  cudaFree(dl);
  cudaFree(dX);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_encode");
  for (size_t i = 0; i < xb.size(); ++i) out[i] = __bfloat162float(xb[i]);
  return BEAMS_OK;
}

// Checkpoint: little-endian blob "BMLP", version, parameter count, step, the
// float32 parameters and Adam moments, and a FNV-1a checksum of all before it.
static uint32_t fnv1a(const unsigned char* p, size_t n, uint32_t h = 2166136261u) {
  for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 16777619u;
  return h;
}

beams_status beams_mlp_save(beams_renderer* r, const char* path) {
  if (!r || !path) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_save: bad arguments");
  if (!r->mlp || !r->mlp->P) return fail(r, BEAMS_ERR_STATE, "no MLP parameters");
  cudaSetDevice(r->device);
  std::vector<float> buf(3 * (size_t)kParams);
  cudaError_t e = cudaMemcpyAsync(buf.data(), r->mlp->P, kParams * 4, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf.data() + kParams, r->mlp->m, kParams * 4, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(buf.data() + 2 * kParams, r->mlp->v, kParams * 4, cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_save");
  std::vector<unsigned char> blob(16 + buf.size() * 4);
  const uint32_t hdr[4] = {0x504c4d42u /* "BMLP" */, 1u, (uint32_t)kParams, (uint32_t)r->mlp->step};
  std::memcpy(blob.data(), hdr, 16);
  std::memcpy(blob.data() + 16, buf.data(), buf.size() * 4);
  const uint32_t sum = fnv1a(blob.data(), blob.size());
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_save: cannot open file");
  const bool ok = std::fwrite(blob.data(), 1, blob.size(), f) == blob.size() && std::fwrite(&sum, 4, 1, f) == 1;
  std::fclose(f);
  return ok ? BEAMS_OK : fail(r, BEAMS_ERR_INTERNAL, "mlp_save: write failed");
}

beams_status beams_mlp_load(beams_renderer* r, const char* path) {
  if (!r || !path) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_load: bad arguments");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(r, BEAMS_ERR_INVALID_ARG, "mlp_load: cannot open file");
  std::vector<unsigned char> blob(16 + 3 * (size_t)kParams * 4 + 4);
  const size_t got = std::fread(blob.data(), 1, blob.size(), f);
  const int extra = std::fgetc(f);
  std::fclose(f);
  if (got != blob.size() || extra != EOF) return fail(r, BEAMS_ERR_CONFIG, "mlp_load: wrong file size");
  uint32_t hdr[4], sum;
  std::memcpy(hdr, blob.data(), 16);
  std::memcpy(&sum, blob.data() + blob.size() - 4, 4);
  if (hdr[0] != 0x504c4d42u || hdr[1] != 1u || hdr[2] != (uint32_t)kParams)
    return fail(r, BEAMS_ERR_CONFIG, "mlp_load: not a version-1 BMLP checkpoint of this network");
  if (fnv1a(blob.data(), blob.size() - 4) != sum) return fail(r, BEAMS_ERR_CONFIG, "mlp_load: checksum mismatch");
  cudaSetDevice(r->device);
  MlpState* st = mlp_state(r);
  beams_status s = alloc_params(r, st);
  if (s != BEAMS_OK) return s;
  const float* fp = (const float*)(blob.data() + 16);
  cudaError_t e = cudaMemcpyAsync(st->P, fp, kParams * 4, cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st->m, fp + kParams, kParams * 4, cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st->v, fp + 2 * kParams, kParams * 4, cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "mlp_load");
  st->step = (int)hdr[3];
  st->ready = true;
  return BEAMS_OK;
}

}  // extern "C"
