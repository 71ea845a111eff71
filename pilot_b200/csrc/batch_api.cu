// batch_api.cu — C ABI of the batched form: resident volumes and batches of
// render requests, run as one persistent launch replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/beams_b200.h"
#include "batch.h"
#include "kernels.h"
#include "renderer.h"

namespace beams {

beams_status make_geo_vol(beams_renderer* r, const beams_volume& v, const beams_camera* cam, ExactGeo& g);
beams_status validate_camera(beams_renderer* r, const beams_camera* cam);
beams_status ensure_buffer(beams_renderer* r, void** buf, size_t* cap, size_t bytes, const char* what);

struct BatchVolume {
  beams_volume vol{};
  void* owned = nullptr;         // device copy of a host field
  float4* quads = nullptr;       // float32 4-corner quads
  unsigned char* occ = nullptr;  // macro-cell occupancy under occ_tf (empty-space skipping)
  unsigned long long occ_tf = ~0ull;
  ~BatchVolume() {
    if (owned) cudaFree(owned);
    if (quads) cudaFree(quads);
    if (occ) cudaFree(occ);
  }
};

struct BatchTuned {
  beams_batch_options opts;
  float ms;
};

struct BatchState {
  std::vector<BatchVolume*> vols;
  beams_batch_options opts{32, 32, 8, 1, 0, 0, 0};
  // autotuner results per batch shape (tuning_key), kept for later calls and files
  std::map<std::string, BatchTuned> tuned;
  // per-signature device state
  std::vector<long long> sig;
  void* arena = nullptr;
  size_t arena_cap = 0;
  std::vector<size_t> map_off, img_off;
  BatchPlan plan{};
  size_t max_ntab = 0;
  size_t smem = 0;
  int grid[2] = {0, 0};
  ExactGeo* h_geos = nullptr;  // pinned staging, copied by the graph's first node
  BatchDesc* h_descs = nullptr;
  ExactGeo* d_geos = nullptr;
  BatchDesc* d_descs = nullptr;
  BatchQueue* d_q = nullptr;
  BatchPlan* d_plan = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;  // capture stream (the renderer's may be the legacy default stream)
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~BatchState() {
    drop_graph();
    for (auto* v : vols) delete v;
    if (arena) cudaFree(arena);
    if (h_geos) cudaFreeHost(h_geos);
    if (h_descs) cudaFreeHost(h_descs);
    if (d_geos) cudaFree(d_geos);
    if (d_descs) cudaFree(d_descs);
    if (d_q) cudaFree(d_q);
    if (d_plan) cudaFree(d_plan);
    if (cap) cudaStreamDestroy(cap);
  }
};

void batch_release(beams_renderer* r) {
  delete r->batch;
  r->batch = nullptr;
}

static BatchState* batch_state(beams_renderer* r) {
  if (!r->batch) r->batch = new BatchState();
  return r->batch;
}

static int log2_brick(int b) {
  switch (b) {
    case 0: return 0;
    case 8: return 3;
    case 16: return 4;
    case 32: return 5;
    case 64: return 6;
    default: return -1;
  }
}

// Map-build work items of one request: kBatchChunk vertex slots each, in rows or bricks.
static int k1_items(const ExactGeo& g, int bl) {
  long long slots = (long long)g.pd[0] * g.pd[1] * g.pd[2];
  if (bl) {
    const long long nb = (long long)((g.pd[0] + (1 << bl) - 1) >> bl) * ((g.pd[1] + (1 << bl) - 1) >> bl) *
                         ((g.pd[2] + (1 << bl) - 1) >> bl);
    slots = nb << (3 * bl);
  }
  return (int)((slots + kBatchChunk - 1) / kBatchChunk);
}

}  // namespace beams

using namespace beams;

extern "C" {

beams_status beams_batch_set_volumes(beams_renderer* r, const beams_volume* vols, int n) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (!vols || n < 1 || n > kMaxRequests) return fail(r, BEAMS_ERR_INVALID_ARG, "batch volumes: 1..256 volumes");
  for (int i = 0; i < n; ++i) {
    const beams_volume& v = vols[i];
    if (!v.data || v.dtype != BEAMS_F32 || v.assoc != BEAMS_ASSOC_POINTS)
      return fail(r, BEAMS_ERR_INVALID_ARG, "batch volumes: float32 point fields with data");
    for (int d = 0; d < 3; ++d)
      if (v.dims[d] < 2 || v.dims[d] > 8192 || !(v.spacing[d] > 0.0) || !std::isfinite(v.origin[d]))
        return fail(r, BEAMS_ERR_INVALID_ARG, "batch volumes: dims in [2, 8192], positive spacing");
    if ((double)(v.dims[0] - 1) * (v.dims[1] - 1) * v.dims[2] >= 4294967296.0)
      return fail(r, BEAMS_ERR_UNSUPPORTED, "batch volumes: volume too large for 32-bit cell indexing");
  }
  cudaSetDevice(r->device);
  BatchState* b = batch_state(r);
  cudaStreamSynchronize(r->stream);
  b->drop_graph();
  b->sig.clear();
  for (auto* v : b->vols) delete v;
  b->vols.clear();
  for (int i = 0; i < n; ++i) {
    BatchVolume* bv = new BatchVolume();
    b->vols.push_back(bv);
    bv->vol = vols[i];
    const size_t count = (size_t)vols[i].dims[0] * vols[i].dims[1] * vols[i].dims[2];
    cudaError_t e = cudaSuccess;
    if (!vols[i].on_device) {
      e = cudaMalloc(&bv->owned, count * sizeof(float));
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(bv->owned, vols[i].data, count * sizeof(float), cudaMemcpyHostToDevice, r->stream);
      bv->vol.data = bv->owned;
      bv->vol.on_device = 1;
    }
    const size_t nq = (size_t)(vols[i].dims[0] - 1) * (vols[i].dims[1] - 1) * vols[i].dims[2];
    if (e == cudaSuccess) e = cudaMalloc((void**)&bv->quads, nq * sizeof(float4));
    if (e == cudaSuccess) e = launch_build_quads(bv->vol.data, BEAMS_F32, bv->quads, BEAMS_F32, vols[i].dims, r->stream);
    if (e != cudaSuccess) {
      for (auto* v : b->vols) delete v;
      b->vols.clear();
      return cuda_fail(r, e, "batch volumes: upload / quad build");
    }
  }
  cudaError_t e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) return cuda_fail(r, e, "batch volumes");
  return BEAMS_OK;
}

beams_status beams_set_batch_options(beams_renderer* r, const beams_batch_options* o) {
  if (!r || !o) return fail(r, BEAMS_ERR_INVALID_ARG, "batch options: NULL argument");
  if (o->tile_w < 8 || o->tile_h < 4 || o->tile_w % 8 || o->tile_h % 4 || o->tile_w * o->tile_h > 16384)
    return fail(r, BEAMS_ERR_INVALID_ARG, "batch options: tile_w a multiple of 8, tile_h of 4, at most 16384 pixels");
  if (log2_brick(o->light_brick) < 0)
    return fail(r, BEAMS_ERR_INVALID_ARG, "batch options: light_brick must be 0, 8, 16, 32 or 64");
  if (o->split != 0 && o->split != 1) return fail(r, BEAMS_ERR_INVALID_ARG, "batch options: split must be 0 or 1");
  BatchState* b = batch_state(r);
  b->opts = *o;
  b->drop_graph();
  b->sig.clear();
  return BEAMS_OK;
}

beams_status beams_render_batch(beams_renderer* r, const beams_request* reqs, int n, beams_timings* t) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  BatchState* b = r->batch;
  if (!b || b->vols.empty()) return fail(r, BEAMS_ERR_STATE, "render_batch: no batch volumes set");
  if (!reqs || n < 1 || n > kMaxRequests) return fail(r, BEAMS_ERR_INVALID_ARG, "render_batch: 1..256 requests");
  if (r->tf_n < 1) return fail(r, BEAMS_ERR_STATE, "render_batch: no colour map set");
  cudaSetDevice(r->device);
  const int bl = log2_brick(b->opts.light_brick);
  // per-request geometry on the host (the renderer's settings stand in for each request's)
  const std::vector<Light> keep_lights = r->lights;
  int keep_m[3];
  std::memcpy(keep_m, r->map_m, sizeof(keep_m));
  const float keep_sd = r->sample_distance, keep_cut = r->cutoff;
  const bool keep_use = r->use_map;
  std::vector<ExactGeo> geos(n);
  std::vector<long long> sig;
  sig.push_back(n);
  sig.push_back(b->opts.tile_w);
  sig.push_back(b->opts.tile_h);
  sig.push_back(bl);
  sig.push_back(b->opts.split);
  beams_status s = BEAMS_OK;
  for (int i = 0; i < n && s == BEAMS_OK; ++i) {
    const beams_request& q = reqs[i];
    if (q.volume < 0 || q.volume >= (int)b->vols.size()) {
      s = fail(r, BEAMS_ERR_INVALID_ARG, "render_batch: request volume index out of range");
      break;
    }
    if (q.map_cells < 1 || q.map_cells > 1024 || !q.rgba_out || !(q.termination_alpha > 0.f) ||
        !(q.termination_alpha <= 1.f) || q.light_kind < 0 || q.light_kind > 1) {
      s = fail(r, BEAMS_ERR_INVALID_ARG, "render_batch: bad map size, output, termination alpha or light");
      break;
    }
    s = validate_camera(r, &q.camera);
    if (s != BEAMS_OK) break;
    Light L;
    L.kind = q.light_kind;
    for (int d = 0; d < 3; ++d) {
      L.v[d] = q.light[d];
      L.color[d] = q.light_color[d];
    }
    L.intensity = q.light_intensity;
    r->lights.assign(1, L);
    r->map_m[0] = r->map_m[1] = r->map_m[2] = q.map_cells;
    r->sample_distance = q.sample_distance;
    r->cutoff = q.termination_alpha;
    r->use_map = true;
    s = make_geo_vol(r, b->vols[q.volume]->vol, &q.camera, geos[i]);
    if (s == BEAMS_OK && (size_t)(geos[i].ntab + 2 * r->tf_n) * 16 > 200 * 1024)
      s = fail(r, BEAMS_ERR_UNSUPPORTED, "render_batch: volume/map axes too long for the shared cell tables");
    const bool direct = q.out_on_device && (((uintptr_t)q.rgba_out & 15) == 0);
    sig.push_back(q.volume);
    sig.push_back(q.map_cells);
    sig.push_back(q.camera.width);
    sig.push_back(q.camera.height);
    sig.push_back(direct ? 1 : 0);
  }
  r->lights = keep_lights;
  std::memcpy(r->map_m, keep_m, sizeof(keep_m));
  r->sample_distance = keep_sd;
  r->cutoff = keep_cut;
  r->use_map = keep_use;
  if (s != BEAMS_OK) return s;

  cudaError_t e = cudaSuccess;
  const int skip = b->opts.no_skip ? 0 : 1;
  sig.push_back(skip);
  if (skip) {
    // occupancy of every volume a request uses, under the current colour map
    for (int i = 0; i < n; ++i) {
      BatchVolume* bv = b->vols[reqs[i].volume];
      if (bv->occ && bv->occ_tf == r->tf_version) continue;
      ExactGeo g;
      s = make_geo_vol(r, bv->vol, nullptr, g);
      if (s != BEAMS_OK) return s;
      if (!bv->occ) e = cudaMalloc((void**)&bv->occ, (size_t)g.occ_n[0] * g.occ_n[1] * g.occ_n[2]);
      if (e == cudaSuccess) e = launch_build_occupancy(g, BEAMS_F32, bv->quads, r->d_tf, bv->occ, r->stream);
      if (e != cudaSuccess) return cuda_fail(r, e, "render_batch: occupancy build");
      bv->occ_tf = r->tf_version;
    }
  }
  if (sig != b->sig) {
    // new shapes: lay out the arena (maps, staging images), the plan, and re-capture
    cudaStreamSynchronize(r->stream);
    b->drop_graph();
    b->sig.clear();
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t off = 0;
    b->map_off.assign(n, 0);
    b->img_off.assign(n, (size_t)-1);
    BatchPlan& P = b->plan;
    std::memset(&P, 0, sizeof(P));
    P.n = n;
    P.tile_w = b->opts.tile_w;
    P.tile_h = b->opts.tile_h;
    P.brick_log2 = bl;
    P.skip = skip;
    P.split = b->opts.split;
    P.test_withhold = (b->opts.reserved == 0x7e57 && !P.split) ? 1 : 0;
    b->max_ntab = 0;
    std::vector<int> k2(n);
    for (int i = 0; i < n; ++i) {
      const ExactGeo& g = geos[i];
      b->map_off[i] = off;
      off = al(off + (size_t)g.pd[0] * g.pd[1] * g.pd[2] * sizeof(float));
      const bool direct = reqs[i].out_on_device && (((uintptr_t)reqs[i].rgba_out & 15) == 0);
      if (!direct) {
        b->img_off[i] = off;
        off = al(off + (size_t)g.width * g.height * sizeof(float4));
      }
      P.k1_items[i] = k1_items(g, bl);
      const int tx = (g.width + P.tile_w - 1) / P.tile_w, ty = (g.height + P.tile_h - 1) / P.tile_h;
      k2[i] = tx * ty;
      b->max_ntab = std::max(b->max_ntab, (size_t)g.ntab);
    }
    // Queue order o[0..n-1]: requests grouped by volume, so that the map build
    // of o[k] and the view march of o[k-1] that runs beside it read the same
    // field through L2; groups with the most work first, so the small requests
    // fill the tail of the launch. Then K1(o0), K1(o_k) and K2(o_{k-1}) for
    // k = 1..n-1, K2(o_{n-1}); split plans K1(o0..o_{n-1}), K2(o0..o_{n-1}).
    std::vector<int> o(n);
    std::vector<double> vwork(b->vols.size(), 0.0);
    for (int i = 0; i < n; ++i) {
      o[i] = i;
      vwork[reqs[i].volume] += (double)P.k1_items[i] + (double)k2[i];
    }
    std::stable_sort(o.begin(), o.end(), [&](int a, int c) {
      const int va = reqs[a].volume, vc = reqs[c].volume;
      if (va != vc) return vwork[va] != vwork[vc] ? vwork[va] > vwork[vc] : va < vc;
      return false;
    });
    int items = 0;
    auto seg = [&](int req, int phase, int count) {
      P.seg_off[P.nseg] = items;
      P.seg_req[P.nseg] = req | (phase == 2 ? 0x10000 : 0);
      ++P.nseg;
      items += count;
    };
    if (P.split) {
      for (int k = 0; k < n; ++k) seg(o[k], 1, P.k1_items[o[k]]);
      P.k1_total = items;
      for (int k = 0; k < n; ++k) seg(o[k], 2, k2[o[k]]);
    } else {
      for (int k = 0; k < n; ++k) {
        seg(o[k], 1, P.k1_items[o[k]]);
        if (k > 0) seg(o[k - 1], 2, k2[o[k - 1]]);
      }
      seg(o[n - 1], 2, k2[o[n - 1]]);
    }
    P.seg_off[P.nseg] = items;
    P.total = items;
    s = ensure_buffer(r, &b->arena, &b->arena_cap, std::max(off, (size_t)256), "allocating batch arena");
    if (s != BEAMS_OK) return s;
    e = batch_launch_config(r->tf_n, b->max_ntab, P, b->smem, b->grid);
    if (e != cudaSuccess) return cuda_fail(r, e, "render_batch: launch configuration");
    if (!b->h_geos) {
      e = cudaMallocHost((void**)&b->h_geos, kMaxRequests * sizeof(ExactGeo));
      if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_descs, kMaxRequests * sizeof(BatchDesc));
      if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_geos, kMaxRequests * sizeof(ExactGeo));
      if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_descs, kMaxRequests * sizeof(BatchDesc));
      if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_q, sizeof(BatchQueue));
      if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_plan, sizeof(BatchPlan));
      if (e != cudaSuccess) return cuda_fail(r, e, "allocating batch staging");
    }
    e = cudaMemcpyAsync(b->d_plan, &P, sizeof(BatchPlan), cudaMemcpyHostToDevice, r->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);  // P is pageable host memory
    if (e != cudaSuccess) return cuda_fail(r, e, "render_batch: plan upload");
  }
  // this call's parameters into the pinned staging the graph copies from
  cudaStreamSynchronize(r->stream);  // the previous replay has read the staging
  for (int i = 0; i < n; ++i) {
    b->h_geos[i] = geos[i];
    BatchDesc& d = b->h_descs[i];
    std::memset(&d, 0, sizeof(d));
    d.quads = b->vols[reqs[i].volume]->quads;
    d.occ = skip ? b->vols[reqs[i].volume]->occ : nullptr;
    d.map = (float*)((char*)b->arena + b->map_off[i]);
    d.out = b->img_off[i] == (size_t)-1 ? (float4*)reqs[i].rgba_out : (float4*)((char*)b->arena + b->img_off[i]);
    d.nvert = geos[i].pd[0] * geos[i].pd[1] * geos[i].pd[2];
    d.tiles_x = (geos[i].width + b->plan.tile_w - 1) / b->plan.tile_w;
  }
  auto enqueue = [&](cudaStream_t sq) -> cudaError_t {
    cudaError_t x = cudaMemcpyAsync(b->d_geos, b->h_geos, n * sizeof(ExactGeo), cudaMemcpyHostToDevice, sq);
    if (x == cudaSuccess)
      x = cudaMemcpyAsync(b->d_descs, b->h_descs, n * sizeof(BatchDesc), cudaMemcpyHostToDevice, sq);
    if (x == cudaSuccess) x = cudaMemsetAsync(b->d_q, 0, sizeof(BatchQueue), sq);
    if (x == cudaSuccess) x = cudaMemsetAsync(r->d_cnt, 0, sizeof(Counters), sq);
    if (x == cudaSuccess)
      x = launch_batch(b->d_geos, b->d_descs, b->d_plan, b->plan.skip, b->plan.split, r->d_tf, b->smem, b->grid,
                       b->d_q, r->d_cnt, sq);
    return x;
  };
  cudaEventRecord(r->ev[0], r->stream);
  if (b->opts.use_graph) {
    if (!b->exec) {
      if (!b->cap) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t x = enqueue(b->cap);
        e = cudaStreamEndCapture(b->cap, &b->graph);
        if (x != cudaSuccess) e = x;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
      if (e != cudaSuccess) {
        b->drop_graph();
        return cuda_fail(r, e, "render_batch: graph capture");
      }
    }
    e = cudaGraphLaunch(b->exec, r->stream);
  } else {
    e = enqueue(r->stream);
  }
  if (e != cudaSuccess) return cuda_fail(r, e, "render_batch launch");
  b->sig = sig;
  cudaEventRecord(r->ev[1], r->stream);
  bool host_out = false;
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    if (b->img_off[i] == (size_t)-1) continue;
    const size_t bytes = (size_t)geos[i].width * geos[i].height * sizeof(float4);
    e = cudaMemcpyAsync(reqs[i].rgba_out, (char*)b->arena + b->img_off[i], bytes,
                        reqs[i].out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->stream);
    host_out |= !reqs[i].out_on_device;
  }
  if (e != cudaSuccess) return cuda_fail(r, e, "render_batch: copying images out");
  cudaEventRecord(r->ev[2], r->stream);
  if (t || host_out) {
    e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "render_batch");
    BatchQueue qh;
    e = cudaMemcpy(&qh, b->d_q, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(r, e, "render_batch: queue");
    if (qh.error) return fail(r, BEAMS_ERR_TIMEOUT, "render_batch: a view tile timed out waiting for its map");
    if (t) {
      std::memset(t, 0, sizeof(*t));
      Counters c;
      e = cudaMemcpy(&c, r->d_cnt, sizeof(c), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cuda_fail(r, e, "reading counters");
      cudaEventElapsedTime(&t->view_march_ms, r->ev[0], r->ev[1]);
      cudaEventElapsedTime(&t->composite_ms, r->ev[1], r->ev[2]);
      cudaEventElapsedTime(&t->total_ms, r->ev[0], r->ev[2]);
      t->lit_samples = c.lit_samples;
      t->rays_hit = c.rays_hit;
      long long nv = 0;
      for (int i = 0; i < n; ++i) nv += (long long)geos[i].pd[0] * geos[i].pd[1] * geos[i].pd[2];
      t->map_vertices = (int)std::min<long long>(nv, 2147483647ll);
      t->kernel_launches = b->plan.split ? 2 : 1;
    }
  }
  return BEAMS_OK;
}

// The shape of a batch as the autotuner sees it: per request the volume's point
// dims, the map size and the image size (cameras and lights vary freely).
static bool tuning_key(const BatchState* b, const beams_request* reqs, int n, std::string& key) {
  std::ostringstream k;
  k << n;
  for (int i = 0; i < n; ++i) {
    const beams_request& q = reqs[i];
    if (q.volume < 0 || q.volume >= (int)b->vols.size()) return false;
    const beams_volume& v = b->vols[q.volume]->vol;
    k << ';' << v.dims[0] << ',' << v.dims[1] << ',' << v.dims[2] << ',' << q.map_cells << ','
      << q.camera.width << ',' << q.camera.height;
  }
  key = k.str();
  return true;
}

beams_status beams_batch_autotune(beams_renderer* r, const beams_request* reqs, int n, beams_batch_options* best,
                                  float* best_ms) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  BatchState* b = r->batch;
  if (!b) return fail(r, BEAMS_ERR_STATE, "batch_autotune: no batch volumes set");
  if (!reqs || n < 1) return fail(r, BEAMS_ERR_INVALID_ARG, "batch_autotune: no requests");
  std::string key;
  const bool keyed = tuning_key(b, reqs, n, key);
  if (keyed) {
    const auto it = b->tuned.find(key);
    if (it != b->tuned.end()) {  // tuned before: keep that result
      beams_status s = beams_set_batch_options(r, &it->second.opts);
      if (s == BEAMS_OK && best) *best = it->second.opts;
      if (s == BEAMS_OK && best_ms) *best_ms = it->second.ms;
      return s;
    }
  }
  const beams_batch_options keep = b->opts;
  cudaEvent_t a, z;
  cudaEventCreate(&a);
  cudaEventCreate(&z);
  beams_status s = BEAMS_OK;
  auto time_opts = [&](const beams_batch_options& o, float& ms_out) -> beams_status {
    beams_status st = beams_set_batch_options(r, &o);
    if (st == BEAMS_OK) st = beams_render_batch(r, reqs, n, nullptr);  // captures the graph
    float tmin = 3.4e38f;
    for (int rep = 0; rep < 2 && st == BEAMS_OK; ++rep) {
      cudaEventRecord(a, r->stream);
      st = beams_render_batch(r, reqs, n, nullptr);
      cudaEventRecord(z, r->stream);
      cudaError_t e = cudaEventSynchronize(z);
      if (e != cudaSuccess && st == BEAMS_OK) st = cuda_fail(r, e, "batch_autotune");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, z);
      tmin = std::min(tmin, ms);
    }
    ms_out = tmin;
    return st;
  };
  // Coordinate descent over skip, the vertex order and the view tile, run per
  // launch plan (one launch; map builds then view marches) from the current
  // options and repeated until a round changes nothing (three rounds at most);
  // the faster plan wins. (A single round that also toggled the plan stayed in
  // whichever plan it started from: 64 small requests tuned 8.7 ms from the
  // mixed batch's one-launch options, and 7.4 ms in one round per plan, against
  // 6.8 ms with 16x16 tiles and no skip in the split plan.)
  beams_batch_options bo = keep;
  bo.reserved = 0;
  float bt = 3.4e38f;
  for (int plan = 0; plan < 2 && s == BEAMS_OK; ++plan) {
    beams_batch_options po = keep;
    po.reserved = 0;
    if (plan == 1) po.split = !keep.split;
    float pt = 3.4e38f;
    s = time_opts(po, pt);
    for (int round = 0; round < 3 && s == BEAMS_OK; ++round) {
      bool moved = false;
      for (int stage = 0; stage < 3 && s == BEAMS_OK; ++stage) {
        std::vector<beams_batch_options> cand;
        beams_batch_options o = po;
        if (stage == 0) {
          o.no_skip = !po.no_skip;
          cand.push_back(o);
        } else if (stage == 1) {
          for (int br : {0, 8, 16, 32, 64})
            if (br != po.light_brick) {
              o.light_brick = br;
              cand.push_back(o);
            }
        } else {
          static const int tiles[][2] = {{8, 8}, {16, 16}, {32, 8}, {8, 32}, {32, 32}, {64, 32}, {64, 64}};
          for (const auto& tw : tiles)
            if (tw[0] != po.tile_w || tw[1] != po.tile_h) {
              o.tile_w = tw[0];
              o.tile_h = tw[1];
              cand.push_back(o);
            }
        }
        for (const auto& c : cand) {
          float ms = 0.f;
          s = time_opts(c, ms);
          if (s != BEAMS_OK) break;
          if (ms < pt) {
            pt = ms;
            po = c;
            moved = true;
          }
        }
      }
      if (!moved) break;
    }
    if (s == BEAMS_OK && pt < bt) {
      bt = pt;
      bo = po;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(z);
  if (s != BEAMS_OK) {
    beams_set_batch_options(r, &keep);
    return s;
  }
  s = beams_set_batch_options(r, &bo);
  if (s == BEAMS_OK && keyed) b->tuned[key] = BatchTuned{bo, bt};
  if (best) *best = bo;
  if (best_ms) *best_ms = bt;
  return s;
}

beams_status beams_batch_tuning_clear(beams_renderer* r) {
  if (!r) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "renderer is NULL");
  if (r->batch) r->batch->tuned.clear();
  return BEAMS_OK;
}

// Text file: a header line, then one line per batch shape:
// <key> <tile_w> <tile_h> <light_brick> <no_skip> <split> <ms>
// (files of format 1, written before the split option, lack <split>: read as 0)
beams_status beams_batch_tuning_save(beams_renderer* r, const char* path) {
  if (!r || !path) return fail(r, BEAMS_ERR_INVALID_ARG, "batch_tuning_save: NULL argument");
  std::ofstream f(path);
  if (!f) return fail(r, BEAMS_ERR_INVALID_ARG, std::string("batch_tuning_save: cannot write ") + path);
  f << "beams-batch-tuning 2\n";
  if (r->batch)
    for (const auto& e : r->batch->tuned)
      f << e.first << ' ' << e.second.opts.tile_w << ' ' << e.second.opts.tile_h << ' '
        << e.second.opts.light_brick << ' ' << e.second.opts.no_skip << ' ' << e.second.opts.split << ' '
        << e.second.ms << '\n';
  if (!f) return fail(r, BEAMS_ERR_INVALID_ARG, std::string("batch_tuning_save: write failed: ") + path);
  return BEAMS_OK;
}

beams_status beams_batch_tuning_load(beams_renderer* r, const char* path) {
  if (!r || !path) return fail(r, BEAMS_ERR_INVALID_ARG, "batch_tuning_load: NULL argument");
  if (!r->batch) return fail(r, BEAMS_ERR_STATE, "batch_tuning_load: no batch volumes set");
  std::ifstream f(path);
  if (!f) return fail(r, BEAMS_ERR_INVALID_ARG, std::string("batch_tuning_load: cannot read ") + path);
  std::string line;
  if (!std::getline(f, line) || (line != "beams-batch-tuning 1" && line != "beams-batch-tuning 2"))
    return fail(r, BEAMS_ERR_CONFIG, "batch_tuning_load: not a batch tuning file");
  const bool v1 = line == "beams-batch-tuning 1";
  std::map<std::string, BatchTuned> got;
  int ln = 1;
  while (std::getline(f, line)) {
    ++ln;
    if (line.empty()) continue;
    std::istringstream is(line);
    std::string key;
    BatchTuned t{};
    t.opts = r->batch->opts;
    t.opts.split = 0;
    if (!(is >> key >> t.opts.tile_w >> t.opts.tile_h >> t.opts.light_brick >> t.opts.no_skip) ||
        (!v1 && !(is >> t.opts.split)) || !(is >> t.ms) ||
        t.opts.tile_w < 8 || t.opts.tile_w % 8 || t.opts.tile_h < 4 || t.opts.tile_h % 4 ||
        t.opts.tile_w * t.opts.tile_h > 16384 || log2_brick(t.opts.light_brick) < 0 ||
        (t.opts.no_skip != 0 && t.opts.no_skip != 1) || (t.opts.split != 0 && t.opts.split != 1))
      return fail(r, BEAMS_ERR_CONFIG, "batch_tuning_load: bad entry on line " + std::to_string(ln));
    t.opts.reserved = 0;
    got[key] = t;
  }
  for (auto& e : got) r->batch->tuned[e.first] = e.second;
  return BEAMS_OK;
}

}  // extern "C"
