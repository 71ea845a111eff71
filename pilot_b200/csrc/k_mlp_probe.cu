// k_mlp_probe.cu — the learned form's per-tile check against the exact light march.
//
// A regular 1-in-P x 1-in-P grid of probe pixels (P = round(1/sqrt(fraction)),
// offset P/2) is re-marched after the network has shaded the frame:
//   1. k_probe_record: each probe pixel's view march (the K2 body, no map)
//      records its compositing samples (sa > 0): position, TF colour and
//      premultiplied alpha, up to kProbeCap per pixel;
//   2. k_probe_check: one warp per probe pixel runs the exact light march
//      (TransmittanceMap.h:279-332) from the light to each recorded sample,
//      composites the samples with that transmittance (the shading of
//      Sampler::operator(), LightedVolumeRenderer.cxx:456-475) and compares
//      with the network's pixel; a kFallbackTile^2 tile whose max |dRGBA|
//      exceeds the tolerance (or that holds no probe, or a probe past the cap)
//      joins the fallback list.
// The host then builds the exact map lazily, only where the listed tiles need
// it (k_mark_view_cells marks the map cells their view rays read,
// k_list_marked_vertices lists the corners of marked cells and K1 marches only
// those; all gated on the list being non-empty),
// and K2 re-renders the listed tiles, so a failing tile is exactly the exact
// form's pixels.
// Compiled with -fmad=false like every kernel file.
#include <cuda_runtime.h>

#include <algorithm>

#include "exact_device.cuh"
#include "kernels.h"
#include "light_march.cuh"
#include "view_march.cuh"

namespace beams {

namespace {

constexpr int kThreadsP = 256;

struct ProbeGrid {
  int P, h, nqx, nqy;  // stride, offset, probes per row / column
};

__host__ __device__ inline int probes_along(int n, int P, int h) { return n > h ? (n - h - 1) / P + 1 : 0; }

// Records compositing samples (sa > 0) of one pixel: {x, y, z, T} and {r, g, b, sa}.
struct SampleRecorder {
  float4* rec;
  int n, cap;
  __device__ __forceinline__ void operator()(const float* p, const float4& tfc, float sa) {
    if (!(sa > 0.f)) return;
    if (n < cap) {
      rec[2 * n] = make_float4(p[0], p[1], p[2], 1.f);
      rec[2 * n + 1] = make_float4(tfc.x, tfc.y, tfc.z, sa);
    }
    ++n;
  }
};

__global__ void __launch_bounds__(kThreadsP) k_probe_record(const ExactGeo g, const float4* __restrict__ quads,
                                                            const float4* __restrict__ tab,
                                                            const float4* __restrict__ tf, ProbeGrid pg, int cap,
                                                            float4* __restrict__ rec, int* __restrict__ count) {
  extern __shared__ float4 s_dyn[];
  float4* s_tab = s_dyn;
  float4* s_tf = s_dyn + g.ntab;
  for (int i = threadIdx.x; i < g.ntab; i += blockDim.x) s_tab[i] = tab[i];
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  const int nprobe = pg.nqx * pg.nqy;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nprobe; q += gridDim.x * blockDim.x) {
    const int x = (q % pg.nqx) * pg.P + pg.h, y = (q / pg.nqx) * pg.P + pg.h;
    SampleRecorder r{rec + (size_t)q * cap * 2, 0, cap};
    float4 color;
    unsigned lit = 0, hit = 0;
    view_march_pixel<float4, false, float, SampleRecorder>(g, quads, s_tab, s_tf, nullptr, x, y, color, lit, hit,
                                                           &r);
    count[q] = r.n;
  }
}

// One warp per probe pixel: the lanes run the exact light march
// (TransmittanceMap.h:279-332, the K1 march) to 32 of the pixel's recorded
// samples at a time, shade them with the exact transmittance (Sampler::operator(),
// LightedVolumeRenderer.cxx:456-475) and the warp composites them in sample order
// (lane j's terms broadcast in turn, so the sums round as a sequential loop
// does). Lane 0 compares with the network's pixel and lists the pixel's
// kFallbackTile^2 tile when max |dRGBA| exceeds the tolerance (or the pixel
// overflowed its record). Threads also list every tile that holds no probe
// pixel: it cannot be checked, so it always falls back.
__global__ void __launch_bounds__(kThreadsP, 3) k_probe_check(const ExactGeo g, const float4* __restrict__ quads,
                                                           const float4* __restrict__ tab,
                                                           const float4* __restrict__ tf, ProbeGrid pg, int cap,
                                                           const float4* __restrict__ rec,
                                                           const int* __restrict__ count,
                                                           const float4* __restrict__ img, float tol,
                                                           unsigned* __restrict__ flags, unsigned* __restrict__ flist,
                                                           unsigned* __restrict__ fcount,
                                                           float* __restrict__ probe_err,
                                                           Counters* __restrict__ cnt) {
  extern __shared__ float4 s_dyn[];
  const int nfield = g.max_off[0];
  float4* s_tab = s_dyn;
  float* s_a = (float*)(s_dyn + nfield);
  for (int i = threadIdx.x; i < nfield; i += blockDim.x) s_tab[i] = tab[i];
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_a[i] = (g.max_alpha > 0.f) ? tf[i].w / g.max_alpha : 0.f;
  __syncthreads();
  const int nprobe = pg.nqx * pg.nqy;
  const int ftx = (g.width + kFallbackTile - 1) / kFallbackTile;
  const int fty = (g.height + kFallbackTile - 1) / kFallbackTile;
  const int ntiles = ftx * fty;
  auto flag = [&](int tile) {
    if (atomicExch(&flags[tile], 1u) == 0u) {
      flist[atomicAdd(fcount, 1u)] = (unsigned)tile;
      atomicAdd(&cnt->fallback_tiles, 1ull);
    }
  };
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntiles; i += gridDim.x * blockDim.x) {
    const int tx = i % ftx, ty = i / ftx;
    const int x0 = tx * kFallbackTile, x1 = min(x0 + kFallbackTile, g.width);
    const int y0 = ty * kFallbackTile, y1 = min(y0 + kFallbackTile, g.height);
    // first probe column/row at or after x0 / y0
    const int kx = x0 <= pg.h ? 0 : (x0 - pg.h + pg.P - 1) / pg.P;
    const int ky = y0 <= pg.h ? 0 : (y0 - pg.h + pg.P - 1) / pg.P;
    const bool has = kx < pg.nqx && kx * pg.P + pg.h < x1 && ky < pg.nqy && ky * pg.P + pg.h < y1;
    if (!has) flag(i);
  }
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const float4* T0 = s_tab + g.ax_off[0];
  const float4* T1 = s_tab + g.ax_off[1];
  const float4* T2 = s_tab + g.ax_off[2];
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nprobe; q += nwarps) {
    const int x = (q % pg.nqx) * pg.P + pg.h, y = (q / pg.nqx) * pg.P + pg.h;
    const int m = count[q];
    float err = __int_as_float(0x7f800000);
    if (m <= cap) {
      const float4* r = rec + (size_t)q * cap * 2;
      float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int base = 0; base < m; base += 32) {
        const int k = base + lane;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, sa = 0.f;
        if (k < m) {
          const float4 pw = r[2 * k], tc = r[2 * k + 1];
          const float P[3] = {pw.x, pw.y, pw.z};
          float L[3];
          light_origin(g, P, L);
          Accum<false> acc;
          unsigned ns = 0;
          march_vertex<float4, false, false>(g, quads, T0, T1, T2, s_a, nullptr, nullptr, P, L,
                                             [](const float*) { return 0.f; }, acc, ns);
          const float tr = 1.f - acc.o;
          s0 = clamp01(tc.x * (tr * g.light_color[0]));
          s1 = clamp01(tc.y * (tr * g.light_color[1]));
          s2 = clamp01(tc.z * (tr * g.light_color[2]));
          sa = tc.w;
        }
        const int nk = min(32, m - base);
        for (int j = 0; j < nk; ++j) {
          const float a0 = __shfl_sync(0xffffffffu, s0, j), a1 = __shfl_sync(0xffffffffu, s1, j);
          const float a2 = __shfl_sync(0xffffffffu, s2, j), aa = __shfl_sync(0xffffffffu, sa, j);
          c.x = c.x + a0 * aa;
          c.y = c.y + a1 * aa;
          c.z = c.z + a2 * aa;
          c.w = aa + c.w;
        }
      }
      const float4 v = img[(size_t)y * g.width + x];
      err = fmaxf(fmaxf(fabsf(v.x - c.x), fabsf(v.y - c.y)), fmaxf(fabsf(v.z - c.z), fabsf(v.w - c.w)));
      if (v.x != v.x || v.y != v.y || v.z != v.z || v.w != v.w) err = __int_as_float(0x7f800000);
    }
    if (lane == 0) {
      if (probe_err) probe_err[q] = err;
      if (!(err <= tol)) flag((y / kFallbackTile) * ftx + x / kFallbackTile);
    }
  }
}

// Also copies the list's length to host-mapped memory (when given) for the
// host's choice of order in the next frame.
__global__ void k_clear_mask_gated(const unsigned* __restrict__ fcount, uint4* __restrict__ mask, size_t n16,
                                   volatile unsigned* host_count) {
  const unsigned nf = *fcount;
  if (host_count && blockIdx.x == 0 && threadIdx.x == 0) *host_count = nf;
  if (nf == 0u) return;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
    mask[i] = make_uint4(0u, 0u, 0u, 0u);
}

int grid_for(size_t n, int threads, int cap_blocks) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (size_t)cap_blocks) b = cap_blocks;
  return (int)b;
}

}  // namespace

cudaError_t launch_mark_fallback_vertices(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                          const unsigned* flist, const unsigned* fcount, unsigned char* vmask,
                                          size_t mask_bytes, unsigned* host_count, Counters* cnt, cudaStream_t st) {
  if (mask_bytes % 16 != 0) return cudaErrorInvalidValue;
  k_clear_mask_gated<<<148 * 4, 256, 0, st>>>(fcount, (uint4*)vmask, mask_bytes / 16, host_count);
  return launch_mark_view_cells(g, quads, tab, tf, vmask, cnt, flist, fcount, st);
}

ProbeLayout probe_layout(int width, int height, float fraction) {
  ProbeLayout L{};
  if (!(fraction > 0.f)) return L;
  int P = (int)lrintf(1.f / sqrtf(fminf(fraction, 1.f)));
  if (P < 1) P = 1;
  L.stride = P;
  L.offset = P / 2;
  L.nqx = probes_along(width, P, L.offset);
  L.nqy = probes_along(height, P, L.offset);
  L.nprobe = L.nqx * L.nqy;
  L.ntiles = ((width + kFallbackTile - 1) / kFallbackTile) * ((height + kFallbackTile - 1) / kFallbackTile);
  L.cap = kProbeCap;
  return L;
}

cudaError_t launch_mlp_probe(const ExactGeo& g, const ProbeLayout& L, const float4* quads, const float4* tab,
                             const float4* tf, const float4* img, float tol, float4* rec, int* count, unsigned* flags,
                             unsigned* flist, unsigned* fcount, float* probe_err, Counters* cnt, cudaStream_t st,
                             bool recorded) {
  if (L.nprobe < 0 || L.cap < 1) return cudaErrorInvalidValue;
  const ProbeGrid pg{L.stride, L.offset, L.nqx, L.nqy};
  cudaError_t e;
  if (L.nprobe > 0) {
    const size_t smem1 = ((size_t)g.ntab + (size_t)g.tf_n) * sizeof(float4);
    e = cudaFuncSetAttribute(k_probe_record, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
    if (e != cudaSuccess) return e;
    if (!recorded)
      k_probe_record<<<grid_for(L.nprobe, 64, 148 * 8), 64, smem1, st>>>(g, quads, tab, tf, pg, L.cap, rec, count);
  }
  const size_t smem2 = (size_t)g.max_off[0] * sizeof(float4) + (size_t)g.tf_n * sizeof(float);
  e = cudaFuncSetAttribute(k_probe_check, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
  if (e != cudaSuccess) return e;
  // one warp per probe pixel, and at least one thread per tile
  const size_t warps_needed = (size_t)(L.nprobe > 0 ? L.nprobe : 1);
  const size_t blocks = std::max((warps_needed + kThreadsP / 32 - 1) / (kThreadsP / 32),
                                 ((size_t)L.ntiles + kThreadsP - 1) / kThreadsP);
  k_probe_check<<<(int)std::max<size_t>(blocks, 1), kThreadsP, smem2, st>>>(g, quads, tab, tf, pg, L.cap, rec, count,
                                                                           img, tol, flags, flist, fcount, probe_err,
                                                                           cnt);
  return cudaGetLastError();
}

}  // namespace beams
