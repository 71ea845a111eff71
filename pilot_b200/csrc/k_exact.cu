// k_exact.cu — exact-form kernels.
//
// K1 light_march: one thread per map vertex ((M+1)^3), restating
//   TransmittanceMapGenerator::operator() (beams/rendering/TransmittanceMap.h:279-332)
//   with the light ray built in registers (LightRayOperations.h:32-43).
// K2 view_march: one thread per pixel, 8x4-pixel warp tiles, restating
//   CalcRayStart (LightedVolumeRenderer.cxx:644-718) and Sampler::operator()
//   (LightedVolumeRenderer.cxx:346-498) with the map lookup of
//   TransmittanceMapEstimator::GetEstimateUsingVertices (TransmittanceMap.h:166-197).
// K2c view_march_cells: SamplerCellAssoc::operator() (LightedVolumeRenderer.cxx:540-641).
//
// Both marches are instruction-bound (the field and map are served from L1/L2),
// so the layout is chosen to cut instructions per sample:
//  * the field is read as 4-corner quads (two 16-byte loads per cell);
//  * per-axis cell tables {lo, hi, RN(1/(hi-lo))} live in shared memory, so a
//    cell search is one guess plus rare fix-ups, and the parametric division is
//    Markstein's correction on the tabulated reciprocal;
//  * blocks are persistent and take 256-ray tiles from an atomic counter.
// Compiled with -fmad=false (see exact_device.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "exact_device.cuh"
#include "kernels.h"
#include "light_march.cuh"
#include "view_march.cuh"

namespace beams {

constexpr int kThreads = 256;

// Loads the cell tables (and nothing else) into shared memory.
__device__ __forceinline__ void load_tables(float4* s_tab, const float4* __restrict__ tab, int ntab) {
  for (int i = threadIdx.x; i < ntab; i += blockDim.x) s_tab[i] = tab[i];
}

// ---------------------------------------------------------------------------
// K1
// ---------------------------------------------------------------------------
// STITCH: the multi-brick Phase 3 — the march starts from the cross-brick
// prefix (stitch_prefix) instead of zero, as GenerateEstimator is re-run on
// the prefix opacities (LightedVolumeRenderer.cxx:1241-1252).
// Blocks per SM: 6 (40 registers) for the plain and the stitching exact march,
// which issue one sample at a time (the 257^3-vertex map of a 512^3 noise
// field: 2.70 ms against 2.78 ms at 4 blocks; the 2x2x2-brick frame 0.7% faster
// than at 4); the skipping, precision and rectilinear marches keep 4 (at 6 they
// spill: the 640^3 precision build went 6.4 -> 9.5 ms).
template <bool STITCH, bool PREC, bool SKIP, bool RECT>
constexpr int k1_blocks_per_sm() {
  return (PREC || SKIP || RECT) ? 4 : 6;
}

// A masked map build (the exact form's lazy map, the learned form's fallback,
// the multi-brick Phase 1): vertex (x, y, z) is built when one of the (up to 8)
// map cells it is a corner of is marked (one byte per cell, x fastest). The
// eight loads (clamped at the faces, where a vertex has fewer cells) are
// issued together.
__device__ __forceinline__ bool vertex_in_marked_cell(const unsigned char* __restrict__ cm, const int pd[3], int x,
                                                      int y, int z) {
  const unsigned mx = pd[0] - 1, mxy = mx * (unsigned)(pd[1] - 1);  // cells per row, per slice
  const unsigned x0 = max(x - 1, 0), x1 = min(x, pd[0] - 2);
  const unsigned y0 = max(y - 1, 0), y1 = min(y, pd[1] - 2);
  const unsigned z0 = max(z - 1, 0), z1 = min(z, pd[2] - 2);
  const unsigned r00 = z0 * mxy + y0 * mx, r01 = z0 * mxy + y1 * mx;
  const unsigned r10 = z1 * mxy + y0 * mx, r11 = z1 * mxy + y1 * mx;
  const unsigned m = __ldg(cm + r00 + x0) | __ldg(cm + r00 + x1) | __ldg(cm + r01 + x0) | __ldg(cm + r01 + x1) |
                     __ldg(cm + r10 + x0) | __ldg(cm + r10 + x1) | __ldg(cm + r11 + x0) | __ldg(cm + r11 + x1);
  return m != 0u;
}

// Blocks of 8^3 map cells: cb[d] = ceil((pd[d] - 1) / 8) per axis.
__host__ __device__ inline void cell_blocks(const int pd[3], int cb[3]) {
  for (int d = 0; d < 3; ++d) cb[d] = (pd[d] - 1 + 7) >> 3;
}

// One byte per 8^3-cell block: 1 when a cell of the block is marked (every
// block written, so nothing needs clearing). One warp per block, 16 cells a lane.
__global__ void __launch_bounds__(256) k_mark_cell_blocks(const ExactGeo g, const unsigned char* __restrict__ cm,
                                                          const unsigned* __restrict__ gate,
                                                          unsigned char* __restrict__ blocks) {
  if (gate && *gate == 0u) return;
  int cb[3];
  cell_blocks(g.pd, cb);
  const int nb = cb[0] * cb[1] * cb[2];
  const unsigned mx = g.pd[0] - 1, my = g.pd[1] - 1, mz = g.pd[2] - 1;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += nwarps) {
    const unsigned bx = b % cb[0], by = (b / cb[0]) % cb[1], bz = b / (cb[0] * cb[1]);
    unsigned any = 0;
#pragma unroll 4
    for (int k = lane; k < 512; k += 32) {
      const unsigned x = (bx << 3) + (k & 7), y = (by << 3) + ((k >> 3) & 7), z = (bz << 3) + (k >> 6);
      if (x < mx && y < my && z < mz) any |= __ldg(cm + (z * my + y) * mx + x);
    }
    any = __any_sync(0xffffffffu, any != 0u);
    if (lane == 0) blocks[b] = any ? 1 : 0;
  }
}

// The work list of a masked map build: the vertices of marked cells
// (vertex_in_marked_cell) in the light march's vertex order, list[1 + i] their
// ids, list[0] their count (zeroed before the launch). A masked build over this
// list takes one tile-counter atomic per 32 listed vertices, where testing every
// vertex took one per 32 vertices of the whole map (the 257^3-vertex map of a
// 512^3 field seen through a 30-degree camera: 31,073 vertices built, 0.41 ms
// for the per-vertex test, most of it atomics on the one counter). One append
// per warp that finds a vertex (lane order kept inside the warp).
__global__ void __launch_bounds__(256) k_list_marked_vertices(const ExactGeo g, const unsigned char* __restrict__ cm,
                                                              const unsigned char* __restrict__ blocks,
                                                              const unsigned* __restrict__ gate,
                                                              unsigned* __restrict__ list) {
  if (gate && *gate == 0u) return;
  int cb[3];
  cell_blocks(g.pd, cb);
  __shared__ int s_bo[8];
  const int bl = g.light_brick_log2;
  if (threadIdx.x == 0 && bl) brick_order_setup(g, bl, s_bo);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  auto append = [&](bool take, int x, int y, int z) {
    const unsigned b = __ballot_sync(0xffffffffu, take);
    if (b == 0u) return;
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(list, (unsigned)__popc(b));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (take) list[1 + base + __popc(b & ((1u << lane) - 1u))] = (unsigned)((z * g.pd[1] + y) * g.pd[0] + x);
  };
  if (bl == 0) {  // row order: 32-vertex tiles of the rows
    const int nvert = g.pd[0] * g.pd[1] * g.pd[2];
    for (int tile = warp; tile < (nvert + 31) >> 5; tile += nwarps) {
      const int id = (tile << 5) + lane;
      const int x = id % g.pd[0], y = (id / g.pd[0]) % g.pd[1], z = id / (g.pd[0] * g.pd[1]);
      append(id < nvert && vertex_in_marked_cell(cm, g.pd, x, y, z), x, y, z);
    }
    return;
  }
  // one warp per vertex brick of the order: the 8^3-cell blocks around the
  // brick's vertices first (a brick with none marked is skipped whole), then
  // the brick's 32-vertex tiles, each vertex tested against its own cells
  const int E = 1 << bl, m = E - 1;
  const int nbricks = s_bo[0] * s_bo[1] * s_bo[2];
  for (int bi = warp; bi < nbricks; bi += nwarps) {
    int v[3];
    pencil_brick(bi, s_bo, v[0], v[1], v[2]);
    int lo[3], n[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int c0 = max(v[d] * E - 1, 0), c1 = min(v[d] * E + m, g.pd[d] - 2);  // cells around the vertices
      lo[d] = c0 >> 3;
      n[d] = (c1 >> 3) - lo[d] + 1;
    }
    bool any = false;
    for (int k = lane; k < n[0] * n[1] * n[2]; k += 32) {
      const int i = k % n[0], j = (k / n[0]) % n[1], l = k / (n[0] * n[1]);
      any |= blocks[((lo[2] + l) * cb[1] + lo[1] + j) * cb[0] + lo[0] + i] != 0;
    }
    if (!__any_sync(0xffffffffu, any)) continue;
    for (int li = lane; li < E * E * E; li += 32) {
      const int x = (v[0] << bl) + (li & m), y = (v[1] << bl) + ((li >> bl) & m), z = (v[2] << bl) + (li >> (2 * bl));
      append(x < g.pd[0] && y < g.pd[1] && z < g.pd[2] && vertex_in_marked_cell(cm, g.pd, x, y, z), x, y, z);
    }
  }
}

// LIST: the vertices come from a work list (k_list_marked_vertices) instead of
// the whole map's vertex order.
template <typename QuadT, bool STITCH, bool PREC, bool SKIP, bool RECT = false, bool LIST = false>
__global__ void __launch_bounds__(kThreads, k1_blocks_per_sm<STITCH, PREC, SKIP, RECT>()) k_light_march(const ExactGeo g, const QuadT* __restrict__ quads,
                                                          const float4* __restrict__ tab,
                                                          const float4* __restrict__ tf,
                                                          const float* __restrict__ tau,
                                                          void* __restrict__ map, int nvert,
                                                          Counters* __restrict__ cnt,
                                                          const BrickRef* __restrict__ refs, int nrefs,
                                                          int self, const unsigned* __restrict__ gate,
                                                          const unsigned char* __restrict__ occ,
                                                          const unsigned* __restrict__ vlist) {
  // gate: the learned form's fallback builds the map only when a tile failed its
  // probes, and (LIST) only the vertices the failing tiles' view rays read
  if (gate && *gate == 0u) return;
  extern __shared__ float4 s_dyn[];
  const int nfield = g.max_off[0];             // field-axis table entries only
  float4* s_tab = s_dyn;
  float* s_a = (float*)(s_dyn + nfield);       // TF alpha / max alpha (TransmittanceMap.h:329)
  float* s_tau = s_a + g.tf_n;                 // -ln(1 - a) (precision form)
  load_tables(s_tab, tab, nfield);
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) {
    s_a[i] = (g.max_alpha > 0.f) ? tf[i].w / g.max_alpha : 0.f;
    if (PREC) s_tau[i] = tau[i];
  }
  __syncthreads();

  const float4* T0 = s_tab + g.ax_off[0];
  const float4* T1 = s_tab + g.ax_off[1];
  const float4* T2 = s_tab + g.ax_off[2];
  // Warps take 32-vertex tiles from a launch-wide counter: no block barriers
  // inside the march, and the tiles in flight sweep the vertex order as one
  // compact window.
  const int lane = threadIdx.x & 31;
  // The brick order's parameters live in shared memory and are re-read per
  // tile, so they occupy no registers across the march (the march is
  // register-bound).
  __shared__ int s_bo[8];
  if (threadIdx.x == 0) brick_order_setup(g, g.light_brick_log2, s_bo);
  __syncthreads();
  const int ntiles = [&] {
    if (LIST) return (int)((vlist[0] + 31u) >> 5);
    const int b0 = g.light_brick_log2;
    return b0 ? (s_bo[0] * s_bo[1] * s_bo[2]) << (3 * b0 - 5) : (nvert + 31) >> 5;
  }();
  unsigned ns = 0, built = 0;

  for (int tile = next_warp_tile(&cnt->tiles_light); tile < ntiles; tile = next_warp_tile(&cnt->tiles_light)) {
    int id;
    float V[3], L[3];
    const int bl = g.light_brick_log2;
    if (LIST) {
      const unsigned i = ((unsigned)tile << 5) + lane;
      if (i >= vlist[0]) continue;
      id = (int)vlist[1 + i];
      map_vertex(g, id, V);
    } else if (bl) {
      // tile -> brick (light-aligned order), lane -> vertex of the brick (x fastest inside the brick)
      const int bi = tile >> (3 * bl - 5);
      const int li = ((tile & ((1 << (3 * bl - 5)) - 1)) << 5) + lane;
      const int m = (1 << bl) - 1;
      int bx, by, bz;
      pencil_brick(bi, s_bo, bx, by, bz);
      const int x = (bx << bl) + (li & m), y = (by << bl) + ((li >> bl) & m);
      const int z = (bz << bl) + (li >> (2 * bl));
      if (x >= g.pd[0] || y >= g.pd[1] || z >= g.pd[2]) continue;
      id = (z * g.pd[1] + y) * g.pd[0] + x;
      V[0] = vtx_coord(g, 0, x);
      V[1] = vtx_coord(g, 1, y);
      V[2] = vtx_coord(g, 2, z);
    } else {
      id = (tile << 5) + lane;
      if (id >= nvert) continue;
      map_vertex(g, id, V);
    }
    ++built;
    light_origin(g, V, L);
    Accum<PREC> acc;
    march_vertex<QuadT, PREC, SKIP, RECT>(g, quads, T0, T1, T2, s_a, s_tau, occ, V, L,
                                    [&](const float dir[3]) {
                                      return STITCH ? stitch_prefix(refs, nrefs, self, L, V, dir) : 0.f;
                                    },
                                    acc, ns);
    acc.store(map, id);
  }
  warp_add(&cnt->light_samples, ns);
  if (LIST) warp_add(&cnt->map_vertices, built);
}

// ---------------------------------------------------------------------------
// K2 (point field)
// ---------------------------------------------------------------------------
template <typename QuadT, bool USE_MAP, typename MapT, bool LIST = false, bool SKIP = false, bool MULTI = false,
          bool RECT = false>
__global__ void __launch_bounds__(kThreads) k_view_march(const ExactGeo g, const QuadT* __restrict__ quads,
                                                         const float4* __restrict__ tab,
                                                         const float4* __restrict__ tf,
                                                         const MapT* __restrict__ map,
                                                         float4* __restrict__ out,
                                                         Counters* __restrict__ cnt,
                                                         const unsigned* __restrict__ flist = nullptr,
                                                         const unsigned* __restrict__ fcount = nullptr,
                                                         const unsigned char* __restrict__ occ = nullptr) {
  extern __shared__ float4 s_dyn[];
  float4* s_tab = s_dyn;
  float4* s_tf = s_dyn + g.ntab;
  load_tables(s_tab, tab, g.ntab);
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  // the pixel window (the whole image except for bricks, see ExactGeo::win)
  const int tiles_x = (g.win[2] + 7) >> 3;
  // flist: only the listed kFallbackTile^2 tiles (32 warp tiles each) are marched
  const int ntiles = LIST ? (int)(*fcount) * 32 : tiles_x * ((g.win[3] + 3) >> 2);
  const int ftx = (g.width + kFallbackTile - 1) / kFallbackTile;
  unsigned lit = 0, hit = 0;
  for (int tile = next_warp_tile(&cnt->tiles_view); tile < ntiles; tile = next_warp_tile(&cnt->tiles_view)) {
    int x, y;
    if (LIST) {
      const int f = (int)flist[tile >> 5], sub = tile & 31, lane = threadIdx.x & 31;
      x = (f % ftx) * kFallbackTile + ((sub & 3) << 3) + (lane & 7);
      y = (f / ftx) * kFallbackTile + ((sub >> 2) << 2) + (lane >> 3);
    } else {
      tile_pixel(tiles_x, tile, x, y);
      // outside the window's own extent: pushed past the image so the test below skips it
      x = (x < g.win[2]) ? x + g.win[0] : g.width;
      y = (y < g.win[3]) ? y + g.win[1] : g.height;
    }
    if (x < g.width && y < g.height) {
      float4 color;
      view_march_pixel<QuadT, USE_MAP, MapT, NoRecord, SKIP, MULTI, RECT>(g, quads, s_tab, s_tf, map, x, y, color,
                                                                           lit,
                                                                     hit, nullptr, occ);
      out[(size_t)y * g.width + x] = color;
    }
  }
  warp_add(&cnt->lit_samples, lit);
  warp_add(&cnt->rays_hit, hit);
}

// The masked map builds' marking pass: the view march without shading (the
// samples and their order do not depend on the map, since early termination
// reads only the colour map's alpha), CellMarker observing every lit sample.
// K2's warp tiles in K2's order over the window, or (LIST) over the listed
// kFallbackTile^2 tiles while *fcount > 0; tile counter cnt->tiles_mark. The
// march reads no map, so only the field axes' cell tables are staged.
template <typename QuadT, bool RECT, bool LIST, bool SKIP = false>
__global__ void __launch_bounds__(kThreads) k_mark_view_cells(const ExactGeo g, const QuadT* __restrict__ quads,
                                                              const float4* __restrict__ tab,
                                                              const float4* __restrict__ tf,
                                                              unsigned char* __restrict__ mask,
                                                              Counters* __restrict__ cnt,
                                                              const unsigned* __restrict__ flist,
                                                              const unsigned* __restrict__ fcount,
                                                              const unsigned char* __restrict__ occ) {
  if (LIST && *fcount == 0u) return;
  extern __shared__ float4 s_dyn[];
  const int nfield = g.max_off[0];
  float4* s_tab = s_dyn;
  float4* s_tf = s_dyn + nfield;
  load_tables(s_tab, tab, nfield);
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  const int tiles_x = (g.win[2] + 7) >> 3;
  const int ntiles = LIST ? (int)(*fcount) * 32 : tiles_x * ((g.win[3] + 3) >> 2);
  const int ftx = (g.width + kFallbackTile - 1) / kFallbackTile;
  for (int tile = next_warp_tile(&cnt->tiles_mark); tile < ntiles; tile = next_warp_tile(&cnt->tiles_mark)) {
    int x, y;
    if (LIST) {
      const int f = (int)flist[tile >> 5], sub = tile & 31, lane = threadIdx.x & 31;
      x = (f % ftx) * kFallbackTile + ((sub & 3) << 3) + (lane & 7);
      y = (f / ftx) * kFallbackTile + ((sub >> 2) << 2) + (lane >> 3);
    } else {
      tile_pixel(tiles_x, tile, x, y);
      x = (x < g.win[2]) ? x + g.win[0] : g.width;
      y = (y < g.win[3]) ? y + g.win[1] : g.height;
    }
    if (x < g.width && y < g.height) {
      CellMarker m{{g.morig[0], g.morig[1], g.morig[2]}, {g.minv[0], g.minv[1], g.minv[2]},
                   {g.pd[0], g.pd[1], g.pd[2]}, mask, 0xffffffffu};
      float4 color;
      unsigned lit = 0, hit = 0;
      view_march_pixel<QuadT, false, float, CellMarker, SKIP, false, RECT>(g, quads, s_tab, s_tf, nullptr, x, y,
                                                                           color, lit, hit, &m, occ);
    }
  }
}

// ---------------------------------------------------------------------------
// K2c (cell field, unlit)
// ---------------------------------------------------------------------------
template <typename FieldT>
__global__ void __launch_bounds__(kThreads) k_view_march_cells(const ExactGeo g,
                                                               const FieldT* __restrict__ field,
                                                               const float4* __restrict__ tab,
                                                               const float4* __restrict__ tf,
                                                               float4* __restrict__ out,
                                                               Counters* __restrict__ cnt) {
  extern __shared__ float4 s_dyn[];
  float4* s_tab = s_dyn;
  float4* s_tf = s_dyn + g.ntab;
  load_tables(s_tab, tab, g.ntab);
  for (int i = threadIdx.x; i < g.tf_n; i += blockDim.x) s_tf[i] = tf[i];
  __syncthreads();
  const int tiles_x = (g.width + 7) >> 3;
  const int ntiles = tiles_x * ((g.height + 3) >> 2);
  unsigned lit = 0, hit = 0;
  for (int tile = next_warp_tile(&cnt->tiles_view); tile < ntiles; tile = next_warp_tile(&cnt->tiles_view)) {
    int x, y;
    tile_pixel(tiles_x, tile, x, y);
    if (!(x < g.width && y < g.height)) continue;
    float4 color = make_float4(0.f, 0.f, 0.f, 0.f);
    float o[3], d[3], minD, maxD;
    if (ray_setup(g, x, y, o, d, minD, maxD)) {
      hit += 1;
      const float qd = (maxD - minD) / g.sd;
      long long budget = (qd < 1e9f) ? (long long)qd + 16 : 1000000000ll;
      float dist = minD + g.mesh_eps;
      float p[3] = {o[0] + dist * d[0], o[1] + dist * d[1], o[2] + dist * d[2]};
      while (!inside_vol(g, p) && dist < maxD && budget-- > 0) {
        dist += g.sd;
        p[0] = o[0] + dist * d[0];
        p[1] = o[1] + dist * d[1];
        p[2] = o[2] + dist * d[2];
      }
      const float sdx = g.sd * d[0], sdy = g.sd * d[1], sdz = g.sd * d[2];
      bool newCell = true;
      float tx = 2.f, ty = 2.f, tz = 2.f;
      float4 sc = make_float4(0.f, 0.f, 0.f, 0.f);
      float bl[3] = {0.f, 0.f, 0.f};
      float inv[3] = {0.f, 0.f, 0.f};
      int c[3] = {0, 0, 0};
      const int n1 = g.tf_n - 1;
      const unsigned cx = (unsigned)(g.n[0] - 1), cxy = (unsigned)(g.n[0] - 1) * (unsigned)(g.n[1] - 1);
      while (inside_vol(g, p) && dist < maxD && budget-- > 0) {
        const float mint = mn(tx, mn(ty, tz));
        const float maxt = mx(tx, mx(ty, tz));
        if (maxt > 1.f || mint < 0.f) newCell = true;
        if (newCell) {
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const float4* T = s_tab + g.ax_off[k];
            float4 e;
            if (p[k] == g.maxp[k]) {
              c[k] = g.n[k] - 2;
              e = T[c[k]];
            } else {
              c[k] = find_cell_walk_t(T, g.n[k] - 2, g.org[k], g.invh[k], p[k], e);
              inv[k] = e.w;
            }
            bl[k] = e.x;
          }
          const unsigned cid = (unsigned)c[2] * cxy + (unsigned)c[1] * cx + (unsigned)c[0];
          const float v = FieldLoad<FieldT>::ld(field, cid);
          const float nsv = (v - g.min_scalar) * g.inv_delta;
          sc = s_tf[tf_index_clamped(nsv * (float)n1, n1)];
          tx = (p[0] - bl[0]) * inv[0];
          ty = (p[1] - bl[1]) * inv[1];
          tz = (p[2] - bl[2]) * inv[2];
          newCell = false;
        }
        const float alpha = sc.w * (1.f - color.w);
        color.x = color.x + sc.x * alpha;
        color.y = color.y + sc.y * alpha;
        color.z = color.z + sc.z * alpha;
        color.w = alpha + color.w;
        ++lit;
        dist += g.sd;
        p[0] = p[0] + sdx;
        p[1] = p[1] + sdy;
        p[2] = p[2] + sdz;
        if (color.w >= g.cutoff) break;
        tx = (p[0] - bl[0]) * inv[0];
        ty = (p[1] - bl[1]) * inv[1];
        tz = (p[2] - bl[2]) * inv[2];
      }
      color.x = mn(color.x, 1.f);
      color.y = mn(color.y, 1.f);
      color.z = mn(color.z, 1.f);
      color.w = mn(color.w, 1.f);
    }
    out[(size_t)y * g.width + x] = color;
  }
  warp_add(&cnt->lit_samples, lit);
  warp_add(&cnt->rays_hit, hit);
}

// ---------------------------------------------------------------------------
// layout builders
// ---------------------------------------------------------------------------
// Cell tables: field axes then map axes, each entry {lo, hi, hi-lo, RN(1/(hi-lo))}
// with lo/hi the same float expressions the marches compare against.
__global__ void k_build_tables(const ExactGeo g, float4* __restrict__ tab) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.ntab) return;
  tab[i] = table_entry(g, i);
}

// Quad element conversion: input element -> stored quad element.
struct CvtF32 { static __device__ __forceinline__ float get(const float* p) { return __ldg(p); } };
struct CvtU16 {
  static __device__ __forceinline__ unsigned short get(const unsigned short* p) { return __ldg(p); }
};
struct CvtF32toBF16 {
  static __device__ __forceinline__ unsigned short get(const float* p) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(__ldg(p)));
  }
};
struct CvtF32toF16 {
  static __device__ __forceinline__ unsigned short get(const float* p) {
    return __half_as_ushort(__float2half_rn(__ldg(p)));
  }
};
template <typename In, typename Cvt> struct QuadOut;
template <> struct QuadOut<float, CvtF32> {
  using T = float4;
  static __device__ __forceinline__ T make(const float* b, int nx) {
    return make_float4(__ldg(b), __ldg(b + 1), __ldg(b + nx), __ldg(b + nx + 1));
  }
};
template <typename In, typename Cvt> struct QuadOut16 {
  static __device__ __forceinline__ uint2 make(const In* b, int nx) {
    const unsigned v0 = Cvt::get(b), v1 = Cvt::get(b + 1), v2 = Cvt::get(b + nx), v3 = Cvt::get(b + nx + 1);
    return make_uint2(v0 | (v1 << 16), v2 | (v3 << 16));
  }
};

template <typename In, typename OutT, typename Maker>
__global__ void k_build_quads(const In* __restrict__ f, OutT* __restrict__ q, int nx, int ny, int nz) {
  const unsigned qx = nx - 1, qxy = (unsigned)(nx - 1) * (ny - 1);
  const size_t total = (size_t)qxy * nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned z = (unsigned)(i / qxy);
    const unsigned r = (unsigned)(i - (size_t)z * qxy);
    const unsigned y = r / qx, x = r - y * qx;
    const In* b = f + ((size_t)z * ny + y) * nx + x;
    q[i] = Maker::make(b, nx);
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int g_num_sms = 0;
static int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

template <typename K>
static cudaError_t persistent_grid(K kernel, size_t smem, int ntiles, int& grid) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  grid = num_sms() * per_sm;
  if (grid > ntiles) grid = ntiles;
  if (grid < 1) grid = 1;
  return cudaSuccess;
}

cudaError_t launch_build_tables(const ExactGeo& g, float4* tab, cudaStream_t st) {
  k_build_tables<<<(g.ntab + 255) / 256, 256, 0, st>>>(g, tab);
  return cudaGetLastError();
}

// in_dtype: dtype of the field (BEAMS_F32/BF16/F16); quad_dtype: stored quads.
cudaError_t launch_build_quads(const void* field, int in_dtype, void* quads, int quad_dtype, const int n[3],
                               cudaStream_t st) {
  const size_t total = (size_t)(n[0] - 1) * (n[1] - 1) * n[2];
  size_t blocks = (total + 255) / 256;
  const size_t cap = (size_t)num_sms() * 16;
  const unsigned grid = (unsigned)(blocks < cap ? blocks : cap);
  if (quad_dtype == 0 && in_dtype == 0) {
    k_build_quads<float, float4, QuadOut<float, CvtF32>><<<grid, 256, 0, st>>>((const float*)field, (float4*)quads,
                                                                               n[0], n[1], n[2]);
  } else if (quad_dtype == 1 && in_dtype == 0) {
    k_build_quads<float, uint2, QuadOut16<float, CvtF32toBF16>><<<grid, 256, 0, st>>>(
        (const float*)field, (uint2*)quads, n[0], n[1], n[2]);
  } else if (quad_dtype == 2 && in_dtype == 0) {
    k_build_quads<float, uint2, QuadOut16<float, CvtF32toF16>><<<grid, 256, 0, st>>>(
        (const float*)field, (uint2*)quads, n[0], n[1], n[2]);
  } else if (quad_dtype == in_dtype && in_dtype != 0) {
    k_build_quads<unsigned short, uint2, QuadOut16<unsigned short, CvtU16>><<<grid, 256, 0, st>>>(
        (const unsigned short*)field, (uint2*)quads, n[0], n[1], n[2]);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename QuadT, bool STITCH, bool PREC>
static cudaError_t launch_k1(const ExactGeo& g, const void* quads, const float4* tab, const float4* tf,
                             const float* tau, void* map, Counters* cnt, cudaStream_t st, const BrickRef* refs,
                             int nrefs, int self, const unsigned* gate = nullptr,
                             const unsigned char* occ = nullptr, const unsigned* vlist = nullptr) {
  const int nvert = g.pd[0] * g.pd[1] * g.pd[2];
  const size_t smem = (size_t)g.max_off[0] * sizeof(float4) + 2 * (size_t)g.tf_n * sizeof(float);
  const int ntiles = (nvert + kThreads - 1) / kThreads;
  int grid = 0;
  // warps take tiles from a launch-wide counter, so the tiles in flight stay a
  // compact window of the brick order however unevenly the rays run
  cudaError_t e = cudaMemsetAsync(&cnt->tiles_light, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  if (g.rect && !PREC) {
    // explicit rectilinear coordinates, exact form: binary-search cell location, no
    // empty-space skipping (the precision form keeps the seeded walk, correct for
    // any increasing coordinates)
    if constexpr (!STITCH && !PREC && std::is_same<QuadT, float4>::value) {
      if (vlist) {
        e = persistent_grid(k_light_march<float4, false, false, false, true, true>, smem, ntiles, grid);
        if (e != cudaSuccess) return e;
        k_light_march<float4, false, false, false, true, true><<<grid, kThreads, smem, st>>>(
            g, (const float4*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, nullptr, vlist);
        return cudaGetLastError();
      }
      e = persistent_grid(k_light_march<float4, false, false, false, true>, smem, ntiles, grid);
      if (e != cudaSuccess) return e;
      k_light_march<float4, false, false, false, true><<<grid, kThreads, smem, st>>>(
          g, (const float4*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, nullptr, nullptr);
      return cudaGetLastError();
    } else {
      return cudaErrorInvalidValue;
    }
  }
  if constexpr (!STITCH && !PREC) {
    if (vlist) {
      if (occ) {
        e = persistent_grid(k_light_march<QuadT, false, false, true, false, true>, smem, ntiles, grid);
        if (e != cudaSuccess) return e;
        k_light_march<QuadT, false, false, true, false, true><<<grid, kThreads, smem, st>>>(
            g, (const QuadT*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, occ, vlist);
      } else {
        e = persistent_grid(k_light_march<QuadT, false, false, false, false, true>, smem, ntiles, grid);
        if (e != cudaSuccess) return e;
        k_light_march<QuadT, false, false, false, false, true><<<grid, kThreads, smem, st>>>(
            g, (const QuadT*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, nullptr, vlist);
      }
      return cudaGetLastError();
    }
  } else if constexpr (!STITCH && PREC) {
    if (vlist) {  // the precision form's lazy map
      if (occ) {
        e = persistent_grid(k_light_march<QuadT, false, true, true, false, true>, smem, ntiles, grid);
        if (e != cudaSuccess) return e;
        k_light_march<QuadT, false, true, true, false, true><<<grid, kThreads, smem, st>>>(
            g, (const QuadT*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, occ, vlist);
      } else {
        e = persistent_grid(k_light_march<QuadT, false, true, false, false, true>, smem, ntiles, grid);
        if (e != cudaSuccess) return e;
        k_light_march<QuadT, false, true, false, false, true><<<grid, kThreads, smem, st>>>(
            g, (const QuadT*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, nullptr, vlist);
      }
      return cudaGetLastError();
    }
  } else if constexpr (STITCH && !PREC) {
    if (vlist) {  // the lazy map of a multi-block scene: the stitched march over a brick's list
      if (occ) return cudaErrorInvalidValue;
      e = persistent_grid(k_light_march<QuadT, true, false, false, false, true>, smem, ntiles, grid);
      if (e != cudaSuccess) return e;
      k_light_march<QuadT, true, false, false, false, true><<<grid, kThreads, smem, st>>>(
          g, (const QuadT*)quads, tab, tf, tau, map, nvert, cnt, refs, nrefs, self, gate, nullptr, vlist);
      return cudaGetLastError();
    }
  } else {
    if (vlist) return cudaErrorInvalidValue;
  }
  if (occ) {
    e = persistent_grid(k_light_march<QuadT, STITCH, PREC, true>, smem, ntiles, grid);
    if (e != cudaSuccess) return e;
    k_light_march<QuadT, STITCH, PREC, true><<<grid, kThreads, smem, st>>>(g, (const QuadT*)quads, tab, tf, tau, map,
                                                                           nvert, cnt, refs, nrefs, self, gate, occ,
                                                                           nullptr);
  } else {
    e = persistent_grid(k_light_march<QuadT, STITCH, PREC, false>, smem, ntiles, grid);
    if (e != cudaSuccess) return e;
    k_light_march<QuadT, STITCH, PREC, false><<<grid, kThreads, smem, st>>>(g, (const QuadT*)quads, tab, tf, tau,
                                                                            map, nvert, cnt, refs, nrefs, self, gate,
                                                                            nullptr, nullptr);
  }
  return cudaGetLastError();
}

template <bool RECT, bool LIST, bool SKIP = false, typename QuadT = float4>
static cudaError_t launch_mark(const ExactGeo& g, const QuadT* quads, const float4* tab, const float4* tf,
                               unsigned char* cell_mask, Counters* cnt, const unsigned* flist,
                               const unsigned* fcount, cudaStream_t st, const unsigned char* occ = nullptr) {
  const size_t smem = ((size_t)g.max_off[0] + (size_t)g.tf_n) * sizeof(float4);
  const int ntiles = ((g.win[2] + 7) >> 3) * ((g.win[3] + 3) >> 2);
  int grid = 0;
  cudaError_t e = persistent_grid(k_mark_view_cells<QuadT, RECT, LIST, SKIP>, smem, ntiles, grid);
  if (e != cudaSuccess) return e;
  k_mark_view_cells<QuadT, RECT, LIST, SKIP><<<grid, kThreads, smem, st>>>(g, quads, tab, tf, cell_mask, cnt, flist,
                                                                            fcount, occ);
  return cudaGetLastError();
}

// The precision form's view march reads the 16-bit quads and never takes the
// rectilinear instantiation (its seeded walk serves both), so its marking
// pass does the same.
cudaError_t launch_mark_view_cells_prec(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tab,
                                        const float4* tf, unsigned char* cell_mask, Counters* cnt, cudaStream_t st,
                                        const unsigned char* occ) {
  cudaError_t e = cudaMemsetAsync(&cnt->tiles_mark, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  if (quad_dtype == 1)
    return occ ? launch_mark<false, false, true>(g, (const QuadBF16*)quads, tab, tf, cell_mask, cnt, nullptr, nullptr,
                                                 st, occ)
               : launch_mark<false, false, false>(g, (const QuadBF16*)quads, tab, tf, cell_mask, cnt, nullptr,
                                                  nullptr, st);
  return occ ? launch_mark<false, false, true>(g, (const QuadF16*)quads, tab, tf, cell_mask, cnt, nullptr, nullptr, st,
                                               occ)
             : launch_mark<false, false, false>(g, (const QuadF16*)quads, tab, tf, cell_mask, cnt, nullptr, nullptr,
                                                st);
}

cudaError_t launch_mark_view_cells(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                   unsigned char* cell_mask, Counters* cnt, const unsigned* flist,
                                   const unsigned* fcount, cudaStream_t st, const unsigned char* occ) {
  if (flist && !fcount) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(&cnt->tiles_mark, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  if (occ && !g.rect && !flist)  // samples in empty macro-cells have alpha 0 and mark nothing
    return launch_mark<false, false, true>(g, quads, tab, tf, cell_mask, cnt, nullptr, nullptr, st, occ);
  if (g.rect)
    return flist ? launch_mark<true, true>(g, quads, tab, tf, cell_mask, cnt, flist, fcount, st)
                 : launch_mark<true, false>(g, quads, tab, tf, cell_mask, cnt, nullptr, nullptr, st);
  return flist ? launch_mark<false, true>(g, quads, tab, tf, cell_mask, cnt, flist, fcount, st)
               : launch_mark<false, false>(g, quads, tab, tf, cell_mask, cnt, nullptr, nullptr, st);
}

size_t marked_list_bytes(const int pd[3]) {
  int cb[3];
  cell_blocks(pd, cb);
  const size_t nvert = (size_t)pd[0] * pd[1] * pd[2];
  return (nvert + 1) * sizeof(unsigned) + (size_t)cb[0] * cb[1] * cb[2];
}

cudaError_t launch_list_marked_vertices(const ExactGeo& g, const unsigned char* cell_mask, const unsigned* gate,
                                        unsigned* list, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(list, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  const size_t nvert = (size_t)g.pd[0] * g.pd[1] * g.pd[2];
  unsigned char* blocks = (unsigned char*)(list + nvert + 1);
  k_mark_cell_blocks<<<num_sms() * 8, 256, 0, st>>>(g, cell_mask, gate, blocks);
  k_list_marked_vertices<<<num_sms() * 8, 256, 0, st>>>(g, cell_mask, blocks, gate, list);
  return cudaGetLastError();
}

cudaError_t launch_light_march_f32(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                   float* map, Counters* cnt, cudaStream_t st, const BrickRef* refs, int nrefs,
                                   int self, const unsigned* gate, const unsigned char* occ, const unsigned* vlist) {
  if (refs)
    return launch_k1<float4, true, false>(g, quads, tab, tf, nullptr, map, cnt, st, refs, nrefs, self, gate, occ,
                                          vlist);
  return launch_k1<float4, false, false>(g, quads, tab, tf, nullptr, map, cnt, st, nullptr, 0, -1, gate, occ, vlist);
}

cudaError_t launch_light_march_prec(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tab,
                                    const float4* tf, const float* tau, __half* map, Counters* cnt, cudaStream_t st,
                                    const unsigned char* occ, const unsigned* vlist) {
  if (quad_dtype == 1)
    return launch_k1<QuadBF16, false, true>(g, quads, tab, tf, tau, map, cnt, st, nullptr, 0, -1, nullptr, occ, vlist);
  return launch_k1<QuadF16, false, true>(g, quads, tab, tf, tau, map, cnt, st, nullptr, 0, -1, nullptr, occ, vlist);
}

// Occupancy of the 8^3-cell macro-cells: 0 when every value the trilinear
// interpolation can produce inside cells [8m - 1, 8m + 8] (per axis) maps to a
// TF entry of alpha 0 that lies inside the TF's index range (so a skipped view
// sample still counts as lit). The corner min / max are widened by a relative
// margin (the interpolation can overshoot its corners by a few ulps) and the TF
// index range by 0.01 on each side; a NaN corner makes the macro-cell occupied,
// and so does touching a volume max face (the view march's max-face rule keeps
// the previous cell's reciprocal there, so those samples are never skipped).
template <typename QuadT>
__global__ void k_build_occupancy(const ExactGeo g, const QuadT* __restrict__ quads, const float4* __restrict__ tf,
                                  unsigned char* __restrict__ occ) {
  const int lane = threadIdx.x & 31;
  const int nm = g.occ_n[0] * g.occ_n[1] * g.occ_n[2];
  unsigned qx, qz;
  QuadLoad<QuadT>::strides(g, qx, qz);
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nm; w += (gridDim.x * blockDim.x) >> 5) {
    const int m0 = w % g.occ_n[0], m1 = (w / g.occ_n[0]) % g.occ_n[1], m2 = w / (g.occ_n[0] * g.occ_n[1]);
    int lo[3], ext[3];
    const int mm[3] = {m0, m1, m2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = max((mm[d] << kMacroLog2) - 1, 0);
      const int hi = min((mm[d] << kMacroLog2) + (1 << kMacroLog2), g.n[d] - 2);
      ext[d] = hi - lo[d] + 1;
    }
    const int count = ext[0] * ext[1] * ext[2];
    float vmin = __int_as_float(0x7f800000), vmax = -vmin;
    bool nan = false;
    for (int i = lane; i < count; i += 32) {
      const int x = lo[0] + i % ext[0], y = lo[1] + (i / ext[0]) % ext[1], z = lo[2] + i / (ext[0] * ext[1]);
      float v[8];
      QuadLoad<QuadT>::cell(quads, (unsigned)z * qz + (unsigned)y * qx + (unsigned)x, qx, qz, v);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        nan |= (v[k] != v[k]);
        vmin = fminf(vmin, v[k]);
        vmax = fmaxf(vmax, v[k]);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
      vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    nan = __any_sync(0xffffffffu, nan);
    if (lane == 0) {
      bool empty = !nan;
#pragma unroll
      for (int d = 0; d < 3; ++d) empty &= (lo[d] + ext[d] - 1 < g.n[d] - 2);  // max face
      if (empty) {
        const double n1 = g.tf_n - 1;
        const double pad = 1e-5 * fmax(fabs((double)vmin), fabs((double)vmax)) + 1e-30;
        const double f0 = ((double)vmin - pad - g.min_scalar) * g.inv_delta * n1;
        const double f1 = ((double)vmax + pad - g.min_scalar) * g.inv_delta * n1;
        double a = fmin(f0, f1) - 0.01, b = fmax(f0, f1) + 0.01;
        empty = a > -1.0 && b < n1 + 1.0;  // every sample passes the view march's range test
        a = fmin(fmax(a, 0.0), n1);
        b = fmin(fmax(b, 0.0), n1);
        if (g.max_alpha > 0.f)
          for (int i = (int)a; i <= (int)b && empty; ++i) empty = (tf[i].w == 0.f);
      }
      occ[w] = empty ? 0 : 1;
    }
  }
}

void occupancy_dims(const int n[3], int occ_n[3]) {
  for (int d = 0; d < 3; ++d) occ_n[d] = ((n[d] - 1) + (1 << kMacroLog2) - 1) >> kMacroLog2;
}

cudaError_t launch_build_occupancy(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tf,
                                   unsigned char* occ, cudaStream_t st) {
  const int nm = g.occ_n[0] * g.occ_n[1] * g.occ_n[2];
  const int blocks = (int)std::min<long long>(((long long)nm * 32 + 255) / 256, 148 * 64);
  if (quad_dtype == 1)
    k_build_occupancy<QuadBF16><<<blocks, 256, 0, st>>>(g, (const QuadBF16*)quads, tf, occ);
  else if (quad_dtype == 2)
    k_build_occupancy<QuadF16><<<blocks, 256, 0, st>>>(g, (const QuadF16*)quads, tf, occ);
  else
    k_build_occupancy<float4><<<blocks, 256, 0, st>>>(g, (const float4*)quads, tf, occ);
  return cudaGetLastError();
}

// K6: sort-last composite of nb brick images in the given order
// (MapperLightedVolume.cxx:284-297): a.rgb += b.rgb*(1-a.a), then a.a += b.a*(1-a.a).
struct CompositeOrder {
  int idx[kMaxBricks];
};

__global__ void k_composite(const float4* __restrict__ imgs, int nb, size_t npix, CompositeOrder order,
                            float4* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
    float4 a = imgs[(size_t)order.idx[0] * npix + i];
    for (int k = 1; k < nb; ++k) {
      const float4 b = imgs[(size_t)order.idx[k] * npix + i];
      a.x = a.x + b.x * (1.f - a.w);
      a.y = a.y + b.y * (1.f - a.w);
      a.z = a.z + b.z * (1.f - a.w);
      a.w = a.w + b.w * (1.f - a.w);
    }
    out[i] = a;
  }
}

cudaError_t launch_composite(const float4* imgs, int nb, size_t npix, const int* order, float4* out,
                             cudaStream_t st) {
  if (nb < 1 || nb > kMaxBricks) return cudaErrorInvalidValue;
  CompositeOrder o;
  for (int i = 0; i < kMaxBricks; ++i) o.idx[i] = i < nb ? order[i] : 0;
  size_t blocks = (npix + 255) / 256;
  const size_t cap = (size_t)num_sms() * 8;
  k_composite<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, st>>>(imgs, nb, npix, o, out);
  return cudaGetLastError();
}

template <typename QuadT, bool USE_MAP, typename MapT>
static cudaError_t launch_k2(const ExactGeo& g, const QuadT* quads, const float4* tab, const float4* tf,
                             const MapT* map, float4* out, Counters* cnt, const unsigned char* occ, cudaStream_t st) {
  const size_t smem = ((size_t)g.ntab + (size_t)g.tf_n) * sizeof(float4);
  const int ntiles = (((g.win[2] + 7) >> 3) * ((g.win[3] + 3) >> 2) + 7) / 8;  // 8 warp tiles per block
  int grid = 0;
  cudaError_t e;
  if (occ) {
    e = persistent_grid(k_view_march<QuadT, USE_MAP, MapT, false, true>, smem, ntiles, grid);
    if (e != cudaSuccess) return e;
    k_view_march<QuadT, USE_MAP, MapT, false, true><<<grid, kThreads, smem, st>>>(g, quads, tab, tf, map, out, cnt,
                                                                                  nullptr, nullptr, occ);
  } else {
    e = persistent_grid(k_view_march<QuadT, USE_MAP, MapT>, smem, ntiles, grid);
    if (e != cudaSuccess) return e;
    k_view_march<QuadT, USE_MAP, MapT><<<grid, kThreads, smem, st>>>(g, quads, tab, tf, map, out, cnt);
  }
  return cudaGetLastError();
}

cudaError_t launch_view_march_f32(const ExactGeo& g, const float* field, const float4* quads, const float4* tab,
                                  const float4* tf, const float* map, float4* out, Counters* cnt, cudaStream_t st,
                                  const unsigned char* occ) {
  const size_t smem = ((size_t)g.ntab + (size_t)g.tf_n) * sizeof(float4);
  const int ntiles = (((g.width + 7) >> 3) * ((g.height + 3) >> 2) + 7) / 8;  // 8 warp tiles per block
  int grid = 0;
  cudaError_t e;
  if (g.assoc_cells) {
    e = persistent_grid(k_view_march_cells<float>, smem, ntiles, grid);
    if (e != cudaSuccess) return e;
    k_view_march_cells<float><<<grid, kThreads, smem, st>>>(g, field, tab, tf, out, cnt);
  } else if (g.rect) {
    // explicit rectilinear coordinates (single light, no empty-space skipping)
    if (g.n_lights > 1) return cudaErrorInvalidValue;
    if (g.use_map) {
      e = persistent_grid(k_view_march<float4, true, float, false, false, false, true>, smem, ntiles, grid);
      if (e != cudaSuccess) return e;
      k_view_march<float4, true, float, false, false, false, true><<<grid, kThreads, smem, st>>>(g, quads, tab, tf,
                                                                                                map, out, cnt);
    } else {
      e = persistent_grid(k_view_march<float4, false, float, false, false, false, true>, smem, ntiles, grid);
      if (e != cudaSuccess) return e;
      k_view_march<float4, false, float, false, false, false, true><<<grid, kThreads, smem, st>>>(
          g, quads, tab, tf, (const float*)nullptr, out, cnt);
    }
  } else if (g.use_map && g.n_lights > 1) {
    // the multi-light extension (empty-space skipping is not combined with it)
    e = persistent_grid(k_view_march<float4, true, float, false, false, true>, smem, ntiles, grid);
    if (e != cudaSuccess) return e;
    k_view_march<float4, true, float, false, false, true><<<grid, kThreads, smem, st>>>(g, quads, tab, tf, map, out,
                                                                                        cnt);
  } else if (g.use_map) {
    return launch_k2<float4, true, float>(g, quads, tab, tf, map, out, cnt, occ, st);
  } else {
    return launch_k2<float4, false, float>(g, quads, tab, tf, (const float*)nullptr, out, cnt, occ, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_view_march_tiles(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                    const float* map, float4* out, Counters* cnt, const unsigned* flist,
                                    const unsigned* fcount, cudaStream_t st) {
  const size_t smem = ((size_t)g.ntab + (size_t)g.tf_n) * sizeof(float4);
  const int ntiles = (((g.width + 7) >> 3) * ((g.height + 3) >> 2) + 7) / 8;  // upper bound
  int grid = 0;
  cudaError_t e = persistent_grid(k_view_march<float4, true, float, true>, smem, ntiles, grid);
  if (e != cudaSuccess) return e;
  k_view_march<float4, true, float, true><<<grid, kThreads, smem, st>>>(g, quads, tab, tf, map, out, cnt, flist,
                                                                        fcount);
  return cudaGetLastError();
}

cudaError_t launch_view_march_prec(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tab,
                                   const float4* tf, const __half* map, float4* out, Counters* cnt, cudaStream_t st,
                                   const unsigned char* occ) {
  if (quad_dtype == 1)
    return g.use_map ? launch_k2<QuadBF16, true, __half>(g, (const QuadBF16*)quads, tab, tf, map, out, cnt, occ, st)
                     : launch_k2<QuadBF16, false, __half>(g, (const QuadBF16*)quads, tab, tf, map, out, cnt, occ, st);
  return g.use_map ? launch_k2<QuadF16, true, __half>(g, (const QuadF16*)quads, tab, tf, map, out, cnt, occ, st)
                   : launch_k2<QuadF16, false, __half>(g, (const QuadF16*)quads, tab, tf, map, out, cnt, occ, st);
}

// ---------------------------------------------------------------------------
// self-test: Markstein division against IEEE division on counting coordinates
// ---------------------------------------------------------------------------
__global__ void k_selftest_division(float org, float h, int ncells, int samples, unsigned long long* bad,
                                    unsigned long long* checked) {
  unsigned nb = 0, nc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)ncells * samples;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / samples);
    const unsigned k = (unsigned)(i - (long long)c * samples);
    const float lo = org + h * (float)c;
    const float hi = org + h * (float)(c + 1);
    const float w = hi - lo;
    const float r = 1.f / w;
    // x spans [-w/2, 3w/2]: a Weyl sequence over the interval plus exact end points.
    float x;
    if (k == 0) x = 0.f;
    else if (k == 1) x = w;
    else if (k == 2) x = w * 0.5f;
    else {
      const float u = (float)((k * 2654435769u) >> 8) * (1.f / 16777216.f);
      x = (u * 2.f - 0.5f) * w;
    }
    const float ref = x / w;  // IEEE (prec-div)
    const float got = div_rn_markstein(x, w, r);
    nb += (__float_as_uint(ref) != __float_as_uint(got)) ? 1u : 0u;
    nc += 1u;
  }
  const unsigned sb = __reduce_add_sync(0xffffffffu, nb), sc = __reduce_add_sync(0xffffffffu, nc);
  if ((threadIdx.x & 31) == 0) {
    if (sb) atomicAdd(bad, (unsigned long long)sb);
    atomicAdd(checked, (unsigned long long)sc);
  }
}

cudaError_t launch_selftest_division(float org, float h, int ncells, int samples, unsigned long long* d_out,
                                     cudaStream_t st) {
  const long long total = (long long)ncells * samples;
  long long blocks = (total + 255) / 256;
  const long long cap = (long long)num_sms() * 32;
  k_selftest_division<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, st>>>(org, h, ncells, samples, d_out,
                                                                              d_out + 1);
  return cudaGetLastError();
}

}  // namespace beams
