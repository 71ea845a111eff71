// kernels.h — launch wrappers shared between the kernel files and the C-ABI layer.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "beams_params.h"

namespace beams {

cudaError_t launch_build_tables(const ExactGeo& g, float4* tab, cudaStream_t st);
cudaError_t launch_build_quads(const void* field, int in_dtype, void* quads, int quad_dtype, const int n[3],
                               cudaStream_t st);
cudaError_t launch_light_march_prec(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tab,
                                    const float4* tf, const float* tau, __half* map, Counters* cnt, cudaStream_t st,
                                    const unsigned char* occ = nullptr, const unsigned* vlist = nullptr);
cudaError_t launch_view_march_prec(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tab,
                                   const float4* tf, const __half* map, float4* out, Counters* cnt, cudaStream_t st,
                                   const unsigned char* occ = nullptr);
cudaError_t launch_light_march_f32(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                   float* map, Counters* cnt, cudaStream_t st, const BrickRef* refs = nullptr,
                                   int nrefs = 0, int self = -1, const unsigned* gate = nullptr,
                                   const unsigned char* occ = nullptr, const unsigned* vlist = nullptr);
// The work list of a masked map build (vlist above): zeroes list[0], then lists
// in list[1..] the vertices of the cells marked in cell_mask (one byte per map
// cell, x fastest), list[0] their count. list spans marked_list_bytes(pd):
// (M+1)^3 + 1 entries, then one byte per 8^3-cell block (scratch).
// gate (non-null): nothing is listed while *gate is 0.
size_t marked_list_bytes(const int pd[3]);
cudaError_t launch_list_marked_vertices(const ExactGeo& g, const unsigned char* cell_mask, const unsigned* gate,
                                        unsigned* list, cudaStream_t st);
// Empty-space occupancy of 8^3-cell macro-cells for the light march's skip.
void occupancy_dims(const int n[3], int occ_n[3]);
cudaError_t launch_build_occupancy(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tf,
                                   unsigned char* occ, cudaStream_t st);
// Learned form's lazy fallback (k_mlp_probe.cu): when the list of failing tiles
// is non-empty, clears the cell mask (one byte per map cell, rounded up to a
// 16-byte multiple) and marks the map cells that the listed tiles' view rays
// read; K1 given the mask builds the vertices of marked cells. host_count (host-mapped
// memory, or null) receives the list's length.
cudaError_t launch_mark_fallback_vertices(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                          const unsigned* flist, const unsigned* fcount, unsigned char* vmask,
                                          size_t mask_bytes, unsigned* host_count, Counters* cnt, cudaStream_t st);
// Marks (one byte per map cell, x fastest; the mask is not cleared here) every
// map cell that the view rays of the frame's window read at samples of alpha
// above 0, or (flist given) of the listed kFallbackTile^2 tiles, *fcount of
// them (nothing while it is 0). occ (window only): the march skips empty
// macro-cells. Zeroes and uses cnt->tiles_mark.
cudaError_t launch_mark_view_cells(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                   unsigned char* cell_mask, Counters* cnt, const unsigned* flist,
                                   const unsigned* fcount, cudaStream_t st, const unsigned char* occ = nullptr);
// The same over the precision form's 16-bit quads (quad_dtype 1: bfloat16,
// else binary16), window only.
cudaError_t launch_mark_view_cells_prec(const ExactGeo& g, int quad_dtype, const void* quads, const float4* tab,
                                        const float4* tf, unsigned char* cell_mask, Counters* cnt, cudaStream_t st,
                                        const unsigned char* occ = nullptr);
// K2 over a device list of kFallbackTile^2 pixel tiles (count in *fcount), with the map.
cudaError_t launch_view_march_tiles(const ExactGeo& g, const float4* quads, const float4* tab, const float4* tf,
                                    const float* map, float4* out, Counters* cnt, const unsigned* flist,
                                    const unsigned* fcount, cudaStream_t st);
size_t mlp_packed_bytes();
// Learned form probe (k_mlp_probe.cu): probe grid and fallback tiles of one frame.
constexpr int kProbeCap = 512;  // compositing samples recorded per probe pixel
struct ProbeLayout {
  int stride, offset, nqx, nqy, nprobe, ntiles, cap;
};
// What the network's view march records for the probe pixels (P = 0: none):
// per probe its compositing samples {x, y, z, 1}, {r, g, b, sa} and their count.
struct MlpProbe {
  int P, h, nqx, nqy, cap;
  float4* rec;
  int* count;
};
// Which pixels one network view march shades: every 8x4 warp tile; or the warp
// tiles outside the kFallbackTile^2 tiles already flagged for the exact path
// (skip = the probe check's flags, ftx tiles per row); or the probe pixels
// only, 32 per warp (probes_only; their lit samples are not counted, the
// later pass or the fallback renders their tiles again).
struct MlpPass {
  const unsigned* skip;
  int ftx;
  int probes_only;
};
ProbeLayout probe_layout(int width, int height, float fraction);
// recorded: the network's view march already recorded the probe samples (no probe march).
cudaError_t launch_mlp_probe(const ExactGeo& g, const ProbeLayout& L, const float4* quads, const float4* tab,
                             const float4* tf, const float4* img, float tol, float4* rec, int* count, unsigned* flags,
                             unsigned* flist, unsigned* fcount, float* probe_err, Counters* cnt, cudaStream_t st,
                             bool recorded = false);
cudaError_t launch_pack_weights(const float* P, uint2* W, float* aux, cudaStream_t st);
cudaError_t launch_composite(const float4* imgs, int nb, size_t npix, const int* order, float4* out,
                             cudaStream_t st);
cudaError_t launch_view_march_f32(const ExactGeo& g, const float* field, const float4* quads, const float4* tab,
                                  const float4* tf, const float* map, float4* out, Counters* cnt, cudaStream_t st,
                                  const unsigned char* occ = nullptr);
cudaError_t launch_selftest_division(float org, float h, int ncells, int samples, unsigned long long* d_out,
                                     cudaStream_t st);

cudaError_t launch_generate_blobs(float* out, const int n[3], const float* d_params, int nblobs,
                                  cudaStream_t st);
cudaError_t launch_generate_noise(float* out, const int n[3], const unsigned char* d_perm, int octaves,
                                  float base_freq, float lacunarity, float gain, cudaStream_t st);
cudaError_t launch_normalise01(float* data, int64_t count, unsigned* d_minmax, cudaStream_t st);

}  // namespace beams
