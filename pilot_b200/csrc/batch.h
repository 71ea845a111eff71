// batch.h — device-side layout of a batch of render requests (k_batch.cu,
// batch_api.cu).
#pragma once
#include <cuda_runtime.h>

#include "beams_params.h"

namespace beams {

constexpr int kMaxRequests = 256;
constexpr int kBatchThreads = 256;
constexpr int kBatchChunk = 2048;  // vertex slots per map-build work item (64 warp tiles)

// What the persistent kernel needs of one request besides its ExactGeo.
struct BatchDesc {
  const float4* quads;        // the request volume's 4-corner quad field (float32)
  const unsigned char* occ;   // its macro-cell occupancy (empty-space skipping), or null
  float* map;                 // (M+1)^3 opacities, 256-byte aligned, private to the request
  float4* out;                // width * height RGBA
  int nvert;
  int tiles_x;                // view tiles per image row
};

// Work items, in queue order over the request order o (requests grouped by
// volume, most work first): the map-build items of o0, then for k = 1..n-1
// the map-build items of o_k followed by the view items of o_{k-1}, and last
// the view items of o_{n-1}. A view item of r waits for r's map items, which
// all precede it in the queue; r's map is then one request old, so it is
// still in L2 when its view tiles read it, and the map build beside them
// reads the same volume. Segment k covers items
// [seg_off[k], seg_off[k+1]) of request seg_req[k] & 0xffff, phase 2 (view)
// when bit 16 is set. Lives in device memory (uploaded when the batch's shapes change).
// Split plans (two launches) order all map items first, o0..o_{n-1}, then all
// view items in the same order; k1_total counts the map items.
struct BatchPlan {
  int n;
  int nseg;
  int total;
  int k1_total;           // split plans: map items [0, k1_total), view items [k1_total, total)
  int split;              // 1: two launches (map items, then view items)
  int tile_w, tile_h;     // view tile: a multiple of 8 x 4 warp tiles
  int brick_log2;         // map-build vertex order inside a request (0 = rows)
  int skip;               // 1: both marches skip empty macro-cells (every desc has occ)
  int test_withhold;      // tests: map items never publish, so view items time out
  int seg_off[2 * kMaxRequests + 1];
  int seg_req[2 * kMaxRequests];
  int k1_items[kMaxRequests];  // map-build items per request (what a view item waits for)
};

// Zeroed before every launch.
struct BatchQueue {
  unsigned next;
  unsigned error;         // 1: a view item gave up waiting for its map (bounded wait)
  unsigned done1[kMaxRequests];
  unsigned next_view;     // split plans: the view launch's counter
};

// Dynamic shared memory and persistent grid(s) of the batch kernel(s) (call
// outside graph capture): grid[0] for the fused or map launch, grid[1] for the
// split plan's view launch.
cudaError_t batch_launch_config(int tf_n, size_t max_ntab, const BatchPlan& plan, size_t& smem, int grid[2]);
cudaError_t launch_batch(const ExactGeo* geos, const BatchDesc* descs, const BatchPlan* plan, int skip, int split,
                         const float4* tf, size_t smem, const int grid[2], BatchQueue* q, Counters* cnt,
                         cudaStream_t st);

}  // namespace beams
