// k_batch.cu — many render requests in one persistent launch.
//
// The reference renders one camera per RenderCells call
// (beams/rendering/MapperLightedVolume.cxx:114-193), each a map build followed
// by a view march. Here a batch of requests (each its own volume, camera,
// light and map size) is one grid of persistent blocks pulling work items from
// a global queue (batch.h): map-build items (kBatchChunk vertex slots of the
// light-aligned brick order each) and view items (a tile of pixels), with the
// map items of one request beside the view items of the one before it. A view
// item of request r waits, with a bounded wait, until all of r's map items have
// completed, so the grid never drains between the two stages. Queue order
// guarantees progress: every item a view item waits on was dequeued earlier by
// a running block that waits on nothing.
//
// The split variant runs the same items as two persistent launches, all map
// items and then all view items (MODE 1 and 2; stream order replaces the
// waits). The fused kernel holds the registers of both marches; it runs four
// blocks per SM like the split kernels by marching light rays one sample at a
// time (see below).
//
// Per item a block keeps the request's geometry and cell tables in shared
// memory (recomputed there when the request changes, so no table buffers or
// table launches exist). Results equal the single-request kernels': the light
// march per vertex is march_vertex (the K1 march) and the view march is
// view_march_pixel. Compiled with -fmad=false like every kernel file.
#include <cuda_runtime.h>

#include "batch.h"
#include "exact_device.cuh"
#include "light_march.cuh"
#include "view_march.cuh"

namespace beams {

namespace {

constexpr long long kWaitCycles = 4000000000ll;  // ~2 s at 2 GHz: a view item's wait for its map

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int find_request(const int* off, int n, int item) {
  int lo = 0, hi = n - 1;  // largest k with off[k] <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// MODE 0: map and view items in one launch; 1: map items only; 2: view items only.
// Four blocks per SM in every mode. The one-launch kernel (MODE 0) holds both
// marches' registers, so its light march issues one sample at a time (no
// two-sample pipeline, which it would otherwise use with SKIP): 64 registers,
// 8 bytes of spills with SKIP. On 64 mixed requests that took the one-launch
// plan from 98.0 ms (three blocks per SM, the pipelined skipping march) to
// 86.7 ms, below one render at a time (88.1 ms).
template <bool SKIP, int MODE>
__global__ void __launch_bounds__(kBatchThreads, 4) k_batch(const ExactGeo* __restrict__ geos,
                                                            const BatchDesc* __restrict__ descs,
                                                            const BatchPlan* __restrict__ pl,
                                                            const float4* __restrict__ tf,
                                                            BatchQueue* __restrict__ q, Counters* __restrict__ cnt) {
  __shared__ ExactGeo sg;
  __shared__ BatchDesc sd;
  __shared__ int s_item, s_req, s_phase, s_skip;
  __shared__ unsigned s_sub;
  __shared__ int s_bo[8];  // the request's light-aligned brick order
  extern __shared__ float4 s_dyn[];
  const int tid = threadIdx.x, lane = tid & 31;
  // shared TF (one colour map for the batch) and its normalised alpha
  const int tf_n = geos[0].tf_n;
  float4* s_tf = s_dyn;
  float* s_a = (float*)(s_tf + tf_n);
  float4* s_tab = (float4*)(s_a + ((tf_n + 3) & ~3));
  const float max_alpha = geos[0].max_alpha;
  for (int i = tid; i < tf_n; i += blockDim.x) {
    const float4 c = tf[i];
    s_tf[i] = c;
    s_a[i] = (max_alpha > 0.f) ? c.w / max_alpha : 0.f;
  }
  if (tid == 0) s_req = -1;
  __syncthreads();
  const BatchPlan& plan = *pl;
  unsigned lit = 0, hit = 0;
  for (;;) {
    if (tid == 0) {
      s_item = MODE == 2 ? plan.k1_total + (int)atomicAdd(&q->next_view, 1u) : (int)atomicAdd(&q->next, 1u);
      s_sub = 0u;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= (MODE == 1 ? plan.k1_total : plan.total)) break;
    const int seg = find_request(plan.seg_off, plan.nseg, item);
    const int phase = MODE == 1 ? 1 : MODE == 2 ? 2 : ((plan.seg_req[seg] >> 16) ? 2 : 1);
    const int req = plan.seg_req[seg] & 0xffff;
    const int li = item - plan.seg_off[seg];  // item index inside the request's phase
    if (req != s_req || phase != s_phase) {
      __syncthreads();  // every thread has read s_req / s_phase
      const int* src = (const int*)(geos + req);
      for (int i = tid; i < (int)(sizeof(ExactGeo) / 4); i += blockDim.x) ((int*)&sg)[i] = src[i];
      if (tid < (int)(sizeof(BatchDesc) / 4)) ((int*)&sd)[tid] = ((const int*)(descs + req))[tid];
      __syncthreads();
      const int ntab = phase == 1 ? sg.max_off[0] : sg.ntab;
      for (int i = tid; i < ntab; i += blockDim.x) s_tab[i] = table_entry(sg, i);
      if (tid == 0 && plan.brick_log2) brick_order_setup(sg, plan.brick_log2, s_bo);
      if (tid == 0) {
        s_req = req;
        s_phase = phase;
      }
      __syncthreads();
    }
    if (phase == 1) {
      // a chunk of kBatchChunk vertex slots; warps take 32-slot tiles from the block's counter
      const int bl = plan.brick_log2;
      const int base = li * kBatchChunk;
      for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(&s_sub, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= (unsigned)(kBatchChunk / 32)) break;
        const int slot = base + (int)(t << 5) + lane;
        int id = -1, x = 0, y = 0, z = 0;
        if (bl) {
          const int bi = slot >> (3 * bl), li = slot & ((1 << (3 * bl)) - 1), m = (1 << bl) - 1;
          // slots past the last brick (the request's last item is padded to a whole item) do nothing
          const int nb = ((const volatile int*)s_bo)[0] * ((const volatile int*)s_bo)[1] * ((const volatile int*)s_bo)[2];
          int bx, by, bz;
          pencil_brick(bi, s_bo, bx, by, bz);
          x = (bx << bl) + (li & m);
          y = (by << bl) + ((li >> bl) & m);
          z = (bz << bl) + (li >> (2 * bl));
          if (bi < nb && x < sg.pd[0] && y < sg.pd[1] && z < sg.pd[2]) id = (z * sg.pd[1] + y) * sg.pd[0] + x;
        } else if (slot < sd.nvert) {
          id = slot;
          x = id % sg.pd[0];
          y = (id / sg.pd[0]) % sg.pd[1];
          z = id / (sg.pd[0] * sg.pd[1]);
        }
        if (id >= 0) {
          const float V[3] = {vtx_coord(sg, 0, x), vtx_coord(sg, 1, y), vtx_coord(sg, 2, z)};
          float L[3];
          light_origin(sg, V, L);
          Accum<false> acc;
          unsigned ns = 0;
          march_vertex<float4, false, SKIP, false, SKIP && MODE != 0, true>(sg, sd.quads, s_tab + sg.ax_off[0], s_tab + sg.ax_off[1],
                                            s_tab + sg.ax_off[2], s_a, nullptr, sd.occ, V, L,
                                            [](const float*) { return 0.f; }, acc, ns);
          acc.store(sd.map, id);
        }
      }
      if (MODE == 0) {
        __threadfence();
        __syncthreads();
        if (tid == 0 && !plan.test_withhold) atomicAdd(&q->done1[req], 1u);
      } else {
        __syncthreads();  // every warp is done with this chunk before s_sub is reset
      }
    } else {
      if (MODE == 0 && tid == 0) {
        const unsigned need = (unsigned)plan.k1_items[req];
        const long long t0 = clock64();
        int skip = 0;
        while (ld_acquire(&q->done1[req]) < need) {
          // give up after the budget, or at once when another block already has
          if (clock64() - t0 > kWaitCycles || ld_acquire(&q->error)) {
            atomicOr(&q->error, 1u);
            skip = 1;
            break;
          }
          __nanosleep(200);
        }
        __threadfence();
        s_skip = skip;
      }
      __syncthreads();
      if (MODE == 0 && s_skip) continue;  // the host reports the timeout; this item's pixels stay unwritten
      // a tile_w x tile_h tile; warps take 8x4 sub-tiles from the block's counter
      const int tx0 = (li % sd.tiles_x) * plan.tile_w, ty0 = (li / sd.tiles_x) * plan.tile_h;
      const int sx = plan.tile_w >> 3, nsub = sx * (plan.tile_h >> 2);
      for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(&s_sub, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= (unsigned)nsub) break;
        const int x = tx0 + (((int)t % sx) << 3) + (lane & 7), y = ty0 + (((int)t / sx) << 2) + (lane >> 3);
        if (x < sg.width && y < sg.height) {
          float4 color;
          view_march_pixel<float4, true, float, NoRecord, SKIP>(sg, sd.quads, s_tab, s_tf, sd.map, x, y, color, lit,
                                                                hit, nullptr, sd.occ);
          sd.out[(size_t)y * sg.width + x] = color;
        }
      }
      __syncthreads();  // every warp is done with this tile before s_sub is reset
    }
  }
  warp_add(&cnt->lit_samples, lit);
  warp_add(&cnt->rays_hit, hit);
}

}  // namespace

template <int MODE>
cudaError_t mode_grid(size_t smem, int items, int& grid) {
  cudaError_t e = cudaFuncSetAttribute(k_batch<false, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_batch<true, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0, per_sm2 = 0, dev = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<false, MODE>, kBatchThreads, smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_batch<true, MODE>, kBatchThreads, smem);
  if (e != cudaSuccess) return e;
  per_sm = per_sm < per_sm2 ? per_sm : per_sm2;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  grid = sms * per_sm;
  if (grid > items) grid = items;
  if (grid < 1) grid = 1;
  return cudaSuccess;
}

cudaError_t batch_launch_config(int tf_n, size_t max_ntab, const BatchPlan& plan, size_t& smem, int grid[2]) {
  smem = (size_t)tf_n * sizeof(float4) + (size_t)((tf_n + 3) & ~3) * sizeof(float) + max_ntab * sizeof(float4);
  grid[1] = 0;
  if (!plan.split) return mode_grid<0>(smem, plan.total, grid[0]);
  cudaError_t e = mode_grid<1>(smem, plan.k1_total, grid[0]);
  if (e == cudaSuccess) e = mode_grid<2>(smem, plan.total - plan.k1_total, grid[1]);
  return e;
}

template <int MODE>
void launch_mode(const ExactGeo* geos, const BatchDesc* descs, const BatchPlan* plan, int skip, const float4* tf,
                 size_t smem, int grid, BatchQueue* q, Counters* cnt, cudaStream_t st) {
  if (skip)
    k_batch<true, MODE><<<grid, kBatchThreads, smem, st>>>(geos, descs, plan, tf, q, cnt);
  else
    k_batch<false, MODE><<<grid, kBatchThreads, smem, st>>>(geos, descs, plan, tf, q, cnt);
}

cudaError_t launch_batch(const ExactGeo* geos, const BatchDesc* descs, const BatchPlan* plan, int skip, int split,
                         const float4* tf, size_t smem, const int grid[2], BatchQueue* q, Counters* cnt,
                         cudaStream_t st) {
  if (!split) {
    launch_mode<0>(geos, descs, plan, skip, tf, smem, grid[0], q, cnt, st);
    return cudaGetLastError();
  }
  launch_mode<1>(geos, descs, plan, skip, tf, smem, grid[0], q, cnt, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  launch_mode<2>(geos, descs, plan, skip, tf, smem, grid[1], q, cnt, st);
  return cudaGetLastError();
}

}  // namespace beams
