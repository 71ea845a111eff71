// k_mlp_tc.cu — the transmittance network on the 5th-generation tensor cores
// (tcgen05): a dense forward pass, and the training step (forward, loss,
// backward, gradient accumulation) fused into one kernel.
//
// Operand layout in shared memory ("chunked"): an R-row x K-column bfloat16
// matrix is stored as K/8 chunks; chunk j holds columns 8j..8j+7 of every row,
// row r at j*R*16 + r*16 (16 bytes per row). One buffer serves three ways:
//  * K-major operand (rows = M or N, reduction over the columns): core
//    matrices are 8 rows x 16 bytes; the leading byte offset (next 8 columns,
//    the K direction) is R*16, the stride byte offset (next 8 rows) is 128, and
//    each 16-wide K slice starts 2*R*16 bytes further;
//  * MN-major operand (rows = K, columns = M or N): the same core matrices
//    read transposed; the stride byte offset (next 8 columns, the MN
//    direction) is R*16, the leading byte offset (next 8 rows, the K
//    direction) is 128, and each 16-row K slice starts 256 bytes further.
// Both are the SWIZZLE_NONE canonical layouts of the tcgen05 shared-memory
// descriptor (version 1). A TMA tiled load of a box {8 columns, 128 rows}
// lands exactly as one chunk, so input tiles arrive in place.
//
// Forward (k_mlp_fwd_tc, one CTA of six warpgroup pipelines per SM):
// 128-row tiles of precomputed features are loaded by TMA; per layer one
// thread of the pipeline issues the tcgen05.mma (M 128, N 64, K 16 per
// instruction, float32 accumulator in TMEM) and commits to an mbarrier; the
// pipeline's four warps read the accumulator back with tcgen05.ld (warp w:
// TMEM lanes 32(w%4).. = its rows), add the bias, apply ReLU, round to
// bfloat16 and write the next layer's operand. Six tiles are in flight per SM.
//
// Training (k_mlp_train_tc, 256 threads, one CTA per SM): per tile the forward
// keeps every layer's activations in shared memory, the head computes T, the
// loss and dz = scale 2 (T - t) T (1 - T), and the backward runs on the tensor
// cores: per layer l, the weight gradient G_W_l += in_l^T dY_l (MN-major A and
// B: M = the layer's inputs padded to 128, N 64, K = the tile's 128 rows) into
// a TMEM accumulator that lives across all the CTA's tiles, and the data
// gradient dY_{l-1} = (dY_l W_l^T) * (in_l > 0) (K-major A, MN-major B).
// Bias and head gradients are column sums on the CUDA cores. At the end the
// accumulators are added to the float32 gradient vector.
//
// Numerics as the CUDA-core kernels of k_mlp_train.cu: bfloat16 weights and
// activations at every product, float32 accumulation; the backward rounds dY
// to bfloat16 where it enters a product. Every mbarrier wait is bounded: a
// uniform timeout decision (BEAMS_ERR_TIMEOUT on the host), TMEM freed and
// copies in flight waited for on every path.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "mlp_common.cuh"
#include "mlp_host.h"

namespace beams {
namespace mlp {
namespace {

constexpr int kTile = 128;                  // rows per tile (tcgen05 M)
constexpr int kThreads = 256;               // eight warps: two per TMEM lane quarter
constexpr unsigned kWaitLimit = 1u << 24;   // mbarrier polls before giving up
constexpr int kXBytes = kTile * kIn * 2;    // 28672: one input tile
constexpr int kHBytes = kTile * kHid * 2;   // 16384: one activation tile
constexpr int kW1Bytes = kHid * kIn * 2;    // 14336
constexpr int kWhBytes = kHid * kHid * 2;   // 8192
constexpr int kWBytes = kW1Bytes + 3 * kWhBytes;  // 38912: all four weight matrices

// byte offset of element (r, k) of an R-row chunked operand
__host__ __device__ constexpr int ch_off(int R, int r, int k) { return (k >> 3) * R * 16 + r * 16 + (k & 7) * 2; }

// Instruction descriptor, kind::f16: D float32, A and B bfloat16, M x N, each
// operand K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
constexpr uint32_t kIdFwd = idesc(kTile, kHid, 0, 0);    // activations x W^T
constexpr uint32_t kIdWgrad = idesc(kTile, kHid, 1, 1);  // in^T x dY
constexpr uint32_t kIdDgrad = idesc(kTile, kHid, 0, 1);  // dY x W

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// The dynamic shared memory rounded up to a 1024-byte boundary (launches ask
// for 1024 bytes more than the layout needs): TMA destinations and operand
// descriptors then sit on known alignments.
__device__ __forceinline__ unsigned char* aligned_smem(unsigned char* raw) {
  const uint32_t a = smem_addr(raw);
  return raw + (((a + 1023u) & ~1023u) - a);
}

// Shared-memory matrix descriptor, SWIZZLE_NONE, version 1 (tcgen05).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         ((uint64_t)1 << 46);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Waits for the phase with the given parity to complete; false if the poll budget ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned parity) {
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// TMA: box {8 columns, 128 rows} of the feature matrix at (col, row) into one chunk.
__device__ __forceinline__ void tma_load_chunk(uint32_t dst, const CUtensorMap* map, int col, int row, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(map), "r"(col), "r"(row), "r"(bar)
      : "memory");
}

// One input tile: 14 chunk loads completing on bar (expect_tx set first).
__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap* map, int row, uint32_t bar) {
  mbar_expect_tx(bar, (uint32_t)kXBytes);
#pragma unroll 1
  for (int j = 0; j < kIn / 8; ++j) tma_load_chunk(dst + j * kTile * 16, map, j * 8, row, bar);
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float v[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// Stages the four weight matrices as bfloat16 B operands (W_l^T: N = 64
// outputs as rows, chunked over the inputs) and the biases, bf16(w5), b5.
__device__ void stage_weights(const float* __restrict__ P, unsigned char* W, float* aux) {
  for (int i = threadIdx.x; i < kIn * kHid; i += blockDim.x) {
    const int k = i / kHid, n = i - k * kHid;  // W1[k][n] at P[oW1 + k * 64 + n]
    *reinterpret_cast<__nv_bfloat16*>(W + ch_off(kHid, n, k)) = __float2bfloat16_rn(P[oW1 + i]);
  }
  const int oW[3] = {oW2, oW3, oW4};
  for (int l = 0; l < 3; ++l)
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
      const int k = i / kHid, n = i - k * kHid;
      *reinterpret_cast<__nv_bfloat16*>(W + kW1Bytes + l * kWhBytes + ch_off(kHid, n, k)) =
          __float2bfloat16_rn(P[oW[l] + i]);
    }
  const int oB[4] = {oB1, oB2, oB3, oB4};
  for (int i = threadIdx.x; i < 4 * kHid; i += blockDim.x) aux[i] = P[oB[i / kHid] + (i % kHid)];
  for (int i = threadIdx.x; i < kHid; i += blockDim.x) aux[4 * kHid + i] = bf16r(P[oW5 + i]);
  if (threadIdx.x == 0) aux[5 * kHid] = P[oB5];
}

__device__ __forceinline__ uint32_t w_addr(uint32_t wbase, int l) {
  return wbase + (l == 0 ? 0u : (uint32_t)(kW1Bytes + (l - 1) * kWhBytes));
}

// Layer l of the forward for one tile: A = the layer's input (chunked, 128
// rows; 112 or 64 columns), B = W_l^T, D = the TMEM accumulator.
__device__ __forceinline__ void issue_fwd(uint32_t d, uint32_t a, uint32_t wbase, int l) {
  const int K = l == 0 ? kIn : kHid;
  const uint32_t b = w_addr(wbase, l);
  for (int s = 0; s < K / 16; ++s)
    mma(d, sdesc(a + s * 2 * kTile * 16, kTile * 16, 128), sdesc(b + s * 2 * kHid * 16, kHid * 16, 128), kIdFwd,
        s > 0 ? 1u : 0u);
}

// Epilogue of a hidden layer for the calling thread's row r and 32 columns
// c0..c0+31: bf16(relu(acc + bias)), written as the chunked operand out when
// out is non-null; with want_h, h receives those bf16 values as floats (the
// head and the backward's ReLU mask read them). Each pair is rounded, clamped
// and packed by one cvt.rn.relu.bf16x2.f32: round-then-clamp equals
// round(max(x, 0)) for every finite x, since rounding keeps the sign (a NaN
// sum stays NaN here, where a float max would give 0). Against a separate
// packed max the dense forward on 2^22 rows went 0.310 -> 0.295 ms.
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem_acc, const float* bias, int r, int c0, float h[32],
                                                unsigned char* out, bool want_h = true) {
  tmem_ld32(tmem_acc + c0, h);
  tmem_wait_ld();
  uint32_t w[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float lo = h[2 * j] + bias[c0 + 2 * j], hi = h[2 * j + 1] + bias[c0 + 2 * j + 1];
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(w[j]) : "f"(hi), "f"(lo));  // lo in the low half
  }
  if (out) {
#pragma unroll
    for (int c = 0; c < 4; ++c)
      *reinterpret_cast<uint4*>(out + ch_off(kTile, r, c0 + c * 8)) =
          make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
  }
  if (want_h) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      h[2 * j] = __uint_as_float(w[j] << 16);
      h[2 * j + 1] = __uint_as_float(w[j] & 0xffff0000u);
    }
  }
}

// Half of the head's dot product: sum over the thread's 32 columns of h * bf16(w5).
__device__ __forceinline__ float head_partial(const float h[32], const float* w5, int c0) {
  float p = 0.f;
#pragma unroll
  for (int j = 0; j < 32; ++j) p = fmaf(h[j], w5[c0 + j], p);
  return p;
}

// T from the two halves (the same expression in both kernels, so their T agree bit for bit).
__device__ __forceinline__ float head_T(float b5, float p0, float p1) {
  const float z = b5 + (p0 + p1);
  return 1.f / (1.f + expf(-z));
}

// ---------------------------------------------------------------------------
// dense forward: six independent tile pipelines per SM
// ---------------------------------------------------------------------------
// One CTA of six warpgroups per SM. Warpgroup p runs its own pipeline over
// tiles p, p + 6*grid, ...: its tile buffer (the TMA-loaded input, then each
// layer's activations over it), two mbarriers and a 64-column TMEM accumulator
// are its own; the weights are shared. While one pipeline waits on its MMA, its
// next tile's load or runs its epilogue, the other five keep the tensor core
// busy; a pipeline's next tile is loaded as soon as its last layer has read the
// activations. Per-pipeline synchronisation uses named barriers (ids 1..6,
// 128 threads). Six pipelines with one buffer each ran 0.39 ms on 2^22 rows,
// four with a separate activation buffer (and the next load under the last
// three layers) 0.44 ms.
constexpr int kPipes = 6;
constexpr int kFwdThreads = 128 * kPipes;
constexpr int kAuxFloats = 5 * kHid + 1;                              // biases, w5, b5
constexpr int kFwdPipeBytes = kXBytes;                                // 28672: input tile, then activations
constexpr int kFwdOffPipe = kWBytes;                                  // 38912
constexpr int kFwdOffAux = kFwdOffPipe + kPipes * kFwdPipeBytes;      // 210944
constexpr int kFwdOffBar = ((kFwdOffAux + kAuxFloats * 4 + 15) / 16) * 16;
constexpr int kFwdSmem = kFwdOffBar + kPipes * 16;
static_assert(kFwdOffPipe % 128 == 0 && kFwdPipeBytes % 128 == 0, "TMA destinations on 128-byte boundaries");
static_assert(kFwdSmem + 1024 <= 227 * 1024, "one CTA of six pipelines fits the shared memory of an SM");
constexpr uint32_t kFwdCols = 512;  // TMEM columns: 64 per pipeline, allocated as a power of two
static_assert(64 * kPipes <= (int)kFwdCols, "TMEM columns");

__device__ __forceinline__ void pipe_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
// Named-barrier OR over the pipeline's 128 threads: a uniform decision.
__device__ __forceinline__ bool pipe_sync_or(int id, bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, 128, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}\n"
      : "=r"(out)
      : "r"((uint32_t)v), "r"(id)
      : "memory");
  return out != 0;
}

__global__ void __launch_bounds__(kFwdThreads, 1) k_mlp_fwd_tc(const __grid_constant__ CUtensorMap xmap, int row0,
                                                               int n, const float* __restrict__ P,
                                                               float* __restrict__ T, unsigned* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  unsigned char* sm = aligned_smem(sm_raw);
  float* aux = reinterpret_cast<float*>(sm + kFwdOffAux);
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, pipe = warp >> 2, q = warp & 3;
  const int ptid = tid & 127, bar_id = 1 + pipe;
  const int r = q * 32 + (tid & 31);  // the thread's row of the tile = its TMEM lane
  unsigned char* H = sm + kFwdOffPipe + pipe * kFwdPipeBytes;  // over the input tile, once layer 0 has read it
  const uint32_t wbase = smem_addr(sm);
  const uint32_t xaddr = smem_addr(sm + kFwdOffPipe + pipe * kFwdPipeBytes), haddr = smem_addr(H);
  const uint32_t bar_load = smem_addr(sm + kFwdOffBar + pipe * 16), bar_mma = bar_load + 8;
  const int ntiles = (n + kTile - 1) / kTile;

  stage_weights(P, sm, aux);
  if (ptid == 0) {
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&s_tmem, kFwdCols);
  fence_async_smem();  // the weights were written by ordinary stores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem + 64u * (uint32_t)pipe;           // this pipeline's columns
  const uint32_t tmem_acc = tmem + ((uint32_t)(q * 32) << 16);   // and this warp's lanes

  const int stride = gridDim.x * kPipes;
  int tile = blockIdx.x * kPipes + pipe;
  if (ptid == 0 && tile < ntiles) tma_load_tile(xaddr, &xmap, row0 + tile * kTile, bar_load);
  bool load_pending = tile < ntiles, ok = true;
  unsigned lph = 0, mph = 0;
  for (; tile < ntiles; tile += stride) {
    ok = mbar_wait(bar_load, lph);
    if (pipe_sync_or(bar_id, !ok)) {
      ok = false;
      break;
    }
    lph ^= 1u;
    load_pending = false;
    float h[32], p0 = 0.f, p1 = 0.f;
    for (int l = 0; l < 4; ++l) {
      if (ptid == 0) {
        tc_fence_after();
        issue_fwd(tmem, l == 0 ? xaddr : haddr, wbase, l);
        mma_commit(bar_mma);
      }
      ok = mbar_wait(bar_mma, mph);
      mph ^= 1u;
      if (pipe_sync_or(bar_id, !ok)) {
        ok = false;
        break;
      }
      tc_fence_after();
      if (l == 3 && tile + stride < ntiles) {
        // the last layer has read the activations: load the next tile in their place
        if (ptid == 0) tma_load_tile(xaddr, &xmap, row0 + (tile + stride) * kTile, bar_load);
        load_pending = true;
      }
      // two halves of the row in turn (32 live accumulator values per thread)
      hidden_epilogue(tmem_acc, aux + l * kHid, r, 0, h, l < 3 ? H : nullptr, l == 3);
      if (l == 3) p0 = head_partial(h, aux + 4 * kHid, 0);
      hidden_epilogue(tmem_acc, aux + l * kHid, r, 32, h, l < 3 ? H : nullptr, l == 3);
      if (l == 3) p1 = head_partial(h, aux + 4 * kHid, 32);
      fence_async_smem();
      tc_fence_before();
      pipe_sync(bar_id);
    }
    if (!ok) break;
    const int row = tile * kTile + r;
    if (row < n && T)
      T[row] = head_T(aux[5 * kHid], p0, p1);
  }
  if (!ok) {
    if (ptid == 0) atomicExch(err, 1u);
    // a load still in flight lands in this CTA's shared memory: wait for it (bounded)
    if (load_pending) mbar_wait(bar_load, lph);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(s_tmem, kFwdCols);
  }
}

// ---------------------------------------------------------------------------
// fused training step
// ---------------------------------------------------------------------------
constexpr int kTrOffX = kWBytes;                       // 38912
constexpr int kTrOffH = kTrOffX + kXBytes;             // 67584: H0..H3
constexpr int kTrOffDY = kTrOffH + 4 * kHBytes;        // 133120
constexpr int kTrOffAux = kTrOffDY + kHBytes;          // 149504
constexpr int kTrAuxFloats = kAuxFloats + 2 * kTile + kTile;  // + head halves, dz per row
constexpr int kTrOffBar = ((kTrOffAux + kTrAuxFloats * 4 + 15) / 16) * 16;
constexpr int kTrSmem = kTrOffBar + 16;
// TMEM columns: forward accumulator, data gradient, weight gradients of layers 0..3
constexpr uint32_t kColFwd = 0, kColDg = 64, kColWg = 128;
constexpr uint32_t kTrCols = 512;

// The wgrad A operand (a layer's input, MN-major, M padded to 128) reads 16
// column chunks = 32 KB from the buffer's start: X (14 chunks) runs into H0,
// H0..H2 (8 chunks) into the next activation buffer. All inside the layout.
static_assert(kTrOffX + 16 * kTile * 16 <= kTrOffDY, "wgrad A read of X stays inside shared memory");
static_assert(kTrOffH + 2 * kHBytes + 16 * kTile * 16 <= kTrOffDY, "wgrad A read of H2 stays inside H3");

__global__ void __launch_bounds__(kThreads, 1) k_mlp_train_tc(const __grid_constant__ CUtensorMap xmap, int row0,
                                                              int n, const float* __restrict__ P,
                                                              const float* __restrict__ target, float scale,
                                                              float* __restrict__ G, float* __restrict__ T,
                                                              float* __restrict__ loss, unsigned* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  unsigned char* sm = aligned_smem(sm_raw);
  float* aux = reinterpret_cast<float*>(sm + kTrOffAux);
  float* part = aux + 5 * kHid + 1;   // [2][kTile]
  float* s_dz = part + 2 * kTile;     // [kTile]
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, q = warp & 3, hf = warp >> 2;
  const int r = q * 32 + (tid & 31), c0 = hf * 32;
  const uint32_t base = smem_addr(sm);
  const uint32_t wbase = base, xaddr = base + kTrOffX, dyaddr = base + kTrOffDY;
  const uint32_t bar_load = smem_addr(sm + kTrOffBar), bar_mma = bar_load + 8;
  unsigned char* H[4] = {sm + kTrOffH, sm + kTrOffH + kHBytes, sm + kTrOffH + 2 * kHBytes, sm + kTrOffH + 3 * kHBytes};
  unsigned char* DY = sm + kTrOffDY;
  const int ntiles = (n + kTile - 1) / kTile;
  const bool bwd = G != nullptr;

  stage_weights(P, sm, aux);
  if (tid == 0) {
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&s_tmem, kTrCols);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t lanes = (uint32_t)(q * 32) << 16;

  // per-thread partial sums: bias gradients of column cn over rows 32*(tid/64)..+31, head
  const int cn = tid & (kHid - 1), rq = tid >> 6;
  float gb[4] = {0.f, 0.f, 0.f, 0.f}, gw5 = 0.f, gb5 = 0.f, lsum = 0.f;
  unsigned lphase = 0, mphase = 0;
  int done_tiles = 0;
  bool ok = true, load_pending = false;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (tid == 0) tma_load_tile(xaddr, &xmap, row0 + tile * kTile, bar_load);
    ok = mbar_wait(bar_load, lphase);
    if (__syncthreads_or(!ok)) {
      ok = false;
      load_pending = true;
      break;
    }
    lphase ^= 1u;
    const int row = tile * kTile + r;
    const bool valid = row < n;
    float h[32];
    // forward: layer l reads X or H[l-1], writes H[l]
    for (int l = 0; l < 4 && ok; ++l) {
      if (tid == 0) {
        tc_fence_after();
        issue_fwd(tmem + kColFwd, l == 0 ? xaddr : smem_addr(H[l - 1]), wbase, l);
        mma_commit(bar_mma);
      }
      ok = mbar_wait(bar_mma, mphase);
      mphase ^= 1u;
      if (__syncthreads_or(!ok)) {
        ok = false;
        break;
      }
      tc_fence_after();
      hidden_epilogue(tmem + kColFwd + lanes, aux + l * kHid, r, c0, h, H[l], l == 3);
      if (l == 3) part[hf * kTile + r] = head_partial(h, aux + 4 * kHid, c0);
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
    }
    if (!ok) break;
    // head, loss, dz; then dY4 = dz * bf16(w5) * (h4 > 0) from the registers of layer 3
    if (hf == 0) {
      float dz = 0.f;
      if (valid) {
        const float t = head_T(aux[5 * kHid], part[r], part[kTile + r]);
        if (T) T[row] = t;
        if (target) {
          const float d = t - target[row];
          lsum += d * d;
          dz = scale * 2.f * d * t * (1.f - t);
        }
      }
      s_dz[r] = dz;
    }
    __syncthreads();
    ++done_tiles;
    if (!bwd) continue;
    {
      const float dz = s_dz[r];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = c * 8 + 2 * j;
          const float a = h[k] > 0.f ? dz * aux[4 * kHid + c0 + k] : 0.f;
          const float b = h[k + 1] > 0.f ? dz * aux[4 * kHid + c0 + k + 1] : 0.f;
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(a, b);
          w[j] = *reinterpret_cast<const uint32_t*>(&b2);
        }
        *reinterpret_cast<uint4*>(DY + ch_off(kTile, r, c0 + c * 8)) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // head gradients: G_w5[k] += sum_b dz[b] h4[b][k], G_b5 += sum_b dz[b]
    for (int b = rq * 32; b < rq * 32 + 32; ++b)
      gw5 = fmaf(s_dz[b], __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(H[3] + ch_off(kTile, b, cn))), gw5);
    if (hf == 0) gb5 += s_dz[r];
    // backward, layer l = 3..0: G_W_l += in_l^T dY_l; dY_{l-1} = (dY_l W_l^T) * (in_l > 0)
    for (int l = 3; l >= 0 && ok; --l) {
      const uint32_t in_addr = l == 0 ? xaddr : smem_addr(H[l - 1]);
      if (tid == 0) {
        tc_fence_after();
        const uint32_t dwg = tmem + kColWg + 64u * (uint32_t)l;
        for (int s = 0; s < kTile / 16; ++s)
          mma(dwg, sdesc(in_addr + s * 256, 128, kTile * 16), sdesc(dyaddr + s * 256, 128, kTile * 16), kIdWgrad,
              (done_tiles > 1 || s > 0) ? 1u : 0u);
        if (l > 0) {
          const uint32_t b = w_addr(wbase, l);
          for (int s = 0; s < kHid / 16; ++s)
            mma(tmem + kColDg, sdesc(dyaddr + s * 2 * kTile * 16, kTile * 16, 128),
                sdesc(b + s * 256, 128, kHid * 16), kIdDgrad, s > 0 ? 1u : 0u);
        }
        mma_commit(bar_mma);
      }
      // bias gradient of layer l: column sums of dY_l (read while the MMAs read it too)
      {
        float s = 0.f;
        for (int b = rq * 32; b < rq * 32 + 32; ++b)
          s += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(DY + ch_off(kTile, b, cn)));
        gb[l] += s;
      }
      ok = mbar_wait(bar_mma, mphase);
      mphase ^= 1u;
      if (__syncthreads_or(!ok)) {
        ok = false;
        break;
      }
      if (l == 0) break;
      tc_fence_after();
      float dx[32];
      tmem_ld32(tmem + kColDg + lanes + c0, dx);
      tmem_wait_ld();
      const unsigned char* in = H[l - 1];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint4 xv = *reinterpret_cast<const uint4*>(in + ch_off(kTile, r, c0 + c * 8));
        const __nv_bfloat16* xb = reinterpret_cast<const __nv_bfloat16*>(&xv);
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = c * 8 + 2 * j;
          const float a = __bfloat162float(xb[2 * j]) > 0.f ? dx[k] : 0.f;
          const float b = __bfloat162float(xb[2 * j + 1]) > 0.f ? dx[k + 1] : 0.f;
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(a, b);
          w[j] = *reinterpret_cast<const uint32_t*>(&b2);
        }
        *reinterpret_cast<uint4*>(DY + ch_off(kTile, r, c0 + c * 8)) = make_uint4(w[0], w[1], w[2], w[3]);
      }
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
    }
    if (!ok) break;
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1u);
    if (load_pending) mbar_wait(bar_load, lphase);  // the tile's load lands here: wait for it (bounded)
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // flush: weight gradients from TMEM (row m of the layer-l accumulator = input m)
  if (ok && bwd && done_tiles > 0) {
    const int oW[4] = {oW1, oW2, oW3, oW4}, Ks[4] = {kIn, kHid, kHid, kHid}, oB[4] = {oB1, oB2, oB3, oB4};
    for (int l = 0; l < 4; ++l) {
      float v[32];
      tmem_ld32(tmem + kColWg + 64u * (uint32_t)l + lanes + c0, v);
      tmem_wait_ld();
      if (r < Ks[l]) {
        float* g = G + oW[l] + r * kHid + c0;
#pragma unroll
        for (int j = 0; j < 32; ++j) atomicAdd(g + j, v[j]);
      }
      atomicAdd(G + oB[l] + cn, gb[l]);
    }
    atomicAdd(G + oW5 + cn, gw5);
  }
  if (ok && done_tiles > 0) {
    float a = lsum, b = gb5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((tid & 31) == 0) {
      if (loss && target) atomicAdd(loss, a);
      if (bwd) atomicAdd(G + oB5, b);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTrCols);
  }
}

// ---------------------------------------------------------------------------
// host: tensor maps and launches
// ---------------------------------------------------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

cudaError_t encode_fn(EncodeTiled* fn) {
  static EncodeTiled cached = nullptr;
  if (!cached) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !p) return cudaErrorNotSupported;
    cached = (EncodeTiled)p;
  }
  *fn = cached;
  return cudaSuccess;
}

// Tensor map of an n x 112 bfloat16 feature matrix (rows 224 bytes apart), box
// {8 columns, 128 rows}; rows past n read as zeros.
cudaError_t feature_map(const __nv_bfloat16* X, int n, CUtensorMap* map) {
  if (((uintptr_t)X & 15) != 0) return cudaErrorMisalignedAddress;
  EncodeTiled fn;
  cudaError_t e = encode_fn(&fn);
  if (e != cudaSuccess) return e;
  const cuuint64_t dims[2] = {(cuuint64_t)kIn, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)kIn * 2};
  const cuuint32_t box[2] = {8, (cuuint32_t)kTile};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)X, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

}  // namespace
}  // namespace mlp

cudaError_t mlp_forward_tc_features(const __nv_bfloat16* X, int n, const float* P, float* T, unsigned* err,
                                    cudaStream_t st) {
  using namespace mlp;
  if (n <= 0) return cudaSuccess;
  CUtensorMap map;
  cudaError_t e = feature_map(X, n, &map);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_mlp_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem + 1024);
  if (e != cudaSuccess) return e;
  const int tiles = (n + kTile - 1) / kTile;
  int grid = sm_count();
  if (grid > (tiles + kPipes - 1) / kPipes) grid = (tiles + kPipes - 1) / kPipes;
  k_mlp_fwd_tc<<<grid, kFwdThreads, kFwdSmem + 1024, st>>>(map, 0, n, P, T, err);
  return cudaGetLastError();
}

cudaError_t mlp_train_step_tc(const float* P, float* G, const __nv_bfloat16* X, const float* target, int n,
                              float scale, float* T, float* loss, unsigned* err, cudaStream_t st) {
  using namespace mlp;
  if (n <= 0) return cudaSuccess;
  CUtensorMap map;
  cudaError_t e = feature_map(X, n, &map);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrSmem + 1024);
  if (e != cudaSuccess) return e;
  const int tiles = (n + kTile - 1) / kTile;
  int grid = sm_count();
  if (grid > tiles) grid = tiles;
  k_mlp_train_tc<<<grid, kThreads, kTrSmem + 1024, st>>>(map, 0, n, P, target, scale, G, T, loss, err);
  return cudaGetLastError();
}

}  // namespace beams
