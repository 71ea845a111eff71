// k_mlp_tc.cu — the transmittance network's forward pass on the 5th-generation
// tensor cores (tcgen05): a dense GEMM chain over 128-row tiles.
//
// One CTA of 128 threads owns a 128 x 64 float32 accumulator in tensor memory
// (TMEM, 64 columns allocated once per CTA). Per tile:
//   1. each thread writes its row's 112 bfloat16 features into shared memory in
//      the canonical K-major no-swizzle layout (8-row x 16-byte core matrices);
//   2. one thread issues the layer's tcgen05.mma (M = 128, N = 64, K = 16 per
//      instruction, A and B from shared memory, D in TMEM) and commits them to
//      an mbarrier; everyone waits on it (bounded);
//   3. each warp reads its 32 TMEM lanes (= its 32 rows) with tcgen05.ld, adds
//      the bias, applies ReLU, rounds to bfloat16 and writes the row back to
//      shared memory as the next layer's A (and, for training, to global memory);
//   4. after the 4th hidden layer the head (64-wide dot product, sigmoid) runs
//      on the CUDA cores.
// The weights stay in shared memory (bfloat16, the same layout, as B = W^T:
// K-major N x K) for all tiles. Numerics as the CUDA-core kernels: bfloat16
// operands, float32 accumulation (in the tensor core's order).
//
// Shared-memory layout of an R-row, K-column bfloat16 operand (R = 128 for A,
// 64 for B): K is cut into 16-wide slices; slice s occupies R * 32 bytes at
// s * R * 32; inside it, element (r, k) sits at (r / 8) * 256 + ((k % 16) / 8)
// * 128 + (r % 8) * 16 + (k % 8) * 2. The descriptor of slice s: start =
// base + s * R * 32, leading byte offset 128 (the two 8-wide K halves), stride
// byte offset 256 (consecutive 8-row groups), layout SWIZZLE_NONE, version 1.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "mlp_common.cuh"
#include "mlp_host.h"

namespace beams {
namespace mlp {
namespace {

constexpr int kTile = 128;                          // rows per tile (tcgen05 M)
constexpr int kTcThreads = 128;                     // one thread per row
constexpr int kA_bytes = kTile * kIn * 2;           // 28672
constexpr int kB1_bytes = kHid * kIn * 2;           // 14336
constexpr int kBh_bytes = kHid * kHid * 2;          // 8192
constexpr int kOffB1 = kA_bytes;
constexpr int kOffB2 = kOffB1 + kB1_bytes;
constexpr int kOffAux = kOffB2 + 3 * kBh_bytes;     // 67584: biases (4 x 64), w5 (64), b5
constexpr int kAuxFloats = 4 * kHid + kHid + 1;
constexpr int kOffBar = ((kOffAux + kAuxFloats * 4 + 15) / 16) * 16;
constexpr int kSmemTc = kOffBar + 16;
constexpr unsigned kWaitLimit = 1u << 24;           // mbarrier polls before giving up

// Offset (bytes) of element (r, k) in an R-row operand.
__host__ __device__ constexpr int op_off(int R, int r, int k) {
  return (k >> 4) * R * 32 + (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (no swizzle, K-major, LBO 128 B, SBO 256 B).
__device__ __forceinline__ uint64_t op_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFFu) >> 4);          // start address, bits [0, 14)
  d |= (uint64_t)(128u >> 4) << 16;                 // leading byte offset, bits [16, 30)
  d |= (uint64_t)(256u >> 4) << 32;                 // stride byte offset, bits [32, 46)
  d |= (uint64_t)1 << 46;                           // version 1 (tcgen05)
  return d;                                         // base offset 0, lbo mode 0, SWIZZLE_NONE
}

// Instruction descriptor: D float32, A and B bfloat16, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kHid >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Waits for the phase to complete; false if the poll budget ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned phase) {
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Row input: precomputed features (training, tests) or positions to encode (rendering).
struct RowsFromFeatures {
  const __nv_bfloat16* X;  // n x 112
  __device__ __forceinline__ void load(int row, unsigned char* A, int r) const {
    const uint4* src = reinterpret_cast<const uint4*>(X + (size_t)row * kIn);
#pragma unroll
    for (int c = 0; c < kIn / 8; ++c) *reinterpret_cast<uint4*>(A + op_off(kTile, r, c * 8)) = src[c];
  }
};

struct RowsFromPositions {
  const float4* pos;       // n x {x, y, z, -}
  Encoding enc;
  float lf[3];
  __device__ __forceinline__ void load(int row, unsigned char* A, int r) const {
    const float4 q = pos[row];
    const float p[3] = {q.x, q.y, q.z};
    float u[3];
    normalised(enc, p, u);
#pragma unroll 1
    for (int c = 0; c < kIn; c += 8) {
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float a, b;
        feature_pair(u, lf, c + 2 * j, a, b);
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        w[j] = *reinterpret_cast<const uint32_t*>(&h);
      }
      *reinterpret_cast<uint4*>(A + op_off(kTile, r, c)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
};

template <typename Rows>
__global__ void __launch_bounds__(kTcThreads) k_mlp_fwd_tc(Rows rows, int n, const float* __restrict__ P,
                                                           __nv_bfloat16* __restrict__ H0,
                                                           __nv_bfloat16* __restrict__ H1,
                                                           __nv_bfloat16* __restrict__ H2,
                                                           __nv_bfloat16* __restrict__ H3, float* __restrict__ T,
                                                           unsigned* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* A = sm;
  float* aux = reinterpret_cast<float*>(sm + kOffAux);
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t bar = smem_addr(sm + kOffBar);

  // weights as B = W^T (N x K, K-major), bfloat16-rounded as every forward does
  for (int i = tid; i < kIn * kHid; i += kTcThreads) {
    const int k = i / kHid, nn = i - k * kHid;  // W1[k][n] at P[oW1 + k * 64 + n]
    *reinterpret_cast<__nv_bfloat16*>(sm + kOffB1 + op_off(kHid, nn, k)) = __float2bfloat16_rn(P[oW1 + i]);
  }
  const int oW[3] = {oW2, oW3, oW4};
  for (int l = 0; l < 3; ++l)
    for (int i = tid; i < kHid * kHid; i += kTcThreads) {
      const int k = i / kHid, nn = i - k * kHid;
      *reinterpret_cast<__nv_bfloat16*>(sm + kOffB2 + l * kBh_bytes + op_off(kHid, nn, k)) =
          __float2bfloat16_rn(P[oW[l] + i]);
    }
  const int oB[4] = {oB1, oB2, oB3, oB4};
  for (int i = tid; i < 4 * kHid; i += kTcThreads) aux[i] = P[oB[i / kHid] + (i % kHid)];
  for (int i = tid; i < kHid; i += kTcThreads) aux[4 * kHid + i] = bf16r(P[oW5 + i]);
  if (tid == 0) {
    aux[5 * kHid] = P[oB5];
    mbar_init(bar, 1);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                 "r"(64u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();  // the weights were written by ordinary stores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  unsigned phase = 0;
  bool ok = true;

  for (int tile = blockIdx.x; ok && tile * kTile < n; tile += gridDim.x) {
    const int row = tile * kTile + tid;
    if (row < n) {
      rows.load(row, A, tid);
    } else {
#pragma unroll 1
      for (int c = 0; c < kIn; c += 8) *reinterpret_cast<uint4*>(A + op_off(kTile, tid, c)) = make_uint4(0, 0, 0, 0);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    for (int l = 0; l < 4; ++l) {
      const int K = l == 0 ? kIn : kHid;
      const uint32_t bbase = smem_addr(sm + (l == 0 ? kOffB1 : kOffB2 + (l - 1) * kBh_bytes));
      if (tid == 0) {
        tc_fence_after();
        const uint32_t abase = smem_addr(A);
        for (int s = 0; s < K / 16; ++s)
          mma_bf16(tmem, op_desc(abase + s * kTile * 32), op_desc(bbase + s * kHid * 32), s > 0 ? 1u : 0u);
        mma_commit(bar);
      }
      const bool done = mbar_wait(bar, phase);
      if (__syncthreads_or(!done)) {  // a uniform decision: every thread leaves together
        ok = false;
        if (tid == 0) atomicExch(err, 1u);
        break;
      }
      phase ^= 1u;
      tc_fence_after();
      float h[kHid];
#pragma unroll
      for (int c = 0; c < kHid; c += 16) tmem_ld16(tmem_row + c, h + c);
      tmem_wait_ld();
      const float* bias = aux + l * kHid;
#pragma unroll
      for (int j = 0; j < kHid; ++j) h[j] = bf16r(fmaxf(h[j] + bias[j], 0.f));
      __nv_bfloat16* Hout = l == 0 ? H0 : (l == 1 ? H1 : (l == 2 ? H2 : H3));
      if (Hout && row < n) {
        uint4* dst = reinterpret_cast<uint4*>(Hout + (size_t)row * kHid);
#pragma unroll
        for (int c = 0; c < kHid / 8; ++c) {
          uint32_t w[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(h[c * 8 + 2 * j], h[c * 8 + 2 * j + 1]);
            w[j] = *reinterpret_cast<const uint32_t*>(&b2);
          }
          dst[c] = make_uint4(w[0], w[1], w[2], w[3]);
        }
      }
      if (l < 3) {
        // this row as the next layer's A (the MMAs that read A have completed)
#pragma unroll
        for (int c = 0; c < kHid / 8; ++c) {
          uint32_t w[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(h[c * 8 + 2 * j], h[c * 8 + 2 * j + 1]);
            w[j] = *reinterpret_cast<const uint32_t*>(&b2);
          }
          *reinterpret_cast<uint4*>(A + op_off(kTile, tid, c * 8)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        fence_async_smem();
      } else if (T && row < n) {
        float z = aux[5 * kHid];
        for (int j = 0; j < kHid; ++j) z = fmaf(h[j], aux[4 * kHid + j], z);
        T[row] = 1.f / (1.f + expf(-z));
      }
      tc_fence_before();
      __syncthreads();
    }
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64u) : "memory");
  }
}

template <typename Rows>
cudaError_t launch_fwd_tc(const Rows& rows, int n, const float* P, __nv_bfloat16* const H[4], float* T,
                          unsigned* err, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_mlp_fwd_tc<Rows>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTc);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_fwd_tc<Rows>, kTcThreads, kSmemTc);
  if (e != cudaSuccess) return e;
  const int tiles = (n + kTile - 1) / kTile;
  int grid = sms * (per_sm > 0 ? per_sm : 1);
  if (grid > tiles) grid = tiles;
  k_mlp_fwd_tc<Rows><<<grid, kTcThreads, kSmemTc, st>>>(rows, n, P, H ? H[0] : nullptr, H ? H[1] : nullptr,
                                                        H ? H[2] : nullptr, H ? H[3] : nullptr, T, err);
  return cudaGetLastError();
}

}  // namespace
}  // namespace mlp

cudaError_t mlp_forward_tc_features(const __nv_bfloat16* X, int n, const float* P, __nv_bfloat16* const H[4],
                                    float* T, unsigned* err, cudaStream_t st) {
  return mlp::launch_fwd_tc(mlp::RowsFromFeatures{X}, n, P, H, T, err, st);
}

cudaError_t mlp_forward_tc_positions(const float4* pos, const mlp::Encoding& enc, const float lf[3], int n,
                                     const float* P, float* T, unsigned* err, cudaStream_t st) {
  mlp::RowsFromPositions rows{pos, enc, {lf[0], lf[1], lf[2]}};
  return mlp::launch_fwd_tc(rows, n, P, nullptr, T, err, st);
}

}  // namespace beams
