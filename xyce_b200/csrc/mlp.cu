// Tensor-core kernels of the learned surrogate (include/xyce_surrogate.h): a BF16 GEMM on the
// 5th-generation tensor cores (tcgen05.mma, FP32 accumulator in tensor memory) with the fused
// epilogues the surrogate's forward and backward passes need, and the small kernels around it
// (loss gradient, bias gradient, split-K reduction, Adam).
//
// GEMM: C[M x N] = A[M x K] * B[N x K]^T, A and B row-major BF16 with K contiguous (K-major
// operands), M a multiple of 128, N = 16 or 128 per tile, K a multiple of 16. One CTA of 128
// threads computes one 128 x N tile over a K range (the whole K, or one split-K slice):
//   * warp 0 allocates N tensor-memory columns (lane m <-> row m of the tile);
//   * per K chunk of 64, all threads copy the A and B sub-tiles from global memory into shared
//     memory in the tensor core's no-swizzle K-major layout (8-row x 16-byte core matrices;
//     consecutive K core matrices 128 B apart, consecutive 8-row groups 1024 B apart);
//   * after a proxy fence and a barrier, one thread issues 4 tcgen05.mma (K = 16 each) and a
//     tcgen05.commit to an mbarrier; every thread waits on it (bounded) before the next chunk
//     overwrites shared memory;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w reads lanes 32w..32w+31, so
//     thread t owns row 32w + t), applies the fused operation and writes global memory.
// Every wait on the mbarrier has an iteration limit; on expiry the kernel records an error code
// in a device flag, stops issuing work, waits (again bounded) for its own in-flight MMA, frees
// its tensor memory and returns, so the context stays usable and the host reports the failure.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/xyce_surrogate.h"

int xd_internal_fail(int code, const std::string &msg);

namespace {

constexpr int kThreads = 128;
constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr long long kSpinLimit = 20000000;  // mbarrier polls before a wait is declared failed

// ---- tcgen05 / mbarrier primitives (inline PTX) ------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Returns true once the barrier's phase `parity` has completed, false after kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor: no swizzle, K-major canonical layout. Fields (bit ranges):
// start address >> 4 [0,14), leading-dimension byte offset >> 4 [16,30) (distance between core
// matrices adjacent in K), stride-dimension byte offset >> 4 [32,46) (distance between 8-row
// groups), descriptor version 1 [46,48), base offset 0, layout type 0 (no swizzle) [61,64).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16: D format F32 [4,6) = 1, A format BF16 [7,10) = 1, B format
// BF16 [10,13) = 1, both K-major (bits 15, 16 = 0), N >> 3 at [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread t of the warp receives lane (base lane + t).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- epilogues -------------------------------------------------------------------------------

// SiLU and its derivative with the fast exponential and approximate division: the surrogate is
// not held to bit parity with a CPU (its outputs only seed Newton iterations).
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Byte offset of element (row r, column k) of a rows x kChunkK bf16 tile in the no-swizzle
// K-major layout: 8 x 8 core matrices of 128 B, K-adjacent ones 128 B apart, row groups 1024 B.
__device__ __forceinline__ uint32_t tile_off(int r, int kc) {
  return (uint32_t)((r >> 3) * 1024 + kc * 128 + (r & 7) * 16);
}

template <int TN>
__global__ void __launch_bounds__(kThreads) gemm_bf16_tc_kernel(xd_gemm_args g, int k_per_split) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // Layout: [A tile 128 x 64 bf16 = 16 KB][B tile TN x 64 bf16][mbarrier][tmem address]
  unsigned char *sA = smem_raw;
  unsigned char *sB = smem_raw + kTileM * kChunkK * 2;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sB + TN * kChunkK * 2);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int m0 = blockIdx.x * kTileM;
  const int n0 = blockIdx.y * TN;
  const int split = blockIdx.z;
  const int k_begin = split * k_per_split;
  int k_end = k_begin + k_per_split;
  if (k_end > g.K) k_end = g.K;
  constexpr uint32_t kCols = TN < 32 ? 32 : TN;  // allocation granularity is 32 columns

  if (warp == 0) tmem_alloc(tmem_slot, kCols);
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = instr_desc_bf16(kTileM, TN);
  const __nv_bfloat16 *A = static_cast<const __nv_bfloat16 *>(g.A);
  const __nv_bfloat16 *B = static_cast<const __nv_bfloat16 *>(g.B);
  __nv_bfloat16 *Zo = static_cast<__nv_bfloat16 *>(g.Z);
  __nv_bfloat16 *Ho = static_cast<__nv_bfloat16 *>(g.H);
  __nv_bfloat16 *HTo = static_cast<__nv_bfloat16 *>(g.HT);
  const __nv_bfloat16 *Zi = static_cast<const __nv_bfloat16 *>(g.Zin);

  uint32_t phase = 0;
  bool ok = true;
  int issued = 0;
  for (int k0 = k_begin; k0 < k_end && ok; k0 += kChunkK) {
    const int kc_n = min(kChunkK, k_end - k0) / 8;  // 8-element K chunks in this step (2, 4, 6 or 8)
    // Copy A (128 rows) and B (TN rows) sub-tiles: one 16-byte core-matrix row per copy.
    for (int i = tid; i < kTileM * kc_n; i += kThreads) {
      const int r = i / kc_n, kc = i % kc_n;
      const int gr = m0 + r;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gr < g.M) v = *reinterpret_cast<const uint4 *>(A + (size_t)gr * g.lda + k0 + kc * 8);
      *reinterpret_cast<uint4 *>(sA + tile_off(r, kc)) = v;
    }
    for (int i = tid; i < TN * kc_n; i += kThreads) {
      const int r = i / kc_n, kc = i % kc_n;
      const int gr = n0 + r;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gr < g.N) v = *reinterpret_cast<const uint4 *>(B + (size_t)gr * g.ldb + k0 + kc * 8);
      *reinterpret_cast<uint4 *>(sB + tile_off(r, kc)) = v;
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
      for (int s = 0; s < kc_n / 2; ++s) {
        const uint64_t ad = smem_desc(a0 + s * 256, 128, 1024);
        const uint64_t bd = smem_desc(b0 + s * 256, 128, 1024);
        mma_bf16(tmem, ad, bd, idesc, (issued > 0 || s > 0) ? 1u : 0u);
      }
      mma_commit(bar);
    }
    ++issued;
    ok = __syncthreads_and(mbar_wait(bar, phase)) != 0;  // uniform across the CTA
    phase ^= 1u;
    tc_fence_after();
  }
  if (!ok) {
    // A wait expired: record it and drain (bounded) before releasing tensor memory.
    if (tid == 0) atomicExch(g.err, 1);
    mbar_wait(bar, phase ^ 1u);
  }
  // Epilogue: thread t of warp w owns tile row 32w + t (tensor-memory lane 32w + t).
  const int row = m0 + warp * 32 + (tid & 31);
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  if (ok && issued > 0) {
#pragma unroll
    for (int c0 = 0; c0 < TN; c0 += (TN >= 32 ? 32 : 16)) {
      float v[32];
      if constexpr (TN >= 32) {
        tmem_ld32(lane_base + c0, v);
      } else {
        float w16[16];
        tmem_ld16(lane_base + c0, w16);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = w16[i];
      }
      constexpr int W = TN >= 32 ? 32 : 16;
      if (row < g.M) {
#pragma unroll
        for (int i = 0; i < W; ++i) {
          const int n = n0 + c0 + i;
          if (n >= g.N) continue;
          float acc = v[i];
          switch (g.epilogue) {
            case XD_EPI_F32: {
              g.C32[(size_t)split * g.M * g.ldc + (size_t)row * g.ldc + n] = acc;
              break;
            }
            case XD_EPI_BIAS_F32: {
              g.C32[(size_t)row * g.ldc + n] = acc + g.bias[n];
              break;
            }
            case XD_EPI_BIAS_SILU: {
              const float z = acc + g.bias[n];
              const float h = silu(z);
              Zo[(size_t)row * g.ldc + n] = __float2bfloat16(z);
              Ho[(size_t)row * g.ldc + n] = __float2bfloat16(h);
              if (HTo) HTo[(size_t)n * g.ldt + row] = __float2bfloat16(h);
              break;
            }
            case XD_EPI_SILU_BACK: {
              const float z = __bfloat162float(Zi[(size_t)row * g.ldc + n]);
              const float d = acc * silu_grad(z);
              Ho[(size_t)row * g.ldc + n] = __float2bfloat16(d);
              if (HTo) HTo[(size_t)n * g.ldt + row] = __float2bfloat16(d);
              break;
            }
            default:
              break;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_free(tmem, kCols);
}

// ---- small kernels ---------------------------------------------------------------------------

// Mean-squared-error gradient of the network output (fp32 [M x ld]) against targets, written as
// BF16 in both layouts for the backward GEMMs, and the per-sample squared error.
__global__ void mse_grad_kernel(int M, int n_out, int ld, const float *__restrict__ y, const float *__restrict__ t,
                                float scale, __nv_bfloat16 *__restrict__ dz, __nv_bfloat16 *__restrict__ dzt,
                                int ldt, float *__restrict__ sq) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= M) return;
  float s = 0.0f;
  for (int n = 0; n < ld; ++n) {
    float d = 0.0f;
    if (n < n_out) {
      const float e = y[(size_t)row * ld + n] - t[(size_t)row * n_out + n];
      s += e * e;
      d = scale * e;
    }
    dz[(size_t)row * ld + n] = __float2bfloat16(d);
    dzt[(size_t)n * ldt + row] = __float2bfloat16(d);
  }
  if (sq) sq[row] = s;
}

// out[n] = sum over `count` rows of in[r * ld + n], one block per column, fixed reduction tree.
__global__ void column_sum_kernel(int rows, int cols, const float *__restrict__ in, int ld, float *__restrict__ out) {
  __shared__ float red[256];
  const int n = blockIdx.x;
  float acc = 0.0f;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) acc += in[(size_t)r * ld + n];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0 && n < cols) out[n] = red[0];
}

// Bias gradient: sum over the batch of the transposed BF16 gradient rows dzt[n][0..M).
__global__ void bias_grad_kernel(int M, int N, const __nv_bfloat16 *__restrict__ dzt, int ldt,
                                 float *__restrict__ db) {
  __shared__ float red[256];
  const int n = blockIdx.x;
  float acc = 0.0f;
  for (int r = threadIdx.x; r < M; r += blockDim.x) acc += __bfloat162float(dzt[(size_t)n * ldt + r]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0 && n < N) db[n] = red[0];
}

// Sums split-K partials part[s][i] for s = 0..splits-1 in order.
__global__ void splitk_sum_kernel(int n, int splits, const float *__restrict__ part, float *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float acc = 0.0f;
  for (int s = 0; s < splits; ++s) acc += part[(size_t)s * n + i];
  out[i] = acc;
}

// Adam on FP32 master parameters; refreshes the BF16 copies (row-major and, for matrices, the
// transpose used by the backward GEMM).
__global__ void adam_kernel(int rows, int cols, float *__restrict__ p, const float *__restrict__ grad,
                            float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2, float eps,
                            float c1, float c2, __nv_bfloat16 *__restrict__ p16, __nv_bfloat16 *__restrict__ p16t,
                            int ld16, int ld16t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const float gr = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gr;
  const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (p16) p16[(size_t)r * ld16 + c] = __float2bfloat16(pi);
  if (p16t) p16t[(size_t)c * ld16t + r] = __float2bfloat16(pi);
}

// First layer in FP32 on the CUDA cores: the network inputs (biases in volts, log-geometry) keep
// full precision, which BF16 (8-bit mantissa, ~4 mV at 1 V) would not give them. One thread per
// (sample, hidden unit): z = W1[u] . x + b1[u]; writes Z, H = silu(z) (BF16) and H transposed.
__global__ void input_layer_kernel(int M, int n_in, int n_hid, const float *__restrict__ x, int ldx,
                                   const float *__restrict__ w1, int ldw, const float *__restrict__ b1,
                                   __nv_bfloat16 *__restrict__ Z, __nv_bfloat16 *__restrict__ H,
                                   __nv_bfloat16 *__restrict__ HT, int ldt) {
  const int u = threadIdx.x;  // hidden unit
  const int row = blockIdx.x;
  if (u >= n_hid || row >= M) return;
  float z = b1[u];
  for (int i = 0; i < n_in; ++i) z += w1[u * ldw + i] * x[(size_t)row * ldx + i];
  const float h = silu(z);
  Z[(size_t)row * n_hid + u] = __float2bfloat16(z);
  H[(size_t)row * n_hid + u] = __float2bfloat16(h);
  if (HT) HT[(size_t)u * ldt + row] = __float2bfloat16(h);
}

// First-layer weight gradient in FP32: gw[u][i] = sum_r dzt[u][r] * x[r][i] for i < n_in, one
// block per hidden unit, fixed reduction tree.
__global__ void input_grad_kernel(int M, int n_in, const __nv_bfloat16 *__restrict__ dzt, int ldt,
                                  const float *__restrict__ x, int ldx, float *__restrict__ gw, int ldw) {
  __shared__ float red[8][256];
  const int u = blockIdx.x;
  float acc[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i] = 0.0f;
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    const float d = __bfloat162float(dzt[(size_t)u * ldt + r]);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (i < n_in) acc[i] += d * x[(size_t)r * ldx + i];
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) red[i][threadIdx.x] = acc[i];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int i = 0; i < 8; ++i) red[i][threadIdx.x] += red[i][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x < n_in) gw[u * ldw + threadIdx.x] = red[threadIdx.x][0];
}

// Surrogate inputs for circuit instances idx[k]: terminal voltages from the solution (ground ->
// 0), differences to the source, scaled by 1 / vmax, then the instance's scaled log W and log L.
__global__ void surrogate_features_kernel(int n, const int *__restrict__ idx, const int *__restrict__ nodes4,
                                          const double *__restrict__ sol, const float *__restrict__ geom2,
                                          float inv_vmax, float *__restrict__ x, int ldx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = idx[k];
  double v[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int nd = nodes4[4 * i + t];
    v[t] = nd >= 0 ? sol[nd] : 0.0;
  }
  x[(size_t)k * ldx + 0] = (float)((v[1] - v[2]) * inv_vmax);  // Vgs
  x[(size_t)k * ldx + 1] = (float)((v[0] - v[2]) * inv_vmax);  // Vds
  x[(size_t)k * ldx + 2] = (float)((v[3] - v[2]) * inv_vmax);  // Vbs
  x[(size_t)k * ldx + 3] = geom2[2 * i];
  x[(size_t)k * ldx + 4] = geom2[2 * i + 1];
}

// Decodes the surrogate's outputs y = asinh(value / scale) for instances idx[k] and stages the
// terminal currents and charges in the exact load's slot layout (slot-major, 16 x n_inst):
// F = (Id, 0, -Id, 0) at (D, G, S, B), Q = (Qd, Qg, -(Qg + Qd + Qb), Qb), limiter slots zero.
__global__ void surrogate_stage_kernel(int n, const int *__restrict__ idx, const float *__restrict__ y, int ldy,
                                       const float *__restrict__ out_scale, int n_inst, double *__restrict__ stage) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = idx[k];
  const float *yr = y + (size_t)k * ldy;
  const double id = sinh((double)yr[0]) * out_scale[0];
  const double qg = sinh((double)yr[1]) * out_scale[1];
  const double qd = sinh((double)yr[2]) * out_scale[2];
  const double qb = sinh((double)yr[3]) * out_scale[3];
  const size_t N = (size_t)n_inst;
  stage[0 * N + i] = id;
  stage[1 * N + i] = 0.0;
  stage[2 * N + i] = -id;
  stage[3 * N + i] = 0.0;
  stage[4 * N + i] = qd;
  stage[5 * N + i] = qg;
  stage[6 * N + i] = -(qg + qd + qb);
  stage[7 * N + i] = qb;
#pragma unroll
  for (int s = 8; s < 16; ++s) stage[s * N + i] = 0.0;
}

// ---- fused inference: the whole 5 -> 128 -> 128 -> 128 -> 128 -> 16 network in one kernel -----

constexpr int kFusedThreads = 256;  // 8 warps: two per tensor-memory lane quarter
constexpr int kHid = 128;
constexpr int kOutPad = 16;
// Shared-memory layout of a 128-row x 128-K BF16 operand: 8 x 8 core matrices, K-adjacent ones
// 128 B apart, 8-row groups 2048 B apart.
__device__ __forceinline__ uint32_t off128(int r, int kc) {
  return (uint32_t)((r >> 3) * 2048 + kc * 128 + (r & 7) * 16);
}

struct FusedSmem {
  unsigned char w[3][kHid * kHid * 2];   // hidden layers 2..4, [out][in] K-major
  unsigned char w5[kOutPad * kHid * 2];  // output layer, 16 x 128
  unsigned char act[kHid * kHid * 2];    // activation tile (A operand), 128 x 128
  float w1[kHid * 8];                    // first layer, FP32, 128 x n_in (n_in <= 8)
  float b[4 * kHid + kOutPad];           // biases of layers 1..5
  uint64_t bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kFusedThreads, 1) mlp_forward_fused_kernel(xd_mlp_net net, int n, const float *x,
                                                                            int ldx, float *y, int ldy, int *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  FusedSmem &S = *reinterpret_cast<FusedSmem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // Stage the weights once per CTA.
  for (int l = 0; l < 3; ++l) {
    const __nv_bfloat16 *W = static_cast<const __nv_bfloat16 *>(net.w[l]);
    for (int i = tid; i < kHid * 16; i += kFusedThreads) {
      const int r = i >> 4, kc = i & 15;
      *reinterpret_cast<uint4 *>(S.w[l] + off128(r, kc)) =
          *reinterpret_cast<const uint4 *>(W + (size_t)r * kHid + kc * 8);
    }
  }
  {
    const __nv_bfloat16 *W = static_cast<const __nv_bfloat16 *>(net.w5);
    for (int i = tid; i < kOutPad * 16; i += kFusedThreads) {
      const int r = i >> 4, kc = i & 15;
      *reinterpret_cast<uint4 *>(S.w5 + off128(r, kc)) = *reinterpret_cast<const uint4 *>(W + (size_t)r * kHid + kc * 8);
    }
  }
  for (int i = tid; i < kHid * net.n_in; i += kFusedThreads) S.w1[(i / net.n_in) * 8 + i % net.n_in] =
      net.w1[(i / net.n_in) * net.ldw1 + i % net.n_in];
  for (int i = tid; i < 4 * kHid + kOutPad; i += kFusedThreads) {
    const int l = i / kHid, u = i % kHid;
    S.b[i] = (l < 4) ? net.b[l][u] : net.b[4][i - 4 * kHid];
  }
  if (warp == 0) tmem_alloc(&S.tmem, kHid);
  if (tid == 0) {
    mbar_init(&S.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t idesc_h = instr_desc_bf16(kTileM, kHid);
  const uint32_t idesc_o = instr_desc_bf16(kTileM, kOutPad);
  const uint32_t act_a = smem_u32(S.act);
  const int quarter = warp & 3;           // tensor-memory lanes 32q .. 32q + 31
  const int half = warp >> 2;             // columns [64 half, 64 half + 64)
  const int row = quarter * 32 + lane;    // the tile row this thread owns in the epilogues
  const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  const int tiles = (n + kTileM - 1) / kTileM;
  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const int g = tile * kTileM + row;
    // Layer 1 on the CUDA cores (FP32): this thread's 64 hidden units of its row.
    {
      float xi[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) xi[i] = (i < net.n_in && g < n) ? x[(size_t)g * ldx + i] : 0.0f;
      for (int c8 = 0; c8 < 8; ++c8) {
        __align__(16) __nv_bfloat16 h8[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int u = half * 64 + c8 * 8 + j;
          float z = S.b[u];
          for (int i = 0; i < net.n_in; ++i) z += S.w1[u * 8 + i] * xi[i];
          h8[j] = __float2bfloat16(g < n ? silu(z) : 0.0f);
        }
        *reinterpret_cast<uint4 *>(S.act + off128(row, half * 8 + c8)) = *reinterpret_cast<uint4 *>(h8);
      }
    }
    // Layers 2..5 on the tensor cores.
    for (int l = 0; l < 4 && ok; ++l) {
      fence_proxy_async_smem();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      const bool last = (l == 3);
      if (tid == 0) {
        const uint32_t wb = last ? smem_u32(S.w5) : smem_u32(S.w[l]);
        for (int s = 0; s < 8; ++s)
          mma_bf16(tmem, smem_desc(act_a + s * 256, 128, 2048), smem_desc(wb + s * 256, 128, 2048),
                   last ? idesc_o : idesc_h, s > 0 ? 1u : 0u);
        mma_commit(&S.bar);
      }
      ok = __syncthreads_and(mbar_wait(&S.bar, phase)) != 0;
      phase ^= 1u;
      tc_fence_after();
      if (!ok) break;
      if (!last) {
        // Epilogue: bias + SiLU, written back as the next layer's operand.
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 32) {
          float v[32];
          tmem_ld32(lane_base + half * 64 + c0, v);
#pragma unroll
          for (int c8 = 0; c8 < 4; ++c8) {
            __align__(16) __nv_bfloat16 h8[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int u = half * 64 + c0 + c8 * 8 + j;
              h8[j] = __float2bfloat16(silu(v[c8 * 8 + j] + S.b[(l + 1) * kHid + u]));
            }
            *reinterpret_cast<uint4 *>(S.act + off128(row, (half * 64 + c0) / 8 + c8)) =
                *reinterpret_cast<uint4 *>(h8);
          }
        }
      } else if (half == 0) {
        float v[16];
        tmem_ld16(lane_base, v);
        if (g < n) {
#pragma unroll
          for (int j = 0; j < kOutPad; ++j) y[(size_t)g * ldy + j] = v[j] + S.b[4 * kHid + j];
        }
      }
      tc_fence_before();
    }
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    mbar_wait(&S.bar, phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_free(tmem, kHid);
}

int cuda_err(cudaError_t e, const char *where) {
  return xd_internal_fail(-3, std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int xd_gemm_bf16(const xd_gemm_args *g, int splits, void *stream) {
  if (!g || !g->A || !g->B || !g->err) return xd_internal_fail(-1, "null GEMM argument");
  if (g->M <= 0 || g->N <= 0 || g->K <= 0 || (g->K % 16) != 0 || (g->lda % 8) != 0 || (g->ldb % 8) != 0)
    return xd_internal_fail(-1, "GEMM needs K and the leading dimensions to be multiples of 16 / 8");
  if ((reinterpret_cast<uintptr_t>(g->A) | reinterpret_cast<uintptr_t>(g->B)) & 15)
    return xd_internal_fail(-1, "GEMM operands must be 16-byte aligned");
  if (g->tile_n != 16 && g->tile_n != 128) return xd_internal_fail(-1, "GEMM tile_n must be 16 or 128");
  if (splits < 1) splits = 1;
  if (splits > 1 && g->epilogue != XD_EPI_F32) return xd_internal_fail(-1, "split-K needs the plain F32 epilogue");
  int k_per = (g->K + splits - 1) / splits;
  k_per = (k_per + kChunkK - 1) / kChunkK * kChunkK;
  const int used = (g->K + k_per - 1) / k_per;
  dim3 grid((g->M + kTileM - 1) / kTileM, (g->N + g->tile_n - 1) / g->tile_n, used);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = (size_t)kTileM * kChunkK * 2 + (size_t)g->tile_n * kChunkK * 2 + 16;
  if (g->tile_n == 128) {
    cudaFuncSetAttribute(gemm_bf16_tc_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    gemm_bf16_tc_kernel<128><<<grid, kThreads, smem, st>>>(*g, k_per);
  } else {
    gemm_bf16_tc_kernel<16><<<grid, kThreads, smem, st>>>(*g, k_per);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "gemm_bf16_tc_kernel launch");
  return used;
}

int xd_mlp_input_layer(int M, int n_in, int n_hid, const float *d_x, int ldx, const float *d_w1, int ldw,
                       const float *d_b1, void *d_z, void *d_h, void *d_ht, int ldt, void *stream) {
  if (M <= 0 || n_in <= 0 || n_in > 8 || n_hid <= 0 || n_hid > 1024 || !d_x || !d_w1 || !d_b1 || !d_z || !d_h)
    return xd_internal_fail(-1, "bad input-layer arguments");
  input_layer_kernel<<<M, n_hid, 0, (cudaStream_t)stream>>>(M, n_in, n_hid, d_x, ldx, d_w1, ldw, d_b1,
                                                            (__nv_bfloat16 *)d_z, (__nv_bfloat16 *)d_h,
                                                            (__nv_bfloat16 *)d_ht, ldt);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "input_layer_kernel");
}

int xd_mlp_input_grad(int M, int n_in, int n_hid, const void *d_dzt, int ldt, const float *d_x, int ldx,
                      float *d_gw, int ldw, void *stream) {
  if (M <= 0 || n_in <= 0 || n_in > 8 || n_hid <= 0 || !d_dzt || !d_x || !d_gw)
    return xd_internal_fail(-1, "bad input-grad arguments");
  input_grad_kernel<<<n_hid, 256, 0, (cudaStream_t)stream>>>(M, n_in, (const __nv_bfloat16 *)d_dzt, ldt, d_x, ldx,
                                                             d_gw, ldw);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "input_grad_kernel");
}

int xd_surrogate_features(int n, const int *d_idx, const int *d_nodes4, const double *d_sol, const float *d_geom2,
                          float vmax, float *d_x, int ldx, void *stream) {
  if (n < 0 || (n > 0 && (!d_idx || !d_nodes4 || !d_sol || !d_geom2 || !d_x)) || ldx < 5 || vmax <= 0.0f)
    return xd_internal_fail(-1, "bad surrogate-feature arguments");
  if (n == 0) return 0;
  surrogate_features_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(n, d_idx, d_nodes4, d_sol, d_geom2,
                                                                               1.0f / vmax, d_x, ldx);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "surrogate_features_kernel");
}

int xd_surrogate_stage(int n, const int *d_idx, const float *d_y, int ldy, const float *d_out_scale, int n_inst,
                       double *d_stage, void *stream) {
  if (n < 0 || (n > 0 && (!d_idx || !d_y || !d_out_scale || !d_stage)) || ldy < 4 || n_inst < n)
    return xd_internal_fail(-1, "bad surrogate-stage arguments");
  if (n == 0) return 0;
  surrogate_stage_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(n, d_idx, d_y, ldy, d_out_scale, n_inst,
                                                                            d_stage);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "surrogate_stage_kernel");
}

int xd_mlp_forward(const xd_mlp_net *net, int n, const float *d_x, int ldx, float *d_y, int ldy, int *d_err,
                   int max_ctas, void *stream) {
  if (!net || !net->w1 || !net->w5 || !d_x || !d_y || !d_err || n < 0 || net->n_in < 1 || net->n_in > 8 ||
      ldy < kOutPad)
    return xd_internal_fail(-1, "bad fused-forward arguments");
  for (int l = 0; l < 3; ++l)
    if (!net->w[l]) return xd_internal_fail(-1, "bad fused-forward weights");
  for (int l = 0; l < 5; ++l)
    if (!net->b[l]) return xd_internal_fail(-1, "bad fused-forward biases");
  if ((reinterpret_cast<uintptr_t>(net->w[0]) | reinterpret_cast<uintptr_t>(net->w[1]) |
       reinterpret_cast<uintptr_t>(net->w[2]) | reinterpret_cast<uintptr_t>(net->w5)) & 15)
    return xd_internal_fail(-1, "fused-forward weights must be 16-byte aligned");
  if (n == 0) return 0;
  const int tiles = (n + kTileM - 1) / kTileM;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid = tiles < sms ? tiles : sms;
  if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
  const size_t smem = sizeof(FusedSmem);
  cudaError_t e = cudaFuncSetAttribute(mlp_forward_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_err(e, "cudaFuncSetAttribute(mlp_forward_fused_kernel)");
  mlp_forward_fused_kernel<<<grid, kFusedThreads, smem, (cudaStream_t)stream>>>(*net, n, d_x, ldx, d_y, ldy, d_err);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "mlp_forward_fused_kernel");
}

int xd_mse_grad(int M, int n_out, int ld, const float *d_y, const float *d_target, float scale, void *d_dz,
                void *d_dzt, int ldt, float *d_sq, void *stream) {
  if (M <= 0 || !d_y || !d_target || !d_dz || !d_dzt) return xd_internal_fail(-1, "bad mse arguments");
  mse_grad_kernel<<<(M + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      M, n_out, ld, d_y, d_target, scale, (__nv_bfloat16 *)d_dz, (__nv_bfloat16 *)d_dzt, ldt, d_sq);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "mse_grad_kernel");
}

int xd_bias_grad(int M, int N, const void *d_dzt, int ldt, float *d_db, void *stream) {
  if (M <= 0 || N <= 0 || !d_dzt || !d_db) return xd_internal_fail(-1, "bad bias-grad arguments");
  bias_grad_kernel<<<N, 256, 0, (cudaStream_t)stream>>>(M, N, (const __nv_bfloat16 *)d_dzt, ldt, d_db);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "bias_grad_kernel");
}

int xd_splitk_sum(int n, int splits, const float *d_part, float *d_out, void *stream) {
  if (n <= 0 || splits <= 0 || !d_part || !d_out) return xd_internal_fail(-1, "bad split-K arguments");
  splitk_sum_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, splits, d_part, d_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "splitk_sum_kernel");
}

int xd_column_sum(int rows, int cols, const float *d_in, int ld, float *d_out, void *stream) {
  if (rows <= 0 || cols <= 0 || !d_in || !d_out) return xd_internal_fail(-1, "bad column-sum arguments");
  column_sum_kernel<<<cols, 256, 0, (cudaStream_t)stream>>>(rows, cols, d_in, ld, d_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "column_sum_kernel");
}

int xd_adam(int rows, int cols, float *d_p, const float *d_grad, float *d_m, float *d_v, const xd_adam_args *a,
            void *d_p16, void *d_p16t, int ld16, int ld16t, void *stream) {
  if (rows <= 0 || cols <= 0 || !d_p || !d_grad || !d_m || !d_v || !a) return xd_internal_fail(-1, "bad Adam args");
  const int n = rows * cols;
  adam_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      rows, cols, d_p, d_grad, d_m, d_v, a->lr, a->beta1, a->beta2, a->eps, a->bias_corr1, a->bias_corr2,
      (__nv_bfloat16 *)d_p16, (__nv_bfloat16 *)d_p16t, ld16, ld16t);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_err(e, "adam_kernel");
}

}  // extern "C"
