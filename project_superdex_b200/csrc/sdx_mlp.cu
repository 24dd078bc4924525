// sdx_mlp.cu — the learned CG warm start: a per-vertex MLP (15 -> 128 -> 128 -> 128 -> 3, GELU) with
// BF16 weights / activations and FP32 accumulation.
//
// Forward: one fused kernel on the 5th-generation tensor cores. Each CTA (one per SM) keeps the four
// weight matrices in shared memory and walks 128-vertex tiles: the input tile and each hidden
// activation tile are written to shared memory in the K-major "core matrix" layout (8 rows x 16 bytes
// per core matrix), one elected thread issues tcgen05.mma (M = 128, K = 16 per instruction) with the
// accumulator in tensor memory (TMEM), completion is signalled through an mbarrier by tcgen05.commit,
// and the 4 warps read the accumulator back with tcgen05.ld (one TMEM lane per vertex) for the
// bias + GELU epilogue. Every mbarrier wait is bounded; on a timeout the kernel records an error,
// stops issuing MMAs and still frees its TMEM.
//
// Training: FP32 SIMT backward kernels and Adam on FP32 master weights (the MLP has 37k parameters;
// a training step costs microseconds), plus the per-vertex feature and warm-start kernels used by the
// Newton driver. There is no counterpart in the reference (its MLP, mochi_core/include/mochi_core/ai/
// mlp.h:295-435, is CPU inference only, without GELU or training).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sdx_internal.cuh"
#include "sdx_mlp.cuh"

namespace sdx {

// ------------------------------------------------------------------------------------------------
// tcgen05 / mbarrier helpers (inline PTX)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row, k) in a K-major tile of `K` bf16 columns made of 8x(8 bf16) core matrices,
// core matrices of one 8-row group adjacent along K (LBO = 128 B), 8-row groups SBO = K * 16 B apart
__device__ __forceinline__ uint32_t core_off(int row, int k, int K) {
  return (uint32_t)(((row >> 3) * (K >> 3) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: K-major, no swizzle, version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor for kind::f16: BF16 x BF16 -> F32, K-major A and B
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// bounded wait for the phase with parity `parity`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 16 consecutive 32-bit columns starting at taddr (lane field in bits 16..31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ------------------------------------------------------------------------------------------------
// fused forward

constexpr int kTile = 128;
constexpr uint32_t kSW1 = 0;                      // 128 x 16
constexpr uint32_t kSW2 = kSW1 + 128 * 16 * 2;    // 128 x 128
constexpr uint32_t kSW3 = kSW2 + 128 * 128 * 2;   // 128 x 128
constexpr uint32_t kSW4 = kSW3 + 128 * 128 * 2;   // 16 x 128
constexpr uint32_t kSX = kSW4 + 16 * 128 * 2;     // 128 x 16
constexpr uint32_t kSH = kSX + 128 * 16 * 2;      // 128 x 128
constexpr uint32_t kSBar = kSH + 128 * 128 * 2;   // mbarrier
constexpr uint32_t kSTmem = kSBar + 16;           // TMEM base address
constexpr uint32_t kSmemUsed = kSTmem + 16;
constexpr uint32_t kSmemBytes = 200 * 1024;       // > half the SM: one CTA per SM (TMEM budget)

// copy a row-major bf16 matrix [rows][K] (global) into the core layout (shared)
__device__ __forceinline__ void load_weight(const __nv_bfloat16* __restrict__ W, int rows, int K, unsigned char* dst) {
  const int chunks = rows * (K / 8);
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int row = c / (K / 8), kc = c % (K / 8);
    const uint4 v = *reinterpret_cast<const uint4*>(W + (size_t)row * K + kc * 8);
    *reinterpret_cast<uint4*>(dst + core_off(row, kc * 8, K)) = v;
  }
}

// 256 threads: warps w and w + 4 read the same TMEM lane quadrant (vertices 32 (w % 4) ..) and split the
// 128 accumulator columns of the bias + GELU epilogue between them
constexpr int kMlpThreads = 256;

__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_forward(MlpForwardArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int lrow = tid & (kTile - 1), half = tid / kTile;  // tile row (TMEM lane) and column half
  const uint32_t base = smem_u32(smem);
  const uint32_t mbar = base + kSBar;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + kSTmem);

  load_weight(a.W1, 128, 16, smem + kSW1);
  load_weight(a.W2, 128, 128, smem + kSW2);
  load_weight(a.W3, 128, 128, smem + kSW3);
  load_weight(a.W4, 16, 128, smem + kSW4);
  if (tid == 0) mbar_init(mbar, 1);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kSTmem), "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const uint32_t my_lanes = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;

  const int n_tiles = (a.n + kTile - 1) / kTile;
  const int n_slices = (a.n + 31) / 32;
  for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
    if (a.env_mask) {  // the same answer in every thread of the CTA
      bool any = false;
#pragma unroll
      for (int q = 0; q < kTile / 32; ++q) {
        const int sl = tile * (kTile / 32) + q;
        any |= sl < n_slices && a.env_mask[a.slice_env[sl]] != 0;
      }
      if (!any) continue;
    }
    const int row = tile * kTile + lrow;  // this thread's vertex (TMEM lane lrow)
    // input tile: 16 features -> bf16 (first column half)
    if (half == 0) {
      float x[16];
      if (row < a.n) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float4 v = reinterpret_cast<const float4*>(a.X + (size_t)row * 16)[i];
          x[4 * i] = v.x;
          x[4 * i + 1] = v.y;
          x[4 * i + 2] = v.z;
          x[4 * i + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = 0.0f;
      }
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16(x[kc * 8 + i]);
        *reinterpret_cast<uint4*>(smem + kSX + core_off(lrow, kc * 8, 16)) = *reinterpret_cast<uint4*>(h);
      }
    }
    for (int layer = 0; layer < 4 && ok; ++layer) {
      const int K = layer == 0 ? 16 : 128;
      const int N = layer == 3 ? 16 : 128;
      const uint32_t sA = base + (layer == 0 ? kSX : kSH);
      const uint32_t sB = base + (layer == 0 ? kSW1 : layer == 1 ? kSW2 : layer == 2 ? kSW3 : kSW4);
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t idesc = instr_desc(128, N);
        for (int k16 = 0; k16 < K / 16; ++k16) {
          const uint64_t da = smem_desc(sA + k16 * 256, 128, K * 16);
          const uint64_t db = smem_desc(sB + k16 * 256, 128, K * 16);
          mma_bf16(tmem, da, db, idesc, k16 > 0 ? 1u : 0u);
        }
        mma_commit(mbar);
      }
      if (!mbar_wait(mbar, phase, 1ll << 24)) {
        ok = false;
        if (tid == 0) atomicExch(a.error, 1);
        break;
      }
      phase ^= 1u;
      tc_fence_after();
      if (layer < 3) {
        const float* bias = layer == 0 ? a.b1 : layer == 1 ? a.b2 : a.b3;
        float* zout = a.Z ? a.Z + (size_t)layer * a.n * 128 : nullptr;
#pragma unroll 1
        for (int c0 = half * 64; c0 < half * 64 + 64; c0 += 16) {
          float acc[16];
          tmem_ld16(my_lanes + c0, acc);
          __align__(16) __nv_bfloat16 h[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float z = acc[i] + bias[c0 + i];
            if (zout && row < a.n) zout[(size_t)row * 128 + c0 + i] = z;
            h[i] = __float2bfloat16(gelu(z));
          }
          *reinterpret_cast<uint4*>(smem + kSH + core_off(lrow, c0, 128)) = *reinterpret_cast<uint4*>(h);
          *reinterpret_cast<uint4*>(smem + kSH + core_off(lrow, c0 + 8, 128)) = *reinterpret_cast<uint4*>(h + 8);
        }
      } else if (half == 0) {  // warp-uniform: the output columns are read by the first four warps
        float acc[16];
        tmem_ld16(my_lanes, acc);
        if (row < a.n) {
#pragma unroll
          for (int i = 0; i < 3; ++i) a.Y[(size_t)row * 3 + i] = acc[i] + a.b4[i];
        }
      }
    }
  }
  // release TMEM on every path (all MMAs issued by this CTA have completed or timed out)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

int launch_mlp_forward(const MlpForwardArgs& a, int num_sms, cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess)
      return -1;
    attr_set = true;
  }
  if (a.n <= 0) return 0;
  const int tiles = (a.n + kTile - 1) / kTile;
  const int grid = tiles < num_sms ? tiles : num_sms;
  k_mlp_forward<<<grid, kMlpThreads, kSmemBytes, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static_assert(kSmemUsed <= kSmemBytes, "shared memory layout exceeds the request");

// ------------------------------------------------------------------------------------------------
// SIMT FP32 GEMM for the backward pass: C[M][N] (+)= sum_k A(m,k) B(k,n), strided operands

__global__ void k_gemm(int M, int N, int K, const float* __restrict__ A, int64_t sam, int64_t sak,
                       const float* __restrict__ B, int64_t sbk, int64_t sbn, float* C, int64_t scm, int accumulate) {
  __shared__ float tA[32][33], tB[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const int m0 = blockIdx.y * 32, n0 = blockIdx.x * 32;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int k0 = 0; k0 < K; k0 += 32) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = ty + 8 * i;
      tA[r][tx] = (m0 + r < M && k0 + tx < K) ? A[(m0 + r) * sam + (k0 + tx) * sak] : 0.0f;
      tB[r][tx] = (k0 + r < K && n0 + tx < N) ? B[(k0 + r) * sbk + (n0 + tx) * sbn] : 0.0f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const float bv = tB[k][tx];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(tA[ty + 8 * i][k], bv, acc[i]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i, n = n0 + tx;
    if (m < M && n < N) {
      float* c = C + m * scm + n;
      *c = accumulate ? *c + acc[i] : acc[i];
    }
  }
}

static void gemm(int M, int N, int K, const float* A, int64_t sam, int64_t sak, const float* B, int64_t sbk,
                 int64_t sbn, float* C, int64_t scm, int accumulate, cudaStream_t st) {
  dim3 grid((N + 31) / 32, (M + 31) / 32);
  k_gemm<<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, scm, accumulate);
}

// H = bf16(gelu(Z)) as FP32 values; G = gelu'(Z)
__global__ void k_act(int64_t n, const float* __restrict__ Z, float* H, float* G) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = Z[i];
  H[i] = __bfloat162float(__float2bfloat16(gelu(z)));
  G[i] = gelu_grad(z);
}

__global__ void k_mul(int64_t n, float* a, const float* __restrict__ b) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] *= b[i];
}

// column sums: out[j] = sum_i A[i][j]  (bias gradients)
__global__ void k_colsum(int rows, int cols, const float* __restrict__ A, float* out) {
  const int j = blockIdx.x;
  float s = 0.0f;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) s += A[(size_t)i * cols + j];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0];
}

// dY = 2 (Y - T) / (3 n), loss partial sums
__global__ void k_mse(int n, const float* __restrict__ Y, const float* __restrict__ T, float* dY, double* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < n) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float d = Y[3 * i + k] - T[3 * i + k];
      dY[3 * i + k] = 2.0f * d / (3.0f * n);
      l += (double)d * d;
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (3.0 * n));
}

// input bf16 copy of X as FP32 (the forward feeds bf16 X to the tensor cores)
__global__ void k_round_bf16(int64_t n, const float* __restrict__ src, float* dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __bfloat162float(__float2bfloat16(src[i]));
}

// Adam (FP32 master) + bf16 shadow for the forward kernel; entries with mask 0 stay fixed
__global__ void k_adam(int n, float* p, const float* __restrict__ g, float* m, float* v, const uint8_t* __restrict__ mask,
                       __nv_bfloat16* pb, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mask[i]) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
  pb[i] = __float2bfloat16(p[i]);
}

__global__ void k_to_bf16(int n, const float* __restrict__ p, __nv_bfloat16* pb, float* pr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pb[i] = __float2bfloat16(p[i]);
  pr[i] = __bfloat162float(pb[i]);
}

void mlp_sync_bf16(const MlpParams& P, cudaStream_t st) {
  k_to_bf16<<<(kMlpParams + 255) / 256, 256, 0, st>>>(kMlpParams, P.p, P.pb, P.pr);
}

MlpForwardArgs mlp_forward_args(const MlpParams& P, const float* X, int n, float* Y, float* Z, int* error) {
  MlpForwardArgs a;
  a.n = n;
  a.X = X;
  a.Y = Y;
  a.Z = Z;
  a.error = error;
  a.W1 = P.pb + kOffW1;
  a.W2 = P.pb + kOffW2;
  a.W3 = P.pb + kOffW3;
  a.W4 = P.pb + kOffW4;
  a.b1 = P.p + kOffB1;
  a.b2 = P.p + kOffB2;
  a.b3 = P.p + kOffB3;
  a.b4 = P.p + kOffB4;
  a.slice_env = nullptr;
  a.env_mask = nullptr;
  return a;
}

// Gradients of the MSE loss w.r.t. all parameters for a batch (X: n x 16, T: n x 3). Runs the tensor-core
// forward with pre-activations, then the FP32 backward. W: scratch of the batch size.
int mlp_gradients(const MlpParams& P, MlpWork& W, const float* X, const float* T, int n, int num_sms,
                  double* loss, int* error, cudaStream_t st) {
  if (launch_mlp_forward(mlp_forward_args(P, X, n, W.Y, W.Z, error), num_sms, st) != 0) return -1;
  const int64_t nh = (int64_t)n * 128;
  float* Z1 = W.Z;
  float* Z2 = W.Z + nh;
  float* Z3 = W.Z + 2 * nh;
  const int th = 256;
  const unsigned blocks = (unsigned)((nh + th - 1) / th);
  k_act<<<blocks, th, 0, st>>>(nh, Z1, W.H1, W.G1);
  k_act<<<blocks, th, 0, st>>>(nh, Z2, W.H2, W.G2);
  k_act<<<blocks, th, 0, st>>>(nh, Z3, W.H3, W.G3);
  k_round_bf16<<<(unsigned)(((int64_t)n * 16 + th - 1) / th), th, 0, st>>>((int64_t)n * 16, X, W.Xb);
  cudaMemsetAsync(loss, 0, sizeof(double), st);
  k_mse<<<(n + th - 1) / th, th, 0, st>>>(n, W.Y, T, W.dY, loss);
  const float* Wr = P.pr;  // bf16-rounded weights as FP32 (what the forward multiplied with)
  float* gW4 = P.g + kOffW4;
  float* gB4 = P.g + kOffB4;
  cudaMemsetAsync(P.g, 0, sizeof(float) * kMlpParams, st);
  // layer 4: Y = H3 W4^T + b4 (rows 0..2 of W4 used)
  gemm(3, 128, n, W.dY, 1, 3, W.H3, 128, 1, gW4, 128, 0, st);            // dW4 = dY^T H3
  k_colsum<<<3, 256, 0, st>>>(n, 3, W.dY, gB4);
  gemm(n, 128, 3, W.dY, 3, 1, Wr + kOffW4, 128, 1, W.dA, 128, 0, st);    // dH3 = dY W4
  k_mul<<<blocks, th, 0, st>>>(nh, W.dA, W.G3);                           // dZ3
  // layer 3
  gemm(128, 128, n, W.dA, 1, 128, W.H2, 128, 1, P.g + kOffW3, 128, 0, st);
  k_colsum<<<128, 256, 0, st>>>(n, 128, W.dA, P.g + kOffB3);
  gemm(n, 128, 128, W.dA, 128, 1, Wr + kOffW3, 128, 1, W.dB, 128, 0, st);  // dH2 = dZ3 W3
  k_mul<<<blocks, th, 0, st>>>(nh, W.dB, W.G2);
  // layer 2
  gemm(128, 128, n, W.dB, 1, 128, W.H1, 128, 1, P.g + kOffW2, 128, 0, st);
  k_colsum<<<128, 256, 0, st>>>(n, 128, W.dB, P.g + kOffB2);
  gemm(n, 128, 128, W.dB, 128, 1, Wr + kOffW2, 128, 1, W.dA, 128, 0, st);  // dH1 = dZ2 W2
  k_mul<<<blocks, th, 0, st>>>(nh, W.dA, W.G1);
  // layer 1
  gemm(128, 16, n, W.dA, 1, 128, W.Xb, 16, 1, P.g + kOffW1, 16, 0, st);
  k_colsum<<<128, 256, 0, st>>>(n, 128, W.dA, P.g + kOffB1);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

void mlp_adam(const MlpParams& P, float lr, int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(kMlpParams, P.p, P.g, P.m, P.v, P.mask, P.pb, lr, b1, b2, eps, c1, c2);
  k_to_bf16<<<(kMlpParams + 255) / 256, 256, 0, st>>>(kMlpParams, P.p, P.pb, P.pr);
}

// ------------------------------------------------------------------------------------------------
// features and warm start (one thread per row)

// raw per-row quantities: u, dt v, the last Newton update dx1, the previous step's update at the same
// Newton iteration dx2 (zero when there is none), D^-1 g (Jacobi-preconditioned Newton gradient)
__global__ void k_feature_raw(int64_t n_rows, const int* __restrict__ slice_env, const uint8_t* __restrict__ env_mask,
                              const double* __restrict__ u, const double* __restrict__ v, double dt,
                              const double* __restrict__ dx1, const double* __restrict__ dx2,
                              const double* __restrict__ g, const float* __restrict__ val,
                              const int* __restrict__ diag_pos, const uint8_t* __restrict__ pin, float* raw) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  if (env_mask && !env_mask[slice_env[r >> 5]]) return;  // envs outside this solve: nothing to predict
  const int dp = diag_pos[r];
  float o[16];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float d = dp >= 0 ? val[val_index(dp, 4 * k)] : 0.0f;
    const bool free = dp >= 0 && !((pin[r] >> k) & 1);
    o[k] = (float)u[3 * r + k];
    o[3 + k] = (float)(dt * v[3 * r + k]);
    o[6 + k] = (float)dx1[3 * r + k];
    o[9 + k] = (float)dx2[3 * r + k];
    o[12 + k] = (free && d != 0.0f) ? (float)(g[3 * r + k] / d) : 0.0f;
  }
  o[15] = 0.0f;
  float4* out = reinterpret_cast<float4*>(raw + 16 * r);  // 64-byte records
#pragma unroll
  for (int q = 0; q < 4; ++q) out[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
}

// per-env sums of squares of the 5 feature groups (u, dt v, dx_{k-1}, dx_{k-2}, D^-1 g). Each warp walks a
// contiguous run of slices and keeps lane-local sums while the env stays the same (slices are env-ordered),
// so the atomics are one per warp and env run instead of one per slice.
__global__ void k_feature_scale(int n_slices, int per_warp, const int* __restrict__ slice_env,
                                const uint8_t* __restrict__ env_mask, const float* __restrict__ raw, double* sumsq) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int s0 = wid * per_warp, s1 = min(n_slices, s0 + per_warp);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int cur = -1;
  auto flush = [&]() {
#pragma unroll
    for (int grp = 0; grp < 5; ++grp) {
      double v = acc[grp];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0 && cur >= 0) atomicAdd(sumsq + 5 * cur + grp, v);
      acc[grp] = 0.0;
    }
  };
  for (int s = s0; s < s1; ++s) {
    const int e = slice_env[s];
    if (e != cur) {
      flush();
      cur = e;
    }
    if (env_mask && !env_mask[e]) continue;
    const float4* o = reinterpret_cast<const float4*>(raw + 16 * ((int64_t)s * 32 + lane));
    const float4 a = o[0], b = o[1], c = o[2], d = o[3];
    const float f[16] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w};
#pragma unroll
    for (int grp = 0; grp < 5; ++grp)
      acc[grp] += (double)f[3 * grp] * f[3 * grp] + (double)f[3 * grp + 1] * f[3 * grp + 1] +
                  (double)f[3 * grp + 2] * f[3 * grp + 2];
  }
  flush();
}

// X[row] = 1-ring average of each raw group / that group's RMS over the env (inputs of order one)
__global__ void k_feature_ring(Matrix A, const uint8_t* __restrict__ env_mask, const float* __restrict__ raw,
                               const double* __restrict__ sumsq, const int* __restrict__ env_rows, float* X) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= A.n_slices) return;
  const int e = A.slice_env[s];
  const int64_t row = (int64_t)s * 32 + lane;
  if (env_mask && !env_mask[e]) {  // outside this solve: zero inputs, no neighbour gathers
    float4* xo = reinterpret_cast<float4*>(X + 16 * row);
#pragma unroll
    for (int q = 0; q < 4; ++q) xo[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  float acc[15];
#pragma unroll
  for (int i = 0; i < 15; ++i) acc[i] = 0.0f;
  int cnt = 0;
  const int base = A.slice_ptr[s], w = A.slice_w[s];
  for (int k = 0; k < w; ++k) {
    const int cj = A.col[base + k * 32 + lane];
    if (cj & kPadBit) continue;
    const float4* o = reinterpret_cast<const float4*>(raw + 16 * (int64_t)cj);  // one 64-byte record
    const float4 a = o[0], b = o[1], c = o[2], d = o[3];
    const float f[15] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z};
#pragma unroll
    for (int i = 0; i < 15; ++i) acc[i] += f[i];
    ++cnt;
  }
  const bool active = !env_mask || env_mask[e];
  float x[16];
#pragma unroll
  for (int grp = 0; grp < 5; ++grp) {
    const double rms = sqrt(sumsq[5 * e + grp] / fmax(1.0, (double)env_rows[e]));
    const float inv = (active && cnt > 0 && rms > 0.0) ? (float)(1.0 / (rms * cnt)) : 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) x[3 * grp + i] = acc[3 * grp + i] * inv;
  }
  x[15] = 0.0f;
  float4* xo = reinterpret_cast<float4*>(X + 16 * row);
#pragma unroll
  for (int q = 0; q < 4; ++q) xo[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
}

// dx0 = MLP(X) on free DoFs of active envs (its scale is set by the solver's energy-optimal scaling)
// Start vectors of the learned warm start: x = h / RMS_env(h), the temporal guess (the previous step's
// update at the same Newton iteration, zero when there is none), and x2 = Y, the network's correction;
// the PCG combines them by a Galerkin step on span{x, x2}. Pinned and padding DoFs are zero.
__global__ void k_warm_start(int64_t n_rows, const int* __restrict__ slice_env, const uint8_t* __restrict__ env_mask,
                             const float* __restrict__ Y, const uint8_t* __restrict__ pin,
                             const int* __restrict__ diag_pos, const double* __restrict__ h,
                             const double* __restrict__ h2, const int* __restrict__ env_rows, double* dx,
                             double* x2) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  const int e = slice_env[r >> 5];
  if (env_mask && !env_mask[e]) return;
  const double hr = sqrt(h2[e] / fmax(1.0, 3.0 * (double)env_rows[e]));
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const bool free = diag_pos[r] >= 0 && !((pin[r] >> k) & 1);
    const double y = (double)Y[3 * r + k];
    const double t = hr > 0.0 ? h[3 * r + k] / hr : 0.0;
    dx[3 * r + k] = (free && isfinite(t)) ? t : 0.0;
    x2[3 * r + k] = (free && isfinite(y)) ? y : 0.0;
  }
}
void launch_features(const Matrix& A, int64_t n_rows, const uint8_t* env_mask, const double* u, const double* v,
                     double dt, const double* dx1, const double* dx2, const double* g, const int* diag_pos,
                     const uint8_t* pin, const int* env_rows, float* raw, double* sumsq, int n_envs, float* X,
                     cudaStream_t st) {
  if (n_rows == 0) return;
  k_feature_raw<<<(unsigned)((n_rows + 255) / 256), 256, 0, st>>>(n_rows, A.slice_env, env_mask, u, v, dt, dx1, dx2, g,
                                                                   A.val, diag_pos, pin, raw);
  cudaMemsetAsync(sumsq, 0, sizeof(double) * 5 * n_envs, st);
  const int64_t t = (int64_t)A.n_slices * 32;
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int warps = 8 * sms;  // one 256-thread block per SM
    const int per_warp = (A.n_slices + warps - 1) / warps;
    k_feature_scale<<<(unsigned)sms, 256, 0, st>>>(A.n_slices, per_warp, A.slice_env, env_mask, raw, sumsq);
  }
  k_feature_ring<<<(unsigned)((t + 255) / 256), 256, 0, st>>>(A, env_mask, raw, sumsq, env_rows, X);
}
void launch_warm_start(int64_t n_rows, const int* slice_env, const uint8_t* env_mask, const float* Y,
                       const uint8_t* pin, const int* diag_pos, const double* h, const double* h2,
                       const int* env_rows, double* dx, double* x2, cudaStream_t st) {
  if (n_rows == 0) return;
  k_warm_start<<<(unsigned)((n_rows + 255) / 256), 256, 0, st>>>(n_rows, slice_env, env_mask, Y, pin, diag_pos, h,
                                                                   h2, env_rows, dx, x2);
}

// training targets: the shape of the update relative to the temporal guess h,
// T[row] = dx / RMS_env(dx) - h / RMS_env(h) (the second term is zero without a guess); dx2 and h2 hold
// |dx|^2 and |h|^2 per env
__global__ void k_targets(int64_t n_rows, const int* __restrict__ slice_env, const double* __restrict__ dx,
                          const double* __restrict__ dx2, const double* __restrict__ h,
                          const double* __restrict__ h2, const int* __restrict__ env_rows, float* T) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  const int e = slice_env[r >> 5];
  const double n3 = fmax(1.0, 3.0 * (double)env_rows[e]);
  const double rms = sqrt(dx2[e] / n3), hr = sqrt(h2[e] / n3);
#pragma unroll
  for (int k = 0; k < 3; ++k)
    T[3 * r + k] = rms > 0.0 ? (float)(dx[3 * r + k] / rms - (hr > 0.0 ? h[3 * r + k] / hr : 0.0)) : 0.0f;
}
void launch_targets(int64_t n_rows, const int* slice_env, const double* dx, const double* dx2, const double* h,
                    const double* h2, const int* env_rows, float* T, cudaStream_t st) {
  if (n_rows == 0) return;
  k_targets<<<(unsigned)((n_rows + 255) / 256), 256, 0, st>>>(n_rows, slice_env, dx, dx2, h, h2, env_rows, T);
}

}  // namespace sdx
