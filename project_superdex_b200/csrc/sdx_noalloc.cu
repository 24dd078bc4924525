// sdx_noalloc.cu — a Jacobi-PCG solve that allocates no memory (sdx_pcg_solve_device_noalloc).
//
// Some callers cannot allocate device memory at the moment they need a solve: a host engine that hands
// every byte of GPU memory to its own pool allocator and forbids cudaMalloc/cudaFree inside its
// per-step callbacks (a cudaMalloc there would synchronize the device and fragment the pool), or a
// real-time control loop that must not take the allocator's locks. This entry point serves them: the
// caller passes its own device buffers for the matrix, right-hand side and solution, and every work
// vector of the solve lives in one fixed-size array compiled into this library (g_scratch below), which
// each GPU that loads the library holds until the process exits.
//
// Limits and sharing rules:
//   * at most kMaxBlockRows block rows (3 * kMaxBlockRows unknowns); larger systems are rejected;
//   * all calls on a device share the one array and it keeps whatever the last call left there; the
//     parts that must start from zero (grid-barrier counters, status words) are cleared by each call,
//     everything else is fully written before it is read;
//   * two calls whose work overlaps on the GPU (different streams or threads without ordering) race on
//     the array and give wrong results; callers serialize them (one stream, or their own events);
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress, which may
//     load this library's device code); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/sdx_b200.h"

namespace sdx_noalloc {

constexpr int kMaxBlockRows = 65536;
constexpr int kMaxCtas = 1024;
constexpr int kSlice = 32;

// byte layout of the scratch array (every region 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kSyncOff = 0;                                     // 8 x uint32
constexpr size_t kOutOff = 256;                                    // status words
constexpr size_t kPartOff = 512;                                   // 2 x kMaxCtas x 3 doubles
constexpr size_t kROff = align256(kPartOff + 2ull * kMaxCtas * 3 * 8);
constexpr size_t kPOff = align256(kROff + 3ull * kMaxBlockRows * 8);  // r: FP64
constexpr size_t kQOff = align256(kPOff + 3ull * kMaxBlockRows * 4);  // p: FP32
constexpr size_t kZOff = align256(kQOff + 3ull * kMaxBlockRows * 4);  // q: FP32
constexpr size_t kDOff = align256(kZOff + 16ull * kMaxBlockRows);     // z: float4
constexpr size_t kBytes = align256(kDOff + 9ull * kMaxBlockRows * 4); // preconditioner: 9 floats

static __device__ __align__(256) unsigned char g_scratch[kBytes];

struct Out {
  int iters;
  int conv;
  int bad_index;
  int pad;
  double res;
  double relres;
};

struct Args {
  int n;  // block rows
  int64_t nnzb;
  const int64_t* row_ptr;
  const int32_t* col;
  const float* val;  // 9 per block: row-major blocks, or the row strips of SDX_BSR_ROW_STRIPS
  int strips;        // 1: entry (lr, lc) of block k of a row is val[9 ptr + 3 (lr len + k) + lc]
  const double* b;
  double* x;
  unsigned char* scratch;
  int precond;
  double rel_tol, abs_tol, rel_div_tol;
  int max_iter, polak_ribiere, replace_every, zero_guess, abort_spd;
  long long spin_limit;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Thread 0's verdict (passed, or the error word set) is broadcast through shared memory, so every thread
// of a CTA returns the same value even when another CTA sets the error word meanwhile.
__device__ __forceinline__ bool grid_barrier(unsigned* sync, unsigned nblocks, long long spin_limit) {
  __shared__ unsigned s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = sync + 1;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned prev = atomicAdd(sync, 1u);
    if (prev == nblocks - 1) {
      atomicExch(sync, 0u);
      __threadfence();
      atomicAdd(sync + 1, 1u);
    } else {
      long long spins = 0;
      while (*vgen == gen) {
        if (++spins > spin_limit) {
          atomicExch(sync + 2, 1u);  // bounded wait: give up, record, unwind
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = *((volatile unsigned*)(sync + 2)) == 0u ? 1u : 0u;
  }
  __syncthreads();
  return s_ok != 0u;
}

// Block range [b0, b1) of a row. A range outside [0, nnzb) or with b1 < b0 (a malformed row_ptr) is
// flagged in *bad and treated as empty, so no load leaves the caller's arrays.
__device__ __forceinline__ void row_range(const Args& a, int row, int64_t& b0, int64_t& b1, int* bad) {
  b0 = a.row_ptr[row];
  b1 = a.row_ptr[row + 1];
  if (b0 < 0 || b1 < b0 || b1 > a.nnzb) {
    *bad = 1;
    b0 = b1 = 0;
  }
}

// Entry e (= 3 lr + lc) of the k-th block of a row whose blocks are [b0, b1).
__device__ __forceinline__ float block_entry(const Args& a, int64_t b0, int64_t b1, int64_t k, int e) {
  return a.strips ? a.val[9 * b0 + 3 * ((e / 3) * (b1 - b0) + k) + e % 3] : a.val[9 * (b0 + k) + e];
}

// y_row = A_row . v for one block row; v is read through L2 (it is written by other CTAs)
template <class V>
__device__ __forceinline__ void row_product(const Args& a, int row, V load, double acc[3], int* bad) {
  acc[0] = acc[1] = acc[2] = 0.0;
  int64_t b0, b1;
  row_range(a, row, b0, b1, bad);
  for (int64_t k = b0; k < b1; ++k) {
    const int j = a.col[k];
    if (j < 0 || j >= a.n) {
      *bad = 1;
      continue;
    }
    double xj[3];
    load(j, xj);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      acc[r] += (double)block_entry(a, b0, b1, k - b0, 3 * r) * xj[0] +
                (double)block_entry(a, b0, b1, k - b0, 3 * r + 1) * xj[1] +
                (double)block_entry(a, b0, b1, k - b0, 3 * r + 2) * xj[2];
  }
}

__device__ __forceinline__ void precondition(const Args& a, const float* D, int row, const double r[3], float z[3]) {
  if (a.precond == 1) {
#pragma unroll
    for (int k = 0; k < 3; ++k) z[k] = (float)(D[9 * row + k] * r[k]);
  } else if (a.precond == 2) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      z[k] = (float)(D[9 * row + 3 * k] * r[0] + D[9 * row + 3 * k + 1] * r[1] + D[9 * row + 3 * k + 2] * r[2]);
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) z[k] = (float)r[k];
  }
}

// Same iteration as the context PCG (phase 1: p, q = A p; phase 2: x, r, z; FP64 true-residual
// replacement every `replace_every` iterations and to confirm convergence), for one system in BSR form.
__global__ void k_pcg_noalloc(Args a) {
  __shared__ double red[32][3];
  __shared__ double tot[3];
  unsigned* sync = reinterpret_cast<unsigned*>(a.scratch + kSyncOff);
  Out* out = reinterpret_cast<Out*>(a.scratch + kOutOff);
  double* part = reinterpret_cast<double*>(a.scratch + kPartOff);
  double* R = reinterpret_cast<double*>(a.scratch + kROff);
  float* P = reinterpret_cast<float*>(a.scratch + kPOff);
  float* Q = reinterpret_cast<float*>(a.scratch + kQOff);
  float4* Z = reinterpret_cast<float4*>(a.scratch + kZOff);
  float* D = reinterpret_cast<float*>(a.scratch + kDOff);
  const unsigned ncta = gridDim.x;
  const int c = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int n_slices = (a.n + kSlice - 1) / kSlice;
  const int s0 = (int)((int64_t)n_slices * c / ncta), s1 = (int)((int64_t)n_slices * (c + 1) / ncta);
  int bad = 0;
  double acc[3] = {0.0, 0.0, 0.0};

  auto cta_reduce = [&](int nq, int buf) {  // warp partials -> one CTA partial per quantity
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double v = warp_sum(acc[k]);
      if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < nq) {
      double v = 0.0;
      for (int w = 0; w < nwarps; ++w) v += red[w][threadIdx.x];
      part[(size_t)buf * kMaxCtas * 3 + (size_t)c * 3 + threadIdx.x] = v;
    }
    acc[0] = acc[1] = acc[2] = 0.0;
  };
  auto grid_total = [&](int nq, int buf) {  // every CTA sums all CTA partials in the same order
    if (warp < nq) {
      double v = 0.0;
      for (unsigned cc = lane; cc < ncta; cc += 32) v += __ldcg(part + (size_t)buf * kMaxCtas * 3 + cc * 3 + warp);
      v = warp_sum(v);
      if (lane == 0) tot[warp] = v;
    }
    __syncthreads();
  };
  auto load_z = [&](int j, double xj[3]) {
    const float4 v = __ldcg(Z + j);
    xj[0] = v.x;
    xj[1] = v.y;
    xj[2] = v.z;
  };
  auto load_x = [&](int j, double xj[3]) {
    xj[0] = __ldcg(a.x + 3 * (int64_t)j);
    xj[1] = __ldcg(a.x + 3 * (int64_t)j + 1);
    xj[2] = __ldcg(a.x + 3 * (int64_t)j + 2);
  };

  // ---- setup: preconditioner, r = b - A x0, z = M^-1 r; totals b.b, r.r, r.z ----
  for (int s = s0 + warp; s < s1; s += nwarps) {
    const int row = s * kSlice + lane;
    if (row >= a.n) continue;
    float blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int64_t b0, b1;
    row_range(a, row, b0, b1, &bad);
    if (row == 0 && b0 != 0) bad = 1;
    if (row == a.n - 1 && a.row_ptr[a.n] != a.nnzb) bad = 1;
    for (int64_t k = b0; k < b1; ++k)
      if (a.col[k] == row)
        for (int e = 0; e < 9; ++e) blk[e] = block_entry(a, b0, b1, k - b0, e);
    if (a.precond == 1) {
      for (int k = 0; k < 3; ++k) D[9 * row + k] = blk[4 * k] != 0.0f ? 1.0f / blk[4 * k] : 1.0f;
    } else if (a.precond == 2) {
      float cf[9];
      cf[0] = blk[4] * blk[8] - blk[5] * blk[7];
      cf[1] = blk[5] * blk[6] - blk[3] * blk[8];
      cf[2] = blk[3] * blk[7] - blk[4] * blk[6];
      cf[3] = blk[2] * blk[7] - blk[1] * blk[8];
      cf[4] = blk[0] * blk[8] - blk[2] * blk[6];
      cf[5] = blk[1] * blk[6] - blk[0] * blk[7];
      cf[6] = blk[1] * blk[5] - blk[2] * blk[4];
      cf[7] = blk[2] * blk[3] - blk[0] * blk[5];
      cf[8] = blk[0] * blk[4] - blk[1] * blk[3];
      const float det = blk[0] * cf[0] + blk[1] * cf[1] + blk[2] * cf[2];
      const float inv = det != 0.0f ? 1.0f / det : 0.0f;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[9 * row + 3 * i + j] = cf[3 * j + i] * inv;
    }
    double r[3];
    if (a.zero_guess) {
      for (int k = 0; k < 3; ++k) {
        a.x[3 * row + k] = 0.0;
        r[k] = a.b[3 * row + k];
      }
    } else {
      double ax[3];
      row_product(a, row, load_x, ax, &bad);
      for (int k = 0; k < 3; ++k) r[k] = a.b[3 * row + k] - ax[k];
    }
    float z[3];
    precondition(a, D, row, r, z);
    for (int k = 0; k < 3; ++k) R[3 * row + k] = r[k];
    Z[row] = make_float4(z[0], z[1], z[2], 0.0f);
    const double bx = a.b[3 * row], by = a.b[3 * row + 1], bz = a.b[3 * row + 2];
    acc[0] += bx * bx + by * by + bz * bz;
    acc[1] += r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    acc[2] += r[0] * z[0] + r[1] * z[1] + r[2] * z[2];
  }
  if (bad) atomicExch(&out->bad_index, 1);
  cta_reduce(3, 0);
  if (!grid_barrier(sync, ncta, a.spin_limit)) return;
  // a malformed matrix (row_ptr or a column index) stops every CTA before the iteration: each reads the
  // word after the barrier that ordered all set-up writes
  if (*((volatile int*)&out->bad_index) != 0) return;
  grid_total(3, 0);
  const double bb = tot[0];
  const double conv_thr = fmax(a.abs_tol * a.abs_tol, (bb * a.rel_tol) * a.rel_tol);
  const double div_thr = (bb * a.rel_div_tol) * a.rel_div_tol;
  double rr = tot[1], rz = tot[2], alpha = 0.0, beta = 0.0;
  int status = 0, iters = 0;
  bool first = true;
  int verify_at = -1;
  if (!isfinite(rr) || rr > div_thr)
    status = 3;
  else if (rr <= conv_thr)
    status = 1;

  for (int it = 1; status == 0; ++it) {
    // phase 1: p = z + beta p, q = A z + beta q, p.q
    for (int s = s0 + warp; s < s1; s += nwarps) {
      const int row = s * kSlice + lane;
      if (row >= a.n) continue;
      double az[3];
      row_product(a, row, load_z, az, &bad);
      const float4 zr = Z[row];
      const float zz[3] = {zr.x, zr.y, zr.z};
      float pn[3], qn[3];
      for (int k = 0; k < 3; ++k) {
        pn[k] = first ? zz[k] : fmaf((float)beta, P[3 * row + k], zz[k]);
        qn[k] = first ? (float)az[k] : fmaf((float)beta, Q[3 * row + k], (float)az[k]);
        P[3 * row + k] = pn[k];
        Q[3 * row + k] = qn[k];
      }
      acc[0] += (double)pn[0] * qn[0] + (double)pn[1] * qn[1] + (double)pn[2] * qn[2];
    }
    cta_reduce(1, 1);
    if (!grid_barrier(sync, ncta, a.spin_limit)) return;
    grid_total(1, 1);
    const double pq = tot[0];
    if (pq <= 0.0 && a.abort_spd) {
      status = 3;
      iters = it;
      break;
    }
    alpha = rz / pq;
    const bool replace = (verify_at == it) || (a.replace_every > 0 && it % a.replace_every == 0);
    // phase 2: x += alpha p, r -= alpha q, z = M^-1 r; r.r, r.z_old, r.z
    for (int s = s0 + warp; s < s1; s += nwarps) {
      const int row = s * kSlice + lane;
      if (row >= a.n) continue;
      double r[3];
      for (int k = 0; k < 3; ++k) {
        a.x[3 * row + k] += alpha * (double)P[3 * row + k];
        r[k] = R[3 * row + k] - alpha * (double)Q[3 * row + k];
      }
      if (replace) continue;
      const float4 zo = Z[row];
      float z[3];
      precondition(a, D, row, r, z);
      for (int k = 0; k < 3; ++k) R[3 * row + k] = r[k];
      Z[row] = make_float4(z[0], z[1], z[2], 0.0f);
      acc[0] += r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      acc[1] += r[0] * zo.x + r[1] * zo.y + r[2] * zo.z;
      acc[2] += r[0] * z[0] + r[1] * z[1] + r[2] * z[2];
    }
    if (replace) {
      if (!grid_barrier(sync, ncta, a.spin_limit)) return;
      for (int s = s0 + warp; s < s1; s += nwarps) {
        const int row = s * kSlice + lane;
        if (row >= a.n) continue;
        double ax[3], r[3];
        row_product(a, row, load_x, ax, &bad);
        for (int k = 0; k < 3; ++k) r[k] = a.b[3 * row + k] - ax[k];
        const float4 zo = Z[row];
        float z[3];
        precondition(a, D, row, r, z);
        for (int k = 0; k < 3; ++k) R[3 * row + k] = r[k];
        Z[row] = make_float4(z[0], z[1], z[2], 0.0f);
        acc[0] += r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        acc[1] += r[0] * zo.x + r[1] * zo.y + r[2] * zo.z;
        acc[2] += r[0] * z[0] + r[1] * z[1] + r[2] * z[2];
      }
    }
    cta_reduce(3, 0);
    if (!grid_barrier(sync, ncta, a.spin_limit)) return;
    grid_total(3, 0);
    rr = tot[0];
    const double rzo = tot[1], rzn = tot[2];
    iters = it;
    if (!isfinite(rr) || rr > div_thr) {
      status = 3;
    } else if (rr <= conv_thr && replace) {
      status = 1;
    } else if (it >= a.max_iter) {
      status = 2;
    } else if (rzn == 0.0) {
      status = 3;
    } else {
      if (rr <= conv_thr) verify_at = it + 1;  // confirm on the FP64 true residual next iteration
      beta = (rzn - ((a.polak_ribiere && !first) ? rzo : 0.0)) / rz;
      rz = rzn;
      first = false;
    }
  }
  if (bad) atomicExch(&out->bad_index, 1);
  if (c == 0 && threadIdx.x == 0) {
    out->iters = iters;
    out->conv = status;
    out->res = sqrt(fmax(rr, 0.0));
    out->relres = bb == 0.0 ? 0.0 : sqrt(fmax(rr, 0.0) / bb);
  }
}

constexpr int kThreads = 512;
constexpr int kMaxDevices = 64;
static std::mutex g_setup_mutex;
static void* g_symbol_address[kMaxDevices];  // set-up result per device (nullptr until looked up)
static int g_ctas[kMaxDevices];

}  // namespace sdx_noalloc

using namespace sdx_noalloc;

namespace sdx {
int record_error(int code, const char* msg, const char* detail);  // sets sdx_last_error() (sdx_host.cu)
long long device_spin_limit();                                     // bound of the device spins (sdx_host.cu)
}

static int fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
  return sdx::record_error(code, msg, e != cudaSuccess ? cudaGetErrorString(e) : nullptr);
}

extern "C" int sdx_pcg_solve_device_noalloc(int block_rows, int64_t nnzb, const int64_t* d_row_ptr,
                                            const int32_t* d_col, const float* d_values, const double* d_b,
                                            double* d_x, int hint, const sdx_linear_params* params,
                                            sdx_linear_status* status, void* stream) {
  if (!d_row_ptr || !d_col || !d_values || !d_b || !d_x || !params || !status)
    return fail(SDX_ERR_INVALID_ARGUMENT, "null argument");
  if (block_rows <= 0 || nnzb <= 0) return fail(SDX_ERR_INVALID_ARGUMENT, "empty system");
  if (params->value_layout != SDX_BSR_ROW_STRIPS && params->value_layout != SDX_BSR_BLOCKS)
    return fail(SDX_ERR_INVALID_ARGUMENT, "value_layout");
  static_assert(kMaxBlockRows == SDX_NOALLOC_MAX_BLOCK_ROWS, "limit must match the header");
  if (block_rows > kMaxBlockRows)
    return fail(SDX_ERR_INVALID_ARGUMENT, "system larger than the no-allocation limit of 65536 block rows");
  if (params->preconditioner < 0 || params->preconditioner > 2 || params->max_iter <= 0)
    return fail(SDX_ERR_INVALID_ARGUMENT, "bad solver parameters");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SDX_ERR_CUDA, "cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return fail(SDX_ERR_UNSUPPORTED, "device index too large");
  void* scratch = nullptr;
  {
    // one-time set-up per device, with that device current: the array's device address
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_symbol_address[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_scratch);
      if (e != cudaSuccess || !ptr) return fail(SDX_ERR_CUDA, "cudaGetSymbolAddress(g_scratch)", e);
      int sms = 0, per_sm = 0;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return fail(SDX_ERR_CUDA, "cudaDeviceGetAttribute", e);
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_noalloc, kThreads, 0);
      if (e != cudaSuccess || per_sm <= 0) return fail(SDX_ERR_CUDA, "occupancy query", e);
      int ctas = sms * per_sm;
      g_ctas[dev] = ctas > kMaxCtas ? kMaxCtas : ctas;
      g_symbol_address[dev] = ptr;
    }
    scratch = g_symbol_address[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  // clear what must start at zero: barrier counters, error word and status words
  e = cudaMemsetAsync(scratch, 0, kPartOff, st);
  if (e != cudaSuccess) return fail(SDX_ERR_CUDA, "cudaMemsetAsync", e);
  Args a;
  memset(&a, 0, sizeof(a));
  a.n = block_rows;
  a.nnzb = nnzb;
  a.strips = params->value_layout == SDX_BSR_ROW_STRIPS;
  a.row_ptr = d_row_ptr;
  a.col = d_col;
  a.val = d_values;
  a.b = d_b;
  a.x = d_x;
  a.scratch = (unsigned char*)scratch;
  a.precond = params->preconditioner;
  a.rel_tol = params->rel_tol;
  a.abs_tol = params->abs_tol;
  a.rel_div_tol = params->rel_div_tol;
  a.max_iter = params->max_iter;
  a.polak_ribiere = params->polak_ribiere;
  a.replace_every = params->replace_every > 0 ? params->replace_every : 32;
  a.zero_guess = hint == SDX_GUESS_ZERO;
  a.abort_spd = params->abort_if_not_spd;
  a.spin_limit = sdx::device_spin_limit();
  void* kargs[] = {&a};
  e = cudaLaunchCooperativeKernel((const void*)k_pcg_noalloc, dim3(g_ctas[dev]), dim3(kThreads), kargs, 0, st);
  if (e != cudaSuccess) return fail(SDX_ERR_CUDA, "cooperative launch", e);
  unsigned flags[8];
  Out out;
  e = cudaMemcpyAsync(flags, (unsigned char*)scratch + kSyncOff, sizeof(flags), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&out, (unsigned char*)scratch + kOutOff, sizeof(out), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(SDX_ERR_CUDA, "result copy", e);
  if (flags[2] != 0u) return fail(SDX_ERR_DEVICE_TIMEOUT, "grid barrier timed out");
  if (out.bad_index) return fail(SDX_ERR_INVALID_ARGUMENT, "row_ptr or a column index out of range");
  status->num_iter = out.iters;
  status->residual_norm = out.res;
  status->relative_residual_norm = out.relres;
  status->convergence = out.conv;
  return SDX_OK;
}
