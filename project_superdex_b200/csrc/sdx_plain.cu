// sdx_plain.cu — the plain FP64 Jacobi-PCG, the reference's CUDA solver path restated on this GPU.
//
// This is the comparison arm of the solver (sdx_linear_params.solver_impl = SDX_SOLVER_PLAIN_FP64), not
// the product path: it reproduces the structure of krylov::CudaPCG_impl
// (mochi_core/src/linear_algebra/cuda/cuda_pcg.cpp:243-525, alpha/beta kernels cuda_pcg.cu:25-42):
// FP64 3x3 BSR matrix applied with cuSPARSE bsrmv, cuBLAS dot / axpy / scal on FP64 vectors, alpha and
// beta computed by one-thread kernels on the device, iterations issued in CUDA-graph bursts of 8 with a
// host-side convergence check (||r||, residual-L2 stop) after each burst, and one solve per env after
// the other (the reference solves each island separately). What it does not include, to its advantage:
// the per-solve host-to-device copy of the matrix that LinearSolver::CudaIterativeSolve performs
// (linear_solver.h:622-624); the FP64 BSR values are converted on the device from the assembled matrix.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusparse.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdx_internal.cuh"
#include "sdx_plain.cuh"

namespace sdx {

namespace {

constexpr int kBurst = 8;

// FP64 BSR values of every env from the SELL FP32 values (pos < 0: the identity block of a padding row).
__global__ void k_sell_to_bsr64(int64_t nb, const int* __restrict__ pos, const float* __restrict__ val,
                                double* __restrict__ out) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int p = pos[b];
#pragma unroll
  for (int e = 0; e < 9; ++e)
    out[9 * b + e] = p >= 0 ? (double)val[val_index(p, e)] : ((e % 4 == 0) ? 1.0 : 0.0);
}

// Jacobi: inverse of the diagonal of each row's diagonal block (1 where it is zero).
__global__ void k_jacobi64(int64_t n_rows, const int64_t* __restrict__ diag, const double* __restrict__ v,
                           double* __restrict__ dinv) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = v[9 * diag[r] + 4 * k];
    dinv[3 * r + k] = d != 0.0 ? 1.0 / d : 1.0;
  }
}

__global__ void k_prec64(int n, const double* __restrict__ dinv, const double* __restrict__ r,
                         double* __restrict__ z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = dinv ? dinv[i] * r[i] : r[i];
}

// scalars: 0 rz, 1 rz_old, 2 pAp, 3 alpha, 4 -alpha, 5 beta (holds r.z_old first for Polak-Ribiere)
__global__ void k_alpha(double* s, int* bad) {
  s[3] = s[0] / s[2];
  s[4] = -s[3];
  if (!isfinite(s[3]) || s[3] <= 0.0) *bad = 1;
}

__global__ void k_beta(double* s) { s[5] = (s[0] - s[5]) / s[1]; }

}  // namespace

PlainSolver::~PlainSolver() {
  if (blas) cublasDestroy(blas);
  if (sparse) cusparseDestroy(sparse);
  if (descr) cusparseDestroyMatDescr(descr);
  for (void* q : {(void*)rp, (void*)col, (void*)pos, (void*)diag, (void*)val, (void*)dinv, (void*)r, (void*)z,
                  (void*)p, (void*)Ap, (void*)s, (void*)bad})
    if (q) cudaFree(q);
}

template <class T>
static int alloc_n(T** ptr, size_t n) {
  return cudaMalloc((void**)ptr, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : -1;
}

int PlainSolver::build(const PlainTopology& t) {
  n_envs = t.n_envs;
  row_off = t.row_off;
  // per env: padded rows of the env, local block CSR; rows past the env's nodes get an identity block
  std::vector<int> h_rp, h_col, h_pos;
  std::vector<int64_t> h_diag;
  env_rp_off.assign(n_envs + 1, 0);
  env_nb_off.assign(n_envs + 1, 0);
  for (int e = 0; e < n_envs; ++e) {
    const int64_t r0 = row_off[e], r1 = row_off[e + 1];
    const int64_t n0 = t.node_off[e], n1 = t.node_off[e + 1];
    env_rp_off[e] = (int64_t)h_rp.size();
    int64_t nb_local = 0;
    for (int64_t r = r0; r < r1; ++r) {
      h_rp.push_back((int)nb_local);
      const int64_t node = n0 + (r - r0);
      if (node < n1) {
        for (int64_t k = t.prow[node]; k < t.prow[node + 1]; ++k) {
          const int64_t cr = t.row_of_node[t.pcol[k]];
          if (cr == r) h_diag.push_back(env_nb_off[e] + nb_local);
          h_col.push_back((int)(cr - r0));
          h_pos.push_back(t.slice_ptr[r >> 5] + (int)(k - t.prow[node]) * kSlice + (int)(r & 31));
          ++nb_local;
        }
      } else {
        h_diag.push_back(env_nb_off[e] + nb_local);
        h_col.push_back((int)(r - r0));
        h_pos.push_back(-1);
        ++nb_local;
      }
    }
    h_rp.push_back((int)nb_local);
    env_nb_off[e + 1] = env_nb_off[e] + nb_local;
  }
  env_rp_off[n_envs] = (int64_t)h_rp.size();
  nb = env_nb_off[n_envs];
  n_rows = row_off[n_envs];
  int64_t max_rows = 0;
  for (int e = 0; e < n_envs; ++e) max_rows = std::max<int64_t>(max_rows, row_off[e + 1] - row_off[e]);
  if ((int64_t)h_diag.size() != n_rows) return -2;
  if (alloc_n(&rp, h_rp.size()) || alloc_n(&col, h_col.size()) || alloc_n(&pos, h_pos.size()) ||
      alloc_n(&diag, h_diag.size()) || alloc_n(&val, 9 * (size_t)nb) || alloc_n(&dinv, 3 * (size_t)n_rows) ||
      alloc_n(&r, 3 * (size_t)max_rows) || alloc_n(&z, 3 * (size_t)max_rows) || alloc_n(&p, 3 * (size_t)max_rows) ||
      alloc_n(&Ap, 3 * (size_t)max_rows) || alloc_n(&s, 8) || alloc_n(&bad, 1))
    return -1;
  cudaMemcpy(rp, h_rp.data(), sizeof(int) * h_rp.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(col, h_col.data(), sizeof(int) * h_col.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(pos, h_pos.data(), sizeof(int) * h_pos.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(diag, h_diag.data(), sizeof(int64_t) * h_diag.size(), cudaMemcpyHostToDevice);
  if (cublasCreate(&blas) != CUBLAS_STATUS_SUCCESS) return -3;
  if (cusparseCreate(&sparse) != CUSPARSE_STATUS_SUCCESS) return -3;
  if (cusparseCreateMatDescr(&descr) != CUSPARSE_STATUS_SUCCESS) return -3;
  cusparseSetMatType(descr, CUSPARSE_MATRIX_TYPE_GENERAL);
  cusparseSetMatIndexBase(descr, CUSPARSE_INDEX_BASE_ZERO);
  const double one_m[2] = {1.0, -1.0};
  cudaMemcpy(s + 6, one_m, sizeof(one_m), cudaMemcpyHostToDevice);  // s[6] = 1, s[7] = -1
  return 0;
}

// One burst of kBurst iterations on the current env (captured into a graph per solve, as the reference
// does), in the order of cuda_pcg.cpp's MakeGraph.
void PlainSolver::issue_burst(int n, int mb, int nnzb, const int* erp, const int* ecol, const double* evalp,
                              const double* edinv, double* x, bool pr, cudaStream_t st) {
  const double one = 1.0, zero = 0.0;
  for (int i = 0; i < kBurst; ++i) {
    cusparseDbsrmv(sparse, CUSPARSE_DIRECTION_ROW, CUSPARSE_OPERATION_NON_TRANSPOSE, mb, mb,
                   nnzb, &one, descr, evalp, erp, ecol, 3, p, &zero, Ap);
    cublasDdot(blas, n, p, 1, Ap, 1, s + 2);
    k_alpha<<<1, 1, 0, st>>>(s, bad);
    cublasDaxpy(blas, n, s + 3, p, 1, x, 1);
    cublasDaxpy(blas, n, s + 4, Ap, 1, r, 1);
    if (pr)
      cublasDdot(blas, n, r, 1, z, 1, s + 5);
    else
      cudaMemsetAsync(s + 5, 0, sizeof(double), st);
    k_prec64<<<(n + 255) / 256, 256, 0, st>>>(n, edinv, r, z);
    cudaMemcpyAsync(s + 1, s + 0, sizeof(double), cudaMemcpyDeviceToDevice, st);
    cublasDdot(blas, n, r, 1, z, 1, s + 0);
    k_beta<<<1, 1, 0, st>>>(s);
    cublasDscal(blas, n, s + 5, p, 1);
    cublasDaxpy(blas, n, s + 6, z, 1, p, 1);
  }
}

int PlainSolver::solve(const float* sell_val, const double* b_all, double* x_all, const uint8_t* h_mask,
                       const sdx_linear_params& lp, bool zero_guess, cudaStream_t st, std::vector<int>& iters,
                       std::vector<int>& conv) {
  if (lp.preconditioner == 2) return -4;  // block Jacobi is not part of this comparison arm
  k_sell_to_bsr64<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(nb, pos, sell_val, val);
  k_jacobi64<<<(unsigned)((n_rows + 255) / 256), 256, 0, st>>>(n_rows, diag, val, dinv);
  cublasSetStream(blas, st);
  cusparseSetStream(sparse, st);
  iters.assign(n_envs, 0);
  conv.assign(n_envs, 0);
  for (int e = 0; e < n_envs; ++e) {
    if (h_mask && !h_mask[e]) continue;
    const int mb = (int)(row_off[e + 1] - row_off[e]);
    const int n = 3 * mb;
    const int enb = (int)(env_nb_off[e + 1] - env_nb_off[e]);
    const int* erp = rp + env_rp_off[e];
    const int* ecol = col + env_nb_off[e];
    const double* evalp = val + 9 * env_nb_off[e];
    const double* edinv = lp.preconditioner == 1 ? dinv + 3 * row_off[e] : nullptr;
    const double* b = b_all + 3 * row_off[e];
    double* x = x_all + 3 * row_off[e];
    const double one = 1.0, mone = -1.0;
    // r = b - A x0
    cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_HOST);
    if (zero_guess) cudaMemsetAsync(x, 0, sizeof(double) * n, st);
    cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    if (!zero_guess)
      cusparseDbsrmv(sparse, CUSPARSE_DIRECTION_ROW, CUSPARSE_OPERATION_NON_TRANSPOSE, mb, mb,
                     enb, &mone, descr, evalp, erp, ecol, 3, x, &one, r);
    k_prec64<<<(n + 255) / 256, 256, 0, st>>>(n, edinv, r, z);
    double bn = 0.0, rn = 0.0;
    cublasDnrm2(blas, n, b, 1, &bn);
    cublasDnrm2(blas, n, r, 1, &rn);
    const double thr = std::max(lp.abs_tol, lp.rel_tol * bn);
    if (rn <= thr || !std::isfinite(rn)) {
      conv[e] = std::isfinite(rn) ? 1 : 3;
      continue;
    }
    cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_DEVICE);
    cublasDdot(blas, n, r, 1, z, 1, s + 0);
    cudaMemsetAsync(bad, 0, sizeof(int), st);
    // capture one burst for this env's pointers
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaStream_t cap = nullptr;
    bool graphed = false;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) == cudaSuccess) {
      cudaEvent_t ready;
      cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
      cudaEventRecord(ready, st);
      cudaStreamWaitEvent(cap, ready, 0);
      cudaEventDestroy(ready);
      cublasSetStream(blas, cap);
      cusparseSetStream(sparse, cap);
      if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        issue_burst(n, mb, enb, erp, ecol, evalp, edinv, x, lp.polak_ribiere != 0, cap);
        if (cudaStreamEndCapture(cap, &g) == cudaSuccess && g &&
            cudaGraphInstantiate(&ge, g, 0) == cudaSuccess)
          graphed = true;
        if (g) cudaGraphDestroy(g);
      }
      cudaGetLastError();
      cublasSetStream(blas, st);
      cusparseSetStream(sparse, st);
      cudaStreamDestroy(cap);
    }
    int it = 0, status = 2;
    const double div_thr = lp.rel_div_tol * bn;
    while (it < lp.max_iter) {
      if (graphed)
        cudaGraphLaunch(ge, st);
      else
        issue_burst(n, mb, enb, erp, ecol, evalp, edinv, x, lp.polak_ribiere != 0, st);
      it += kBurst;
      int hbad = 0;
      cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_HOST);
      cublasDnrm2(blas, n, r, 1, &rn);  // synchronous: the host check after each burst
      cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_DEVICE);
      if (lp.abort_if_not_spd) {
        cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost);
        if (hbad) {
          status = 3;
          break;
        }
      }
      if (!std::isfinite(rn) || rn > div_thr) {
        status = 3;
        break;
      }
      if (rn <= thr) {
        status = 1;
        break;
      }
    }
    if (ge) cudaGraphExecDestroy(ge);
    iters[e] = it;
    conv[e] = status;
  }
  cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_HOST);
  return cudaGetLastError() == cudaSuccess ? 0 : -5;
}

}  // namespace sdx
