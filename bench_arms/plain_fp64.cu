// plain_fp64.cu — libsdx_plain_fp64.so: the plain FP64 Jacobi-PCG, the reference's CUDA solver path
// restated on this GPU. A comparison arm of the benchmark, not part of libsdx_b200.so: the benchmark plugs
// it into sdx_step through sdx_set_linear_solver, so every Newton system of the step is solved here.
//
// It reproduces the structure of krylov::CudaPCG_impl (mochi_core/src/linear_algebra/cuda/cuda_pcg.cpp:
// 243-525, alpha/beta kernels cuda_pcg.cu:25-42): FP64 3x3 BSR matrix applied with cuSPARSE bsrmv, cuBLAS
// dot / axpy / scal on FP64 vectors, alpha and beta computed by one-thread kernels on the device,
// iterations issued in CUDA-graph bursts of 8 with a host-side convergence check (||r||, residual-L2 stop)
// after each burst, and one solve per env after the other (the reference solves each island separately).
// What it leaves out, to its advantage: the per-solve host-to-device copy of the matrix that
// LinearSolver::CudaIterativeSolve performs (linear_solver.h:622-624); the FP64 BSR values are converted on
// the device from the FP32 system the hook receives.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusparse.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../include/sdx_b200.h"

namespace {

constexpr int kBurst = 8;

__global__ void k_to_f64(int64_t n, const float* __restrict__ in, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)in[i];
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

template <class T>
int alloc_n(T** ptr, size_t n) {
  return cudaMalloc((void**)ptr, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : -1;
}

struct PlainSolver {
  int n_envs = 0;
  int64_t nb = 0, n_nodes = 0;
  std::vector<int64_t> node_off, env_nb_off;
  int *rp = nullptr, *col = nullptr, *bad = nullptr;  // per env local block CSR, concatenated
  int64_t* diag = nullptr;
  double *val = nullptr, *dinv = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *s = nullptr;
  cublasHandle_t blas = nullptr;
  cusparseHandle_t sparse = nullptr;
  cusparseMatDescr_t descr = nullptr;

  ~PlainSolver() {
    if (blas) cublasDestroy(blas);
    if (sparse) cusparseDestroy(sparse);
    if (descr) cusparseDestroyMatDescr(descr);
    for (void* q : {(void*)rp, (void*)col, (void*)diag, (void*)val, (void*)dinv, (void*)r, (void*)z, (void*)p,
                    (void*)Ap, (void*)s, (void*)bad})
      if (q) cudaFree(q);
  }

  // Local BSR structure of every env from the system's global pattern (columns stay inside the env).
  int build(const sdx_device_system& sys) {
    n_envs = sys.n_envs;
    n_nodes = sys.n_nodes;
    nb = sys.nnzb;
    node_off.assign(sys.node_offsets, sys.node_offsets + n_envs + 1);
    std::vector<int64_t> grp(n_nodes + 1);
    std::vector<int32_t> gcol(nb);
    if (cudaMemcpy(grp.data(), sys.row_ptr, sizeof(int64_t) * (n_nodes + 1), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(gcol.data(), sys.col, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost) != cudaSuccess)
      return -5;
    std::vector<int> h_rp, h_col;
    std::vector<int64_t> h_diag(n_nodes, -1);
    env_nb_off.assign(n_envs + 1, 0);
    for (int e = 0; e < n_envs; ++e) {
      const int64_t n0 = node_off[e], n1 = node_off[e + 1];
      env_nb_off[e] = grp[n0];
      for (int64_t i = n0; i <= n1; ++i) h_rp.push_back((int)(grp[i] - grp[n0]));
      for (int64_t i = n0; i < n1; ++i)
        for (int64_t k = grp[i]; k < grp[i + 1]; ++k) {
          if (gcol[k] < n0 || gcol[k] >= n1) return -2;
          if (gcol[k] == i) h_diag[i] = k;
        }
    }
    env_nb_off[n_envs] = nb;
    h_col.resize(nb);
    for (int e = 0; e < n_envs; ++e)
      for (int64_t k = grp[node_off[e]]; k < grp[node_off[e + 1]]; ++k) h_col[k] = (int)(gcol[k] - node_off[e]);
    for (int64_t i = 0; i < n_nodes; ++i)
      if (h_diag[i] < 0) return -2;
    int64_t max_nodes = 0;
    for (int e = 0; e < n_envs; ++e) max_nodes = std::max<int64_t>(max_nodes, node_off[e + 1] - node_off[e]);
    if (alloc_n(&rp, h_rp.size()) || alloc_n(&col, h_col.size()) || alloc_n(&diag, h_diag.size()) ||
        alloc_n(&val, 9 * (size_t)nb) || alloc_n(&dinv, 3 * (size_t)n_nodes) || alloc_n(&r, 3 * (size_t)max_nodes) ||
        alloc_n(&z, 3 * (size_t)max_nodes) || alloc_n(&p, 3 * (size_t)max_nodes) ||
        alloc_n(&Ap, 3 * (size_t)max_nodes) || alloc_n(&s, 8) || alloc_n(&bad, 1))
      return -1;
    cudaMemcpy(rp, h_rp.data(), sizeof(int) * h_rp.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(col, h_col.data(), sizeof(int) * h_col.size(), cudaMemcpyHostToDevice);
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
  void issue_burst(int n, int mb, int nnzb, const int* erp, const int* ecol, const double* evalp,
                   const double* edinv, double* x, bool pr, cudaStream_t st) {
    const double one = 1.0, zero = 0.0;
    for (int i = 0; i < kBurst; ++i) {
      cusparseDbsrmv(sparse, CUSPARSE_DIRECTION_ROW, CUSPARSE_OPERATION_NON_TRANSPOSE, mb, mb, nnzb, &one, descr,
                     evalp, erp, ecol, 3, p, &zero, Ap);
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

  int solve(const sdx_device_system& sys, const sdx_linear_params& lp, int* iters) {
    if (lp.preconditioner == SDX_PREC_BLOCK_JACOBI) return SDX_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)sys.stream;
    k_to_f64<<<(unsigned)((9 * nb + 255) / 256), 256, 0, st>>>(9 * nb, sys.values, val);
    k_jacobi64<<<(unsigned)((n_nodes + 255) / 256), 256, 0, st>>>(n_nodes, diag, val, dinv);
    cublasSetStream(blas, st);
    cusparseSetStream(sparse, st);
    const bool zero_guess = sys.zero_guess != 0;
    for (int e = 0; e < n_envs; ++e) {
      if (sys.env_mask && !sys.env_mask[e]) continue;
      const int mb = (int)(node_off[e + 1] - node_off[e]);
      const int n = 3 * mb;
      const int enb = (int)(env_nb_off[e + 1] - env_nb_off[e]);
      const int* erp = rp + node_off[e] + e;  // env e's local row pointers (mb + 1 of them)
      const int* ecol = col + env_nb_off[e];
      const double* evalp = val + 9 * env_nb_off[e];
      const double* edinv = lp.preconditioner == SDX_PREC_JACOBI ? dinv + 3 * node_off[e] : nullptr;
      const double* b = sys.b + 3 * node_off[e];
      double* x = sys.x + 3 * node_off[e];
      const double one = 1.0, mone = -1.0;
      // r = b - A x0
      cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_HOST);
      if (zero_guess) cudaMemsetAsync(x, 0, sizeof(double) * n, st);
      cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
      if (!zero_guess)
        cusparseDbsrmv(sparse, CUSPARSE_DIRECTION_ROW, CUSPARSE_OPERATION_NON_TRANSPOSE, mb, mb, enb, &mone, descr,
                       evalp, erp, ecol, 3, x, &one, r);
      k_prec64<<<(n + 255) / 256, 256, 0, st>>>(n, edinv, r, z);
      double bn = 0.0, rn = 0.0;
      cublasDnrm2(blas, n, b, 1, &bn);
      cublasDnrm2(blas, n, r, 1, &rn);
      const double thr = std::max(lp.abs_tol, lp.rel_tol * bn);
      if (rn <= thr || !std::isfinite(rn)) {
        iters[e] = 0;
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
          if (cudaStreamEndCapture(cap, &g) == cudaSuccess && g && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess)
            graphed = true;
          if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        cublasSetStream(blas, st);
        cusparseSetStream(sparse, st);
        cudaStreamDestroy(cap);
      }
      int it = 0;
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
          if (hbad) break;
        }
        if (!std::isfinite(rn) || rn > div_thr || rn <= thr) break;
      }
      if (ge) cudaGraphExecDestroy(ge);
      iters[e] = it;
    }
    cublasSetPointerMode(blas, CUBLAS_POINTER_MODE_HOST);
    return cudaGetLastError() == cudaSuccess ? SDX_OK : SDX_ERR_CUDA;
  }
};

}  // namespace

extern "C" {

// A solver instance for one sdx_context (its structure is built on the first solve).
void* sdx_plain_fp64_create(void) { return new PlainSolver(); }

void sdx_plain_fp64_destroy(void* h) { delete static_cast<PlainSolver*>(h); }

// The sdx_linear_solve_fn hook: user = a handle from sdx_plain_fp64_create.
int sdx_plain_fp64_solve(void* user, const sdx_device_system* sys, const sdx_linear_params* lp, int* iters) {
  PlainSolver* ps = static_cast<PlainSolver*>(user);
  if (!ps || !sys || !lp || !iters) return SDX_ERR_INVALID_ARGUMENT;
  if (ps->n_envs == 0) {
    const int rc = ps->build(*sys);
    if (rc != 0) return rc == -1 ? SDX_ERR_OUT_OF_MEMORY : SDX_ERR_CUDA;
  } else if (ps->n_envs != sys->n_envs || ps->nb != sys->nnzb) {
    return SDX_ERR_INVALID_ARGUMENT;  // one instance per uploaded batch
  }
  return ps->solve(*sys, *lp, iters);
}

}  // extern "C"
