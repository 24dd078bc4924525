// sdx_plain.cuh — the plain FP64 Jacobi-PCG comparison arm (sdx_plain.cu).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusparse.h>
#include <stdint.h>

#include <vector>

#include "../../include/sdx_b200.h"

namespace sdx {

// Host topology of the uploaded batch (owned by the context).
struct PlainTopology {
  int n_envs;
  std::vector<int64_t> row_off;   // padded rows per env (n_envs + 1)
  std::vector<int64_t> node_off;  // user nodes per env (n_envs + 1)
  const int64_t* prow;            // user block pattern (per node, sorted columns of user node ids)
  const int32_t* pcol;
  const int32_t* row_of_node;     // user node -> row
  const int* slice_ptr;           // sliced-ELL slice starts (block positions)
};

struct PlainSolver {
  int n_envs = 0;
  int64_t nb = 0, n_rows = 0;
  std::vector<int64_t> row_off, env_rp_off, env_nb_off;
  int *rp = nullptr, *col = nullptr, *pos = nullptr, *bad = nullptr;
  int64_t* diag = nullptr;
  double *val = nullptr, *dinv = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *s = nullptr;
  cublasHandle_t blas = nullptr;
  cusparseHandle_t sparse = nullptr;
  cusparseMatDescr_t descr = nullptr;

  ~PlainSolver();
  // 0 on success
  int build(const PlainTopology& t);
  // Solves every env with h_mask[e] != 0 (NULL: all); b and x in row space (3 doubles per row).
  int solve(const float* sell_val, const double* b, double* x, const uint8_t* h_mask, const sdx_linear_params& lp,
            bool zero_guess, cudaStream_t st, std::vector<int>& iters, std::vector<int>& conv);

 private:
  void issue_burst(int n, int mb, int nnzb, const int* erp, const int* ecol, const double* evalp,
                   const double* edinv, double* x, bool pr, cudaStream_t st);
};

}  // namespace sdx
