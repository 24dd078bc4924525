// sdx_mlp.cuh — parameter layout and launch wrappers of the learned warm-start MLP (sdx_mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sdx_internal.cuh"

namespace sdx {

// Flat parameter vector (FP32 master copy), row-major [out][in] weight matrices:
//   W1 128 x 16 (input 15 features + one zero pad), b1 128, W2 128 x 128, b2 128, W3 128 x 128, b3 128,
//   W4 16 x 128 (rows 0..2 used: the 3-vector output), b4 16 (entries 0..2 used).
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + 128 * 16;
constexpr int kOffW2 = kOffB1 + 128;
constexpr int kOffB2 = kOffW2 + 128 * 128;
constexpr int kOffW3 = kOffB2 + 128;
constexpr int kOffB3 = kOffW3 + 128 * 128;
constexpr int kOffW4 = kOffB3 + 128;
constexpr int kOffB4 = kOffW4 + 16 * 128;
constexpr int kMlpParams = kOffB4 + 16;

struct MlpParams {
  float* p = nullptr;           // FP32 master
  float* g = nullptr;           // gradient
  float* m = nullptr;           // Adam moments
  float* v = nullptr;
  float* pr = nullptr;          // bf16-rounded copy as FP32 (backward operands)
  __nv_bfloat16* pb = nullptr;  // bf16 copy (tensor-core operands)
  uint8_t* mask = nullptr;      // trainable entries
  int step = 0;
};

struct MlpWork {
  int cap = 0;  // rows
  float *Y = nullptr, *Z = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr, *G1 = nullptr, *G2 = nullptr,
        *G3 = nullptr, *dY = nullptr, *dA = nullptr, *dB = nullptr, *Xb = nullptr;
};

struct MlpForwardArgs {
  int n;
  const float* X;  // n x 16
  float* Y;        // n x 3
  float* Z;        // optional 3 x n x 128 pre-activations (training)
  int* error;
  const __nv_bfloat16 *W1, *W2, *W3, *W4;
  const float *b1, *b2, *b3, *b4;
  // optional (NULL: every tile): 128-row tiles whose four 32-row slices all belong to envs outside the
  // mask are skipped (their Y rows are left as they are)
  const int* slice_env;
  const uint8_t* env_mask;
};

int launch_mlp_forward(const MlpForwardArgs& a, int num_sms, cudaStream_t st);
MlpForwardArgs mlp_forward_args(const MlpParams& P, const float* X, int n, float* Y, float* Z, int* error);
void mlp_sync_bf16(const MlpParams& P, cudaStream_t st);
int mlp_gradients(const MlpParams& P, MlpWork& W, const float* X, const float* T, int n, int num_sms, double* loss,
                  int* error, cudaStream_t st);
void mlp_adam(const MlpParams& P, float lr, int step, cudaStream_t st);
void launch_features(const Matrix& A, int64_t n_rows, const uint8_t* env_mask, const double* u, const double* v,
                     double dt, const double* dx1, const double* dx2, const double* g, const int* diag_pos,
                     const uint8_t* pin, const int* env_rows, float* raw, double* sumsq, int n_envs, float* X,
                     cudaStream_t st);
void launch_warm_start(int64_t n_rows, const int* slice_env, const uint8_t* env_mask, const float* Y,
                       const uint8_t* pin, const int* diag_pos, const double* h, const double* h2,
                       const int* env_rows, double* dx, double* x2, cudaStream_t st);
void launch_targets(int64_t n_rows, const int* slice_env, const double* dx, const double* dx2, const double* h,
                    const double* h2, const int* env_rows, float* T, cudaStream_t st);

}  // namespace sdx
