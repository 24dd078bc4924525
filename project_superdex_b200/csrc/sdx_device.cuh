// sdx_device.cuh — device math for the soft-body step (sm_100a).
//
// Smith et al. 2018 stable Neo-Hookean, as in the reference's
// mochi_core/src/materials/batched_smith_neo_hookean.cpp:29-269:
//   * energy and first Piola-Kirchhoff stress in FP64 (they feed the Newton residual and the
//     line-search residual norms, whose stopping test at rel 1e-6 needs FP64);
//   * the 9x9 tangent in FP32 (it only feeds the FP32 block Hessian), with the PSD projection done by
//     clamping the analytic eigensystem (scaling / twist / flip modes) of the tangent.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sdx {

// ------------------------------------------------------------------------------------------------
// small dense helpers (row-major 3x3)

template <class T>
__device__ __forceinline__ T det3(const T F[9]) {
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

// cof(F)_ij = dJ/dF_ij
template <class T>
__device__ __forceinline__ void cof3(const T F[9], T C[9]) {
  C[0] = F[4] * F[8] - F[5] * F[7];
  C[1] = F[5] * F[6] - F[3] * F[8];
  C[2] = F[3] * F[7] - F[4] * F[6];
  C[3] = F[2] * F[7] - F[1] * F[8];
  C[4] = F[0] * F[8] - F[2] * F[6];
  C[5] = F[1] * F[6] - F[0] * F[7];
  C[6] = F[1] * F[5] - F[2] * F[4];
  C[7] = F[2] * F[3] - F[0] * F[5];
  C[8] = F[0] * F[4] - F[1] * F[3];
}

// Levi-Civita sign of distinct (a, b, c) in {0,1,2}.
__host__ __device__ constexpr int levi(int a, int b, int c) {
  return (a == b || b == c || a == c) ? 0 : (((b - a + 3) % 3) == 1 ? 1 : -1);
}

// Entry (ab) of the 9x9 Hessian of J = det F: d2J/dF_ij dF_kl = eps_ikn eps_jlq F_nq, i.e. a single
// signed entry of F when i != k and j != l (material_utils.h:182-218 writes the same skew blocks).
__host__ __device__ constexpr int hj_sign(int a, int b) {
  return ((a / 3) == (b / 3) || (a % 3) == (b % 3))
             ? 0
             : levi(a / 3, b / 3, 3 - a / 3 - b / 3) * levi(a % 3, b % 3, 3 - a % 3 - b % 3);
}
__host__ __device__ constexpr int hj_index(int a, int b) {
  return (3 - a / 3 - b / 3) * 3 + (3 - a % 3 - b % 3);
}

// ------------------------------------------------------------------------------------------------
// FP64 energy + PK1 (batched_smith_neo_hookean.cpp:46-69, 127-136)

struct SnhConsts {
  double muHat, lambdaHat, alpha;
};

__device__ __forceinline__ SnhConsts snh_consts(double mu, double lambda) {
  SnhConsts c;
  c.muHat = mu * (4.0 / 3.0);
  c.lambdaHat = lambda + mu * (5.0 / 6.0);
  c.alpha = 1.0 + 0.75 * c.muHat / c.lambdaHat;
  return c;
}

__device__ __forceinline__ void snh_pk1_f64(const SnhConsts& k, const double F[9], double P[9]) {
  double Ic = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) Ic = fma(F[i], F[i], Ic);
  const double J = det3(F);
  double cof[9];
  cof3(F, cof);
  const double c0 = k.muHat * (1.0 - 1.0 / (Ic + 1.0));
  const double c1 = k.lambdaHat * (J - k.alpha);
#pragma unroll
  for (int i = 0; i < 9; ++i) P[i] = c0 * F[i] + c1 * cof[i];
}

__device__ __forceinline__ double snh_energy_f64(const SnhConsts& k, const double F[9]) {
  double Ic = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) Ic = fma(F[i], F[i], Ic);
  const double Jma = det3(F) - k.alpha;
  return 0.5 * k.muHat * (Ic - 3.0) + 0.5 * k.lambdaHat * Jma * Jma - 0.5 * k.muHat * log(Ic + 1.0);
}

// ------------------------------------------------------------------------------------------------
// FP32 symmetric 3x3 eigen-decomposition (cyclic Jacobi rotations).
// In: A (row-major, symmetric). Out: w (eigenvalues), V columns = eigenvectors (V[r*3+c]).

__device__ __forceinline__ void jacobi_rot(float A[9], float V[9], int p, int q) {
  const float apq = A[p * 3 + q];
  if (fabsf(apq) < 1e-30f) return;
  const float theta = (A[q * 3 + q] - A[p * 3 + p]) / (2.0f * apq);
  const float t = copysignf(1.0f, theta) / (fabsf(theta) + sqrtf(fmaf(theta, theta, 1.0f)));
  const float c = rsqrtf(fmaf(t, t, 1.0f));
  const float s = t * c;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float akp = A[k * 3 + p], akq = A[k * 3 + q];
    A[k * 3 + p] = c * akp - s * akq;
    A[k * 3 + q] = s * akp + c * akq;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float apk = A[p * 3 + k], aqk = A[q * 3 + k];
    A[p * 3 + k] = c * apk - s * aqk;
    A[q * 3 + k] = s * apk + c * aqk;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float vkp = V[k * 3 + p], vkq = V[k * 3 + q];
    V[k * 3 + p] = c * vkp - s * vkq;
    V[k * 3 + q] = s * vkp + c * vkq;
  }
}

__device__ __forceinline__ void sym_eig3(const float Ain[9], float w[3], float V[9]) {
  float A[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) A[i] = Ain[i];
#pragma unroll
  for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? 1.0f : 0.0f;
  for (int sweep = 0; sweep < 8; ++sweep) {
    const float off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    const float dg = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
    if (off <= 1e-14f * dg) break;
    jacobi_rot(A, V, 0, 1);
    jacobi_rot(A, V, 0, 2);
    jacobi_rot(A, V, 1, 2);
  }
  w[0] = A[0];
  w[1] = A[4];
  w[2] = A[8];
}

// Rotation-variant SVD F = U diag(s) V^T with det U = det V = +1 and s[2] < 0 iff det F < 0
// (the convention of the reference's BatchedRotationVariantSvd3x3). V from the eigenvectors of F^T F
// sorted by decreasing eigenvalue; U from F V with Gram-Schmidt and a cross product.
__device__ __forceinline__ void svd3_rv(const float F[9], float U[9], float s[3], float V[9]) {
  float S[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      S[i * 3 + j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] + F[2 * 3 + i] * F[2 * 3 + j];
  float w[3];
  sym_eig3(S, w, V);
  // sort descending (3-element network), swapping V columns alongside
#define SDX_SWAP_COL(a, b)                                   \
  {                                                          \
    float tw = w[a];                                         \
    w[a] = w[b];                                             \
    w[b] = tw;                                               \
    _Pragma("unroll") for (int r = 0; r < 3; ++r) {          \
      float tv = V[r * 3 + a];                               \
      V[r * 3 + a] = V[r * 3 + b];                           \
      V[r * 3 + b] = tv;                                     \
    }                                                        \
  }
  if (w[0] < w[1]) SDX_SWAP_COL(0, 1);
  if (w[0] < w[2]) SDX_SWAP_COL(0, 2);
  if (w[1] < w[2]) SDX_SWAP_COL(1, 2);
#undef SDX_SWAP_COL
  // det V = +1
  const float dv = det3(V);
  if (dv < 0.0f) {
    V[2] = -V[2];
    V[5] = -V[5];
    V[8] = -V[8];
  }
  float fv[3][3];  // F v_k
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      fv[k][r] = F[r * 3 + 0] * V[0 * 3 + k] + F[r * 3 + 1] * V[1 * 3 + k] + F[r * 3 + 2] * V[2 * 3 + k];
  float u0[3], u1[3], u2[3];
  float n0 = sqrtf(fv[0][0] * fv[0][0] + fv[0][1] * fv[0][1] + fv[0][2] * fv[0][2]);
  if (n0 > 1e-30f) {
    u0[0] = fv[0][0] / n0;
    u0[1] = fv[0][1] / n0;
    u0[2] = fv[0][2] / n0;
  } else {
    u0[0] = 1.0f;
    u0[1] = 0.0f;
    u0[2] = 0.0f;
  }
  float d01 = u0[0] * fv[1][0] + u0[1] * fv[1][1] + u0[2] * fv[1][2];
  u1[0] = fv[1][0] - d01 * u0[0];
  u1[1] = fv[1][1] - d01 * u0[1];
  u1[2] = fv[1][2] - d01 * u0[2];
  float n1 = sqrtf(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  if (n1 > 1e-6f * fmaxf(n0, 1e-30f)) {
    u1[0] /= n1;
    u1[1] /= n1;
    u1[2] /= n1;
  } else {
    // any unit vector orthogonal to u0
    float a[3] = {fabsf(u0[0]) < 0.9f ? 1.0f : 0.0f, fabsf(u0[0]) < 0.9f ? 0.0f : 1.0f, 0.0f};
    float dd = a[0] * u0[0] + a[1] * u0[1] + a[2] * u0[2];
    u1[0] = a[0] - dd * u0[0];
    u1[1] = a[1] - dd * u0[1];
    u1[2] = a[2] - dd * u0[2];
    float nn = rsqrtf(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    u1[0] *= nn;
    u1[1] *= nn;
    u1[2] *= nn;
  }
  u2[0] = u0[1] * u1[2] - u0[2] * u1[1];
  u2[1] = u0[2] * u1[0] - u0[0] * u1[2];
  u2[2] = u0[0] * u1[1] - u0[1] * u1[0];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    U[r * 3 + 0] = u0[r];
    U[r * 3 + 1] = u1[r];
    U[r * 3 + 2] = u2[r];
  }
  s[0] = u0[0] * fv[0][0] + u0[1] * fv[0][1] + u0[2] * fv[0][2];
  s[1] = u1[0] * fv[1][0] + u1[1] * fv[1][1] + u1[2] * fv[1][2];
  s[2] = u2[0] * fv[2][0] + u2[1] * fv[2][1] + u2[2] * fv[2][2];
}

// ------------------------------------------------------------------------------------------------
// Projected tangent of an isotropic energy from its analytic eigensystem (Smith et al. 2018; Kim and
// Eberle, "Analytic Eigensystems for Isotropic Distortion Energies"): F = U diag(s) V^T; the 9 modes are
// the 3 scaling modes U diag(q_i) V^T (q_i the eigenvectors of the 3x3 scaling matrix A), the twists
// (u_j v_k^T - u_k v_j^T)/sqrt(2) and the flips (u_j v_k^T + u_k v_j^T)/sqrt(2) for the pairs
// (j,k) = (1,2), (0,2), (0,1). Eigenvalues are clamped at min_eig (psd 1) or |l| then min_eig (psd 2).

// The element stiffness is never formed as a 9x9 tangent: every 3x3 block K_fg = vol B_f^T C B_g of
// fem::StressWork (fem_stress.h:218-241) is evaluated from a factored form of the tangent C = dP/dF and the
// shape-function gradients d_f, d_g of the two nodes (TanForm, tan_block). Kinds:
//   kTanModal   C = sum_i l_i m_i m_i^T over the 9 modes above (eigenvalues clamped):
//               K_fg = U H(y_f, y_g) U^T with y = V^T d, H_ab = Ah_ab y_f[a] y_g[b] for the scaling block
//               Ah = Va diag(l_a) Va^T, and per pair (j, k) of twist l_t / flip l_f with sp = (l_t + l_f) / 2,
//               sm = (l_f - l_t) / 2: H_jj += sp y_f[k] y_g[k], H_kk += sp y_f[j] y_g[j],
//               H_jk += sm y_f[k] y_g[j], H_kj += sm y_f[j] y_g[k]; plus c_iso (d_f . d_g) I (ARAP's mu I);
//   kTanSnh     the direct Smith Neo-Hookean tangent c3 F (x) F + lambdaHat cof (x) cof + c2 I + d2c d2J/dF2:
//               K_fg = c3 a_f a_g^T + lambdaHat b_f b_g^T + c2 (d_f . d_g) I + d2c [F (d_f x d_g)]_x with
//               a = F d, b = cof(F) d and [z]_x_rc = eps_rcx z_x;
//   kTanStvk    the direct St. Venant-Kirchhoff tangent: K_fg = lambda a_f a_g^T + mu a_g a_f^T + (d_g^T S d_f) I
//               + mu (d_f . d_g) F F^T;
//   kTanLinear  K_fg = mu (d_f . d_g) I + mu d_g d_f^T + lambda d_f d_g^T.
// The register footprint is a few dozen floats instead of the 81 of C (and 81 more for the modes).
constexpr int kTanModal = 0, kTanSnh = 1, kTanStvk = 2, kTanLinear = 3;

struct TanForm {
  int kind;
  float c0, c1, c2, c3;  // Snh: c3, lambdaHat, c2, d2c; Stvk: lambda, mu; Linear: mu, lambda; Modal: c_iso
  float q0[9];           // Modal: U; Snh / Stvk: F
  float q1[9];           // Modal: V; Snh: cof F; Stvk: S
  float q2[6];           // Modal: Ah (00, 11, 22, 12, 02, 01); Stvk: F F^T (same order)
  float sp[3], sm[3];    // Modal: pair coefficients
};

__device__ __forceinline__ void mat3_vec(const float M[9], const float d[3], float o[3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) o[r] = M[r * 3 + 0] * d[0] + M[r * 3 + 1] * d[1] + M[r * 3 + 2] * d[2];
}

__device__ __forceinline__ void mat3t_vec(const float M[9], const float d[3], float o[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) o[c] = M[0 * 3 + c] * d[0] + M[1 * 3 + c] * d[1] + M[2 * 3 + c] * d[2];
}

// K (row-major 3x3, without the volume factor) of the node pair (f, g) with gradients df, dg.
__device__ __forceinline__ void tan_block(const TanForm& T, const float df[3], const float dg[3], float K[9]) {
  const float dd = df[0] * dg[0] + df[1] * dg[1] + df[2] * dg[2];
  if (T.kind == kTanModal) {
    float yf[3], yg[3];
    mat3t_vec(T.q1, df, yf);
    mat3t_vec(T.q1, dg, yg);
    float H[9];
    H[0] = T.q2[0] * yf[0] * yg[0];
    H[4] = T.q2[1] * yf[1] * yg[1];
    H[8] = T.q2[2] * yf[2] * yg[2];
    H[5] = T.q2[3] * yf[1] * yg[2];
    H[7] = T.q2[3] * yf[2] * yg[1];
    H[2] = T.q2[4] * yf[0] * yg[2];
    H[6] = T.q2[4] * yf[2] * yg[0];
    H[1] = T.q2[5] * yf[0] * yg[1];
    H[3] = T.q2[5] * yf[1] * yg[0];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const int j = (n == 0) ? 1 : 0;
      const int k = (n == 2) ? 1 : 2;
      H[j * 3 + j] += T.sp[n] * yf[k] * yg[k];
      H[k * 3 + k] += T.sp[n] * yf[j] * yg[j];
      H[j * 3 + k] += T.sm[n] * yf[k] * yg[j];
      H[k * 3 + j] += T.sm[n] * yf[j] * yg[k];
    }
    float HU[9];  // H U^T
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        HU[a * 3 + c] = H[a * 3 + 0] * T.q0[c * 3 + 0] + H[a * 3 + 1] * T.q0[c * 3 + 1] + H[a * 3 + 2] * T.q0[c * 3 + 2];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        K[r * 3 + c] = T.q0[r * 3 + 0] * HU[0 * 3 + c] + T.q0[r * 3 + 1] * HU[1 * 3 + c] + T.q0[r * 3 + 2] * HU[2 * 3 + c] +
                       (r == c ? T.c0 * dd : 0.0f);
  } else if (T.kind == kTanSnh) {
    float af[3], ag[3], bf[3], bg[3], w[3], z[3];
    mat3_vec(T.q0, df, af);
    mat3_vec(T.q0, dg, ag);
    mat3_vec(T.q1, df, bf);
    mat3_vec(T.q1, dg, bg);
    w[0] = df[1] * dg[2] - df[2] * dg[1];
    w[1] = df[2] * dg[0] - df[0] * dg[2];
    w[2] = df[0] * dg[1] - df[1] * dg[0];
    mat3_vec(T.q0, w, z);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) K[r * 3 + c] = T.c0 * af[r] * ag[c] + T.c1 * bf[r] * bg[c] + (r == c ? T.c2 * dd : 0.0f);
    K[1] += T.c3 * z[2];
    K[2] -= T.c3 * z[1];
    K[3] -= T.c3 * z[2];
    K[5] += T.c3 * z[0];
    K[6] += T.c3 * z[1];
    K[7] -= T.c3 * z[0];
  } else if (T.kind == kTanStvk) {
    float af[3], ag[3], sf[3];
    mat3_vec(T.q0, df, af);
    mat3_vec(T.q0, dg, ag);
    mat3_vec(T.q1, df, sf);
    const float dsd = dg[0] * sf[0] + dg[1] * sf[1] + dg[2] * sf[2];
    const float FFt[9] = {T.q2[0], T.q2[5], T.q2[4], T.q2[5], T.q2[1], T.q2[3], T.q2[4], T.q2[3], T.q2[2]};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        K[r * 3 + c] = T.c0 * af[r] * ag[c] + T.c1 * ag[r] * af[c] + T.c1 * dd * FFt[r * 3 + c] + (r == c ? dsd : 0.0f);
  } else {  // kTanLinear
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        K[r * 3 + c] = T.c0 * dg[r] * df[c] + T.c1 * df[r] * dg[c] + (r == c ? T.c0 * dd : 0.0f);
  }
}

// Modal form from the SVD F = U diag(s) V^T, the 3x3 scaling block A (singular basis) and the twist / flip
// eigenvalues, every eigenvalue clamped at min_eig (psd 1) or |l| then min_eig (psd 2).
__device__ __forceinline__ void modal_tanform(const float U[9], const float V[9], const float A[9], const float tw[3],
                                              const float fl[3], int psd, float min_eig, TanForm& T) {
  float wa[3], Va[9];
  sym_eig3(A, wa, Va);
  auto clamp = [&](float l) { return fmaxf(psd == 2 ? fabsf(l) : l, min_eig); };
#pragma unroll
  for (int i = 0; i < 3; ++i) wa[i] = clamp(wa[i]);
  auto ah = [&](int a, int b) { return Va[a * 3 + 0] * wa[0] * Va[b * 3 + 0] + Va[a * 3 + 1] * wa[1] * Va[b * 3 + 1] +
                                       Va[a * 3 + 2] * wa[2] * Va[b * 3 + 2]; };
  T.kind = kTanModal;
  T.c0 = 0.0f;
  T.q2[0] = ah(0, 0);
  T.q2[1] = ah(1, 1);
  T.q2[2] = ah(2, 2);
  T.q2[3] = ah(1, 2);
  T.q2[4] = ah(0, 2);
  T.q2[5] = ah(0, 1);
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const float lt = clamp(tw[n]), lf = clamp(fl[n]);
    T.sp[n] = 0.5f * (lt + lf);
    T.sm[n] = 0.5f * (lf - lt);
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    T.q0[i] = U[i];
    T.q1[i] = V[i];
  }
}

// ------------------------------------------------------------------------------------------------
// FP32 tangent dP/dF in factored form (TanForm) with the reference's PSD handling.
// psd: 0 none, 1 projection (max(l, eps)), 2 |l| projection, 3 fast (drop d2J when indefinite).

__device__ __forceinline__ void snh_tanform(float mu, float lambda, const float F[9], int project,
                                            int psd, float min_eig, TanForm& T) {
  const float muHat = mu * (4.0f / 3.0f);
  const float lambdaHat = lambda + mu * (5.0f / 6.0f);
  const float alpha = 1.0f + 0.75f * muHat / lambdaHat;
  float Ic = 0.0f;
#pragma unroll
  for (int i = 0; i < 9; ++i) Ic = fmaf(F[i], F[i], Ic);
  const float IcPlus1 = Ic + 1.0f, IcPlus1Inv = 1.0f / IcPlus1;
  const float J = det3(F), Jma = J - alpha;
  const float c2 = muHat * (1.0f - IcPlus1Inv);
  const float c3 = 2.0f * muHat * IcPlus1Inv * IcPlus1Inv;

  bool projecting = project && psd != 0;
  if (projecting) {
    // PSD oracle "Correct" (batched_smith_neo_hookean.cpp:81-104). The conservative bound Ic >=
    // max sigma^2 decides cheaply when it proves definiteness; otherwise the SVD values decide.
    const float muHatK2 = c2 * c2;
    const float lhsBase = (lambdaHat * Jma) * (lambdaHat * Jma);
    bool indefinite = (J < 0.0f) || (lhsBase * Ic > muHatK2);
    if (indefinite && J >= 0.0f) {
      float S[9], w[3], Vt[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          S[i * 3 + j] = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];
      sym_eig3(S, w, Vt);
      const float maxs2 = fmaxf(w[0], fmaxf(w[1], w[2]));
      indefinite = lhsBase * maxs2 > muHatK2;
    }
    projecting = indefinite;
  }

  if (projecting && (psd == 1 || psd == 2)) {
    // Eigensystem path (batched_smith_neo_hookean.cpp:141-203, Smith et al. 2018).
    float U[9], s[3], V[9];
    svd3_rv(F, U, s, V);
    const float coeff0 = muHat - muHat * IcPlus1Inv;
    const float coeff1 = lambdaHat * Jma;
    float tw[3], fl[3];
    tw[0] = coeff1 * s[0] + coeff0;  // twist, pair (1,2)
    tw[1] = coeff1 * s[1] + coeff0;  // twist, pair (0,2)
    tw[2] = coeff1 * s[2] + coeff0;  // twist, pair (0,1)
    fl[0] = -coeff1 * s[0] + coeff0; // flip
    fl[1] = -coeff1 * s[1] + coeff0;
    fl[2] = -coeff1 * s[2] + coeff0;
    const float Ic2inv = IcPlus1Inv * IcPlus1Inv;
    const float mu2 = 2.0f * muHat;
    const float J2al = (2.0f * J - alpha) * lambdaHat;
    const float s0 = s[0] * s[0], s1 = s[1] * s[1], s2 = s[2] * s[2];
    float A[9];
    A[0] = (mu2 * s0 - muHat * IcPlus1) * Ic2inv + lambdaHat * s1 * s2 + muHat;
    A[4] = (mu2 * s1 - muHat * IcPlus1) * Ic2inv + lambdaHat * s0 * s2 + muHat;
    A[8] = (mu2 * s2 - muHat * IcPlus1) * Ic2inv + lambdaHat * s0 * s1 + muHat;
    A[1] = A[3] = J2al * s[2] + mu2 * s[0] * s[1] * Ic2inv;
    A[2] = A[6] = J2al * s[1] + mu2 * s[0] * s[2] * Ic2inv;
    A[5] = A[7] = J2al * s[0] + mu2 * s[1] * s[2] * Ic2inv;
    modal_tanform(U, V, A, tw, fl, psd, min_eig, T);
    return;
  }

  // Direct tangent (batched_smith_neo_hookean.cpp:204-266): c3 F (x) F + lambdaHat cof (x) cof + c2 I +
  // d2c d2J/dF2 (the last dropped by the fast strategy when indefinite).
  T.kind = kTanSnh;
  cof3(F, T.q1);
#pragma unroll
  for (int i = 0; i < 9; ++i) T.q0[i] = F[i];
  T.c0 = c3;
  T.c1 = lambdaHat;
  T.c2 = c2;
  T.c3 = (projecting && psd == 3) ? 0.0f : lambdaHat * Jma;
}

// ------------------------------------------------------------------------------------------------
// St. Venant-Kirchhoff (mochi_core/src/materials/batched_st_venant_kirchhoff.cpp:29-203) and linear
// elasticity (batched_linear_elastic.cpp:25-97): FP64 energy and PK1, FP32 tangent.

__device__ __forceinline__ void stvk_green(const double F[9], double G[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      G[i * 3 + j] = 0.5 * (F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j] - (i == j ? 1.0 : 0.0));
}

// psi = mu |G|^2 + lambda/2 tr(G)^2 ; P = F (2 mu G + lambda tr(G) I)
__device__ __forceinline__ void stvk_energy_pk1_f64(double mu, double lambda, const double F[9], double* energy,
                                                    double P[9]) {
  double G[9];
  stvk_green(F, G);
  const double trG = G[0] + G[4] + G[8];
  if (energy) {
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) n2 += G[i] * G[i];
    *energy = mu * n2 + 0.5 * lambda * trG * trG;
  }
  if (P) {
    double S[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) S[i] = 2.0 * mu * G[i] + ((i % 4 == 0) ? lambda * trG : 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        P[r * 3 + c] = F[r * 3 + 0] * S[c] + F[r * 3 + 1] * S[3 + c] + F[r * 3 + 2] * S[6 + c];
  }
}

__device__ __forceinline__ void stvk_tanform(float mu, float lambda, const float F[9], int project, int psd,
                                             float min_eig, TanForm& T) {
  if (project && (psd == 1 || psd == 2)) {
    // eigensystem (batched_st_venant_kirchhoff.cpp:96-154): base = -mu + lambda (I2 - 3) / 2
    float U[9], s[3], V[9];
    svd3_rv(F, U, s, V);
    const float s0 = s[0] * s[0], s1 = s[1] * s[1], s2 = s[2] * s[2];
    const float base = -mu + 0.5f * lambda * (s0 + s1 + s2 - 3.0f);
    float tw[3], fl[3];
    tw[0] = base + mu * (s1 + s2 - s[1] * s[2]);
    tw[1] = base + mu * (s0 + s2 - s[0] * s[2]);
    tw[2] = base + mu * (s0 + s1 - s[0] * s[1]);
    fl[0] = base + mu * (s1 + s2 + s[1] * s[2]);
    fl[1] = base + mu * (s0 + s2 + s[0] * s[2]);
    fl[2] = base + mu * (s0 + s1 + s[0] * s[1]);
    const float dc = lambda + 3.0f * mu;
    float A[9];
    A[0] = base + dc * s0;
    A[4] = base + dc * s1;
    A[8] = base + dc * s2;
    A[1] = A[3] = lambda * s[0] * s[1];
    A[2] = A[6] = lambda * s[0] * s[2];
    A[5] = A[7] = lambda * s[1] * s[2];
    modal_tanform(U, V, A, tw, fl, psd, min_eig, T);
    return;
  }
  // direct tangent dP_rc/dF_ij = delta_ri S_jc + mu F_rj F_ic + mu delta_jc (F F^T)_ri + lambda F_ij F_rc
  // (:156-197); Fast (psd 3) keeps only the non-negative stretches of G inside S
  float G[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      G[i * 3 + j] = 0.5f * (F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j] - (i == j ? 1.0f : 0.0f));
  if (project && psd == 3) {
#pragma unroll
    for (int i = 0; i < 9; ++i) G[i] = (i % 4 == 0) ? fmaxf(G[i], 0.0f) : 0.0f;
  }
  const float trG = G[0] + G[4] + G[8];
  T.kind = kTanStvk;
  T.c0 = lambda;
  T.c1 = mu;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    T.q0[i] = F[i];
    T.q1[i] = 2.0f * mu * G[i] + ((i % 4 == 0) ? lambda * trG : 0.0f);  // S
  }
  auto fft = [&](int r, int i) { return F[r * 3 + 0] * F[i * 3 + 0] + F[r * 3 + 1] * F[i * 3 + 1] + F[r * 3 + 2] * F[i * 3 + 2]; };
  T.q2[0] = fft(0, 0);
  T.q2[1] = fft(1, 1);
  T.q2[2] = fft(2, 2);
  T.q2[3] = fft(1, 2);
  T.q2[4] = fft(0, 2);
  T.q2[5] = fft(0, 1);
}

// eps = (F + F^T)/2 - I ; psi = mu eps:eps + lambda/2 tr(eps)^2 ; P = 2 mu eps + lambda tr(eps) I
__device__ __forceinline__ void linear_energy_pk1_f64(double mu, double lambda, const double F[9], double* energy,
                                                      double P[9]) {
  double e[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) e[r * 3 + c] = 0.5 * (F[r * 3 + c] + F[c * 3 + r]) - (r == c ? 1.0 : 0.0);
  const double tr = e[0] + e[4] + e[8];
  if (energy) {
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) n2 += e[i] * e[i];
    *energy = mu * n2 + 0.5 * lambda * tr * tr;
  }
  if (P) {
#pragma unroll
    for (int i = 0; i < 9; ++i) P[i] = 2.0 * mu * e[i] + ((i % 4 == 0) ? lambda * tr : 0.0);
  }
}

// constant, PSD: dP_rc/dF_ij = mu (d_ri d_cj + d_ci d_rj) + lambda d_rc d_ij
// ------------------------------------------------------------------------------------------------
// As-rigid-as-possible (batched_arap.cpp:29-136): energy 1/2 mu |s - 1|^2 over the rotation-variant
// singular values, PK1 mu (F - U V^T), tangent mu I + sum_n l_n T_n (x) T_n over the twist modes
// T_n = u_k v_j^T - u_j v_k^T with l_n = -mu / (s_j + s_k) (the exact Hessian), the twist eigenvalues
// mu + 2 l_n clamped under projection (the other six are mu).

// FP64 symmetric 3x3 eigen-decomposition and rotation-variant SVD: the constructions of sym_eig3 /
// svd3_rv in double precision.
__device__ __forceinline__ void jacobi_rot_f64(double A[9], double V[9], int p, int q) {
  const double apq = A[p * 3 + q];
  if (fabs(apq) < 1e-300) return;
  const double theta = (A[q * 3 + q] - A[p * 3 + p]) / (2.0 * apq);
  const double t = copysign(1.0, theta) / (fabs(theta) + sqrt(fma(theta, theta, 1.0)));
  const double c = 1.0 / sqrt(fma(t, t, 1.0));
  const double s = t * c;
  for (int k = 0; k < 3; ++k) {
    const double akp = A[k * 3 + p], akq = A[k * 3 + q];
    A[k * 3 + p] = c * akp - s * akq;
    A[k * 3 + q] = s * akp + c * akq;
  }
  for (int k = 0; k < 3; ++k) {
    const double apk = A[p * 3 + k], aqk = A[q * 3 + k];
    A[p * 3 + k] = c * apk - s * aqk;
    A[q * 3 + k] = s * apk + c * aqk;
  }
  for (int k = 0; k < 3; ++k) {
    const double vkp = V[k * 3 + p], vkq = V[k * 3 + q];
    V[k * 3 + p] = c * vkp - s * vkq;
    V[k * 3 + q] = s * vkp + c * vkq;
  }
}

__device__ __forceinline__ void svd3_rv_f64(const double F[9], double U[9], double s[3], double V[9]) {
  double A[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      A[i * 3 + j] = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];
  for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 16; ++sweep) {
    const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    const double dg = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
    if (off <= 1e-32 * dg) break;
    jacobi_rot_f64(A, V, 0, 1);
    jacobi_rot_f64(A, V, 0, 2);
    jacobi_rot_f64(A, V, 1, 2);
  }
  double w[3] = {A[0], A[4], A[8]};
  // descending eigenvalues, V columns alongside
  for (int a = 0; a < 2; ++a)
    for (int b = a + 1; b < 3; ++b)
      if (w[a] < w[b]) {
        const double tw = w[a];
        w[a] = w[b];
        w[b] = tw;
        for (int r = 0; r < 3; ++r) {
          const double tv = V[r * 3 + a];
          V[r * 3 + a] = V[r * 3 + b];
          V[r * 3 + b] = tv;
        }
      }
  if (det3(V) < 0.0) {
    V[2] = -V[2];
    V[5] = -V[5];
    V[8] = -V[8];
  }
  double fv[3][3];
  for (int k = 0; k < 3; ++k)
    for (int r = 0; r < 3; ++r)
      fv[k][r] = F[r * 3 + 0] * V[0 * 3 + k] + F[r * 3 + 1] * V[1 * 3 + k] + F[r * 3 + 2] * V[2 * 3 + k];
  double u0[3], u1[3], u2[3];
  const double n0 = sqrt(fv[0][0] * fv[0][0] + fv[0][1] * fv[0][1] + fv[0][2] * fv[0][2]);
  for (int r = 0; r < 3; ++r) u0[r] = n0 > 0.0 ? fv[0][r] / n0 : (r == 0 ? 1.0 : 0.0);
  const double d01 = u0[0] * fv[1][0] + u0[1] * fv[1][1] + u0[2] * fv[1][2];
  for (int r = 0; r < 3; ++r) u1[r] = fv[1][r] - d01 * u0[r];
  double n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  if (!(n1 > 1e-12 * fmax(n0, 1e-300))) {  // rank < 2: any unit vector orthogonal to u0
    const double a0 = fabs(u0[0]) < 0.9 ? 1.0 : 0.0, a1 = 1.0 - a0;
    const double dd = a0 * u0[0] + a1 * u0[1];
    u1[0] = a0 - dd * u0[0];
    u1[1] = a1 - dd * u0[1];
    u1[2] = -dd * u0[2];
    n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  }
  for (int r = 0; r < 3; ++r) u1[r] /= n1;
  u2[0] = u0[1] * u1[2] - u0[2] * u1[1];
  u2[1] = u0[2] * u1[0] - u0[0] * u1[2];
  u2[2] = u0[0] * u1[1] - u0[1] * u1[0];
  for (int r = 0; r < 3; ++r) {
    U[r * 3 + 0] = u0[r];
    U[r * 3 + 1] = u1[r];
    U[r * 3 + 2] = u2[r];
  }
  s[0] = u0[0] * fv[0][0] + u0[1] * fv[0][1] + u0[2] * fv[0][2];
  s[1] = u1[0] * fv[1][0] + u1[1] * fv[1][1] + u1[2] * fv[1][2];
  s[2] = u2[0] * fv[2][0] + u2[1] * fv[2][1] + u2[2] * fv[2][2];
}

__device__ __forceinline__ void arap_energy_pk1_f64(double mu, const double F[9], double* psi, double P[9]) {
  double U[9], s[3], V[9];
  svd3_rv_f64(F, U, s, V);
  if (psi) *psi = 0.5 * mu * ((s[0] - 1.0) * (s[0] - 1.0) + (s[1] - 1.0) * (s[1] - 1.0) + (s[2] - 1.0) * (s[2] - 1.0));
  if (P) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        P[i * 3 + j] = mu * (F[i * 3 + j] - (U[i * 3] * V[j * 3] + U[i * 3 + 1] * V[j * 3 + 1] + U[i * 3 + 2] * V[j * 3 + 2]));
  }
}

// ARAP (batched_arap.cpp:29-136): C = mu I + sum_n l_n T_n T_n^T over the three twists T_n = U (e_k e_j^T -
// e_j e_k^T) V^T, l_n = -mu / (s_j + s_k) (projected: 2 l + mu clamped). In modal form: twist eigenvalue 2 l_n
// and flip eigenvalue 0 of the normalized modes, no scaling block, plus mu I.
__device__ __forceinline__ void arap_tanform(float mu, const float F[9], int project, int psd, float min_eig,
                                             TanForm& T) {
  float U[9], s[3], V[9];
  svd3_rv(F, U, s, V);
  T.kind = kTanModal;
  T.c0 = mu;
#pragma unroll
  for (int i = 0; i < 6; ++i) T.q2[i] = 0.0f;
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const int j = (n == 0) ? 1 : 0;
    const int k = (n == 2) ? 1 : 2;
    float l = -mu / (s[j] + s[k]);
    if (project && psd != 0) {
      const float e = 2.0f * l + mu;
      l = 0.5f * (fmaxf(psd == 2 ? fabsf(e) : e, min_eig) - mu);
    }
    T.sp[n] = l;
    T.sm[n] = -l;
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    T.q0[i] = U[i];
    T.q1[i] = V[i];
  }
}

__device__ __forceinline__ void linear_tanform(float mu, float lambda, TanForm& T) {
  T.kind = kTanLinear;
  T.c0 = mu;
  T.c1 = lambda;
}

// ------------------------------------------------------------------------------------------------
// Rayleigh stiffness damping (viscous stress), fem_stress_damping.h:29-501, isotropic reference stiffness:
// dE = E(F) - E(F_stage) in Voigt order [00, 11, 22, 12, 02, 01] with engineering shear,
// Sv = kappa lambda tr(dE) + 2 kappa mu dE (normal), kappa mu dE (shear).

__device__ __forceinline__ void visc_stress_f64(const double F[9], const double Fs[9], double kl, double km,
                                                double dE[6], double Sv[6]) {
  constexpr int vi[6] = {0, 1, 2, 1, 0, 0}, vj[6] = {0, 1, 2, 2, 2, 1};
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    double acc = 0.0;
#pragma unroll
    for (int p = 0; p < 3; ++p) acc += F[p * 3 + vi[a]] * F[p * 3 + vj[a]] - Fs[p * 3 + vi[a]] * Fs[p * 3 + vj[a]];
    dE[a] = a < 3 ? 0.5 * acc : acc;
  }
  const double tr = dE[0] + dE[1] + dE[2];
#pragma unroll
  for (int a = 0; a < 6; ++a) Sv[a] = a < 3 ? kl * tr + 2.0 * km * dE[a] : km * dE[a];
}

// symmetric 3x3 to eigenvalues >= FLT_EPSILON unless the leading minors prove it SPD
// (BatchedProjectSymPsd, decomposition_utils_inl.h:1558)
__device__ __forceinline__ void project_sym3_f32(float S[9]) {
  const float m1 = S[0], m2 = S[0] * S[4] - S[1] * S[1];
  const float m3 = S[0] * (S[4] * S[8] - S[5] * S[5]) - S[1] * (S[1] * S[8] - S[5] * S[2]) +
                   S[2] * (S[1] * S[5] - S[4] * S[2]);
  if (m1 > 0.0f && m2 > 0.0f && m3 > 0.0f) return;
  float w[3], V[9];
  sym_eig3(S, w, V);
#pragma unroll
  for (int i = 0; i < 3; ++i) w[i] = fmaxf(w[i], 1.1920928955078125e-07f);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      S[a * 3 + b] = V[a * 3 + 0] * w[0] * V[b * 3 + 0] + V[a * 3 + 1] * w[1] * V[b * 3 + 1] + V[a * 3 + 2] * w[2] * V[b * 3 + 2];
}

// ------------------------------------------------------------------------------------------------
// contact helpers (FP64): PolyReLU and the analytic collider SDFs

// activations.h:113-130
__device__ __forceinline__ void polyrelu(double x, double t, double shift, double& f, double& df,
                                         double& ddf) {
  x -= shift;
  if (t <= 0.0 || fabs(x) > t) {
    f = x > 0.0 ? x : 0.0;
    df = x < 0.0 ? 0.0 : 1.0;
    ddf = 0.0;
    return;
  }
  const double xt = x / t, x2 = xt * xt, x3 = x2 * xt;
  const double fv = (3.0 / 16.0) * t + (0.5 + (3.0 / 8.0) * xt - (1.0 / 16.0) * x3) * x;
  const double dfv = 0.5 + 0.75 * xt - 0.25 * x3;
  const double ddfv = 0.75 * (1.0 - x2) / t;
  f = fmax(fv, 0.0);
  df = fmin(fmax(dfv, 0.0), 1.0);
  ddf = fmax(ddfv, 0.0);
}

// Coulomb smoothing of the tangential displacement x >= 0 over the width t: value f, f'' and f'/x.
// cinf = false: the C1 step of Incremental Potential Contact (Li et al. 2020), f' = 2x/t - x^2/t^2 on
// [0, t), 1 above (activations.h:150-168); cinf = true: f = sqrt(x^2 + t^2/4) - t/2 with t clamped to the
// FP64 machine epsilon (activations.h:188-207).
__device__ __forceinline__ void friction_smoother(bool cinf, double x, double t, double& f, double& ddf,
                                                  double& dfx) {
  if (cinf) {
    const double e = fmax(t, 2.220446049250313e-16);
    const double e2 = 0.25 * e * e;
    const double sq = sqrt(x * x + e2);
    f = sq - 0.5 * e;
    dfx = 1.0 / sq;
    ddf = e2 / (sq * sq * sq);
    return;
  }
  if (x >= t) {
    f = x - t / 3.0;
    ddf = 0.0;
    dfx = x == 0.0 ? 0.0 : 1.0 / x;
    return;
  }
  const double r = x / t;
  f = x * r * (1.0 - r / 3.0);
  ddf = 2.0 * (1.0 - r) / t;
  dfx = (2.0 - r) / t;
}

// Dissipative part of one unmasked contact sample (ComputeBatchContactDissipationForceDForce,
// contact_utils.h:627-960, GradTarget::Current): Coulomb / viscous friction in the plane normal to n and
// normal viscous damping, scaled by the normal force fP, for the displacement prel relative to the
// collider. Adds to the energy E, the force F and the symmetric dforce D (xx, yy, zz, xy, xz, yz).
__device__ __forceinline__ void dissipation_response(double coulomb, double falloff, double viscous,
                                                     double ndamp, bool fitted, bool cinf, double fP,
                                                     const double n[3], const double prel[3], double& E,
                                                     double F[3], double D[6]) {
  const double pn = prel[0] * n[0] + prel[1] * n[1] + prel[2] * n[2];
  double pt[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) pt[i] = prel[i] - pn * n[i];
  const double tn = sqrt(pt[0] * pt[0] + pt[1] * pt[1] + pt[2] * pt[2]);
  double ef = 0.0, eigP = 0.0, eigN = 0.0, eigDT = 0.0;
  if (coulomb > 0.0) {
    double f, ddf, dfx;
    friction_smoother(cinf, tn, falloff, f, ddf, dfx);
    ef = coulomb * f;
    const double c = coulomb * fP * dfx;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[i] -= c * pt[i];
    eigP = -c;
    if (!fitted && tn > 1e-11) eigDT = -coulomb * fP * ddf - eigP;
  }
  if (viscous > 0.0) {
    ef += 0.5 * viscous * tn * tn;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[i] -= viscous * fP * pt[i];
    eigP -= viscous * fP;
  }
  if (ndamp > 0.0) {
    ef += 0.5 * ndamp * pn * pn;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[i] -= ndamp * fP * pn * n[i];
    eigN = -ndamp * fP;
  }
  const double dn = eigN - eigP;
  D[0] += eigP + dn * n[0] * n[0];
  D[1] += eigP + dn * n[1] * n[1];
  D[2] += eigP + dn * n[2] * n[2];
  D[3] += dn * n[0] * n[1];
  D[4] += dn * n[0] * n[2];
  D[5] += dn * n[1] * n[2];
  if (eigDT != 0.0) {
    const double inv = 1.0 / (tn + 2.2250738585072014e-308), w = eigDT * inv * inv;
    D[0] += w * pt[0] * pt[0];
    D[1] += w * pt[1] * pt[1];
    D[2] += w * pt[2] * pt[2];
    D[3] += w * pt[0] * pt[1];
    D[4] += w * pt[0] * pt[2];
    D[5] += w * pt[1] * pt[2];
  }
  E += fP * ef;
}

// collider row: (type, p[6], radius, vel[3])
__device__ __forceinline__ void collider_sdf(const double* c, const double x[3], double t, double& d,
                                             double g[3]) {
  if (c[0] == 0.0) {  // plane
    const double o = c[4] + (c[1] * c[8] + c[2] * c[9] + c[3] * c[10]) * t;
    d = c[1] * x[0] + c[2] * x[1] + c[3] * x[2] - o;
    g[0] = c[1];
    g[1] = c[2];
    g[2] = c[3];
    return;
  }
  double a[3], ab[3], ax[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    a[i] = c[1 + i] + c[8 + i] * t;
    ab[i] = c[4 + i] - c[1 + i];
    ax[i] = x[i] - a[i];
  }
  const double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
  double s = l2 > 0.0 ? (ax[0] * ab[0] + ax[1] * ab[1] + ax[2] * ab[2]) / l2 : 0.0;
  s = fmin(fmax(s, 0.0), 1.0);
  double df[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) df[i] = ax[i] - s * ab[i];
  const double dist = sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
  d = dist - c[7];
  if (dist > 0.0) {
    g[0] = df[0] / dist;
    g[1] = df[1] / dist;
    g[2] = df[2] / dist;
  } else {
    g[0] = 0.0;
    g[1] = 0.0;
    g[2] = 1.0;
  }
}

}  // namespace sdx
