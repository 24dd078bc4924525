/*
 * sdx_oracle.c — CPU oracle (test infrastructure only; never on the product path).
 *
 * Plain-C FP64 restatement of the reference's implicit soft-body step. Each function cites the
 * reference lines it follows (paths inside superdex_physics/libraries/mochi/). Parallel loops use
 * OpenMP; accumulation into shared rows uses atomics, so results are reproducible to rounding only.
 */
#include "sdx_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------------------------- */
/* small dense helpers                                                                          */

static double det3(const double F[9]) {
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

/* cofactor(F)_ij = dJ/dF_ij */
static void cof3(const double F[9], double C[9]) {
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

/* Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major, overwritten).
 * Eigenvalues end up on the diagonal; eigenvectors (columns of V) are returned when V != NULL. */
static void jacobi_eig(int n, double* A, double* V) {
  if (V) {
    for (int i = 0; i < n * n; ++i) V[i] = 0.0;
    for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
  }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i) {
      diag += A[i * n + i] * A[i * n + i];
      for (int j = i + 1; j < n; ++j) off += A[i * n + j] * A[i * n + j];
    }
    if (off <= 1e-32 * diag || off == 0.0) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (apq == 0.0) continue;
        double app = A[p * n + p], aqq = A[q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        if (V) {
          for (int k = 0; k < n; ++k) {
            double vkp = V[k * n + p], vkq = V[k * n + q];
            V[k * n + p] = c * vkp - s * vkq;
            V[k * n + q] = s * vkp + c * vkq;
          }
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------------------------- */
/* material                                                                                     */

void or_lame(double E, double nu, double* lambda, double* mu) {
  /* material_utils.h:331-339 */
  *lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  *mu = E / (2.0 * (1.0 + nu));
}

static const int kLevi[3][3][3] = {{{0, 0, 0}, {0, 0, 1}, {0, -1, 0}},
                                   {{0, 0, -1}, {0, 0, 0}, {1, 0, 0}},
                                   {{0, 1, 0}, {-1, 0, 0}, {0, 0, 0}}};

void or_smith_nh(double mu, double lambda, const double F[9], int project, int psd_strategy,
                 double min_eig, double* energy, double P[9], double Cout[81]) {
  /* Reparameterised Lame constants, batched_smith_neo_hookean.cpp:51-55. */
  const double muHat = mu * (4.0 / 3.0);
  const double lambdaHat = lambda + mu * (5.0 / 6.0);
  const double alpha = 1.0 + 0.75 * muHat / lambdaHat;
  double Ic = 0.0;
  for (int i = 0; i < 9; ++i) Ic += F[i] * F[i];
  const double IcPlus1 = Ic + 1.0, IcPlus1Inv = 1.0 / IcPlus1;
  const double J = det3(F), Jma = J - alpha;

  if (energy) /* :65-69 */
    *energy = 0.5 * muHat * (Ic - 3.0) + 0.5 * lambdaHat * Jma * Jma - 0.5 * muHat * log(IcPlus1);

  double cofF[9];
  cof3(F, cofF);
  if (P) { /* :127-136 */
    const double c0 = muHat * (1.0 - IcPlus1Inv), c1 = lambdaHat * Jma;
    for (int i = 0; i < 9; ++i) P[i] = c0 * F[i] + c1 * cofF[i];
  }
  if (!Cout) return;

  /* Direct tangent, :204-266: c3 F(x)F + lambdaHat cof(x)cof + lambdaHat(J-alpha) d2J + c2 I. */
  const double c2 = muHat * (1.0 - IcPlus1Inv);
  const double c3 = 2.0 * muHat * IcPlus1Inv * IcPlus1Inv;
  int projecting = project && psd_strategy != OR_PSD_NONE;
  int indefinite = 1;
  if (projecting) {
    /* PSD oracle "Correct", :81-104: lambdaHat^2 (J-alpha)^2 max sigma^2 > muHatK^2, or J < 0. */
    double S[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += F[k * 3 + i] * F[k * 3 + j];
        S[i * 3 + j] = s;
      }
    jacobi_eig(3, S, NULL);
    double maxSigSq = fmax(S[0], fmax(S[4], S[8]));
    const double muHatK = muHat * (1.0 - IcPlus1Inv);
    const double lhsBase = (lambdaHat * Jma) * (lambdaHat * Jma);
    indefinite = (lhsBase * maxSigSq > muHatK * muHatK) || (J < 0.0);
    projecting = indefinite;
  }
  double d2JCoeff = lambdaHat * Jma;
  if (projecting && psd_strategy == OR_PSD_FAST) d2JCoeff = 0.0; /* :214-239 */
  for (int a = 0; a < 9; ++a)
    for (int b = 0; b < 9; ++b) Cout[a * 9 + b] = c3 * F[a] * F[b] + lambdaHat * cofF[a] * cofF[b];
  for (int a = 0; a < 9; ++a) Cout[a * 9 + a] += c2;
  /* d2J/dF_ij dF_kl = sum_{n,q} eps_ikn eps_jlq F_nq (material_utils.h:182-218). */
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) {
          double h = 0.0;
          for (int n = 0; n < 3; ++n)
            for (int q = 0; q < 3; ++q) h += kLevi[i][k][n] * kLevi[j][l][q] * F[n * 3 + q];
          Cout[(i * 3 + j) * 9 + (k * 3 + l)] += d2JCoeff * h;
        }
  if (projecting && (psd_strategy == OR_PSD_PROJECTION || psd_strategy == OR_PSD_ABS_EIGEN)) {
    /* Eigensystem path, :141-203: clamp the 9 tangent eigenvalues at kMinProjectedEigenvalue
     * (max(l, eps) for Projection, max(|l|, eps) for AbsEigenProjection). The reference builds the
     * eigensystem analytically (Smith et al. 2018); the oracle diagonalises the 9x9 tangent directly,
     * which gives the same spectral projection. */
    double A[81], V[81], lam[9];
    memcpy(A, Cout, sizeof(A));
    jacobi_eig(9, A, V);
    for (int i = 0; i < 9; ++i) {
      double l = A[i * 9 + i];
      if (psd_strategy == OR_PSD_ABS_EIGEN) l = fabs(l);
      lam[i] = l > min_eig ? l : min_eig;
    }
    for (int a = 0; a < 9; ++a)
      for (int b = 0; b < 9; ++b) {
        double s = 0.0;
        for (int i = 0; i < 9; ++i) s += V[a * 9 + i] * lam[i] * V[b * 9 + i];
        Cout[a * 9 + b] = s;
      }
  }
}

/* Clamp the 9 eigenvalues of a symmetric tangent: max(l, eps) (Projection) or max(|l|, eps). */
static void or_project_tangent(double C[81], int abs_eig, double min_eig) {
  double A[81], V[81], lam[9];
  memcpy(A, C, sizeof(A));
  jacobi_eig(9, A, V);
  for (int i = 0; i < 9; ++i) {
    double l = A[i * 9 + i];
    if (abs_eig) l = fabs(l);
    lam[i] = l > min_eig ? l : min_eig;
  }
  for (int a = 0; a < 9; ++a)
    for (int b = 0; b < 9; ++b) {
      double s = 0.0;
      for (int i = 0; i < 9; ++i) s += V[a * 9 + i] * lam[i] * V[b * 9 + i];
      C[a * 9 + b] = s;
    }
}

void or_stvk(double mu, double lambda, const double F[9], int project, int psd_strategy, double min_eig,
             double* energy, double P[9], double C[81]) {
  /* Green strain, batched_st_venant_kirchhoff.cpp:53-63 */
  double G[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double g = 0.0;
      for (int k = 0; k < 3; ++k) g += F[k * 3 + i] * F[k * 3 + j];
      G[i * 3 + j] = 0.5 * (g - (i == j ? 1.0 : 0.0));
    }
  double trG = G[0] + G[4] + G[8];
  if (energy) {
    double n2 = 0.0;
    for (int i = 0; i < 9; ++i) n2 += G[i] * G[i];
    *energy = mu * n2 + 0.5 * lambda * trG * trG;
  }
  if (P) {
    double S[9];
    for (int i = 0; i < 9; ++i) S[i] = 2.0 * mu * G[i];
    for (int i = 0; i < 3; ++i) S[i * 4] += lambda * trG;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double v = 0.0;
        for (int m = 0; m < 3; ++m) v += F[r * 3 + m] * S[m * 3 + c];
        P[r * 3 + c] = v;
      }
  }
  if (!C) return;
  const int eigen = project && (psd_strategy == OR_PSD_PROJECTION || psd_strategy == OR_PSD_ABS_EIGEN);
  if (project && psd_strategy == OR_PSD_FAST) { /* :158-169 */
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) G[i * 3 + j] = (i == j) ? (G[i * 4] > 0.0 ? G[i * 4] : 0.0) : 0.0;
    trG = G[0] + G[4] + G[8];
  }
  double S[9], FFt[9];
  for (int i = 0; i < 9; ++i) S[i] = 2.0 * mu * G[i];
  for (int i = 0; i < 3; ++i) S[i * 4] += lambda * trG;
  for (int r = 0; r < 3; ++r)
    for (int i = 0; i < 3; ++i) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += F[r * 3 + k] * F[i * 3 + k];
      FFt[r * 3 + i] = v;
    }
  /* dP_rc/dF_ij = delta_ri S_jc + mu F_rj F_ic + mu delta_jc (F F^T)_ri + lambda F_ij F_rc (:171-197) */
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double v = mu * F[r * 3 + j] * F[i * 3 + c] + lambda * F[i * 3 + j] * F[r * 3 + c];
          if (r == i) v += S[j * 3 + c];
          if (j == c) v += mu * FFt[r * 3 + i];
          C[(r * 3 + c) * 9 + (i * 3 + j)] = v;
        }
  if (eigen) or_project_tangent(C, psd_strategy == OR_PSD_ABS_EIGEN, min_eig); /* :96-154 */
}

void or_linear_elastic(double mu, double lambda, const double F[9], double* energy, double P[9], double C[81]) {
  double e[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) e[r * 3 + c] = 0.5 * (F[r * 3 + c] + F[c * 3 + r]) - (r == c ? 1.0 : 0.0);
  const double tr = e[0] + e[4] + e[8];
  if (energy) {
    double n2 = 0.0;
    for (int i = 0; i < 9; ++i) n2 += e[i] * e[i];
    *energy = mu * n2 + 0.5 * lambda * tr * tr;
  }
  if (P) {
    for (int i = 0; i < 9; ++i) P[i] = 2.0 * mu * e[i];
    for (int i = 0; i < 3; ++i) P[i * 4] += lambda * tr;
  }
  if (C) /* dP_rc/dF_ij = mu (d_ri d_cj + d_ci d_rj) + lambda d_rc d_ij (:72-94) */
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            C[(r * 3 + c) * 9 + (i * 3 + j)] =
                mu * ((r == i && c == j) + (c == i && r == j)) + lambda * (r == c && i == j);
}

/* symmetric 3x3 projected to eigenvalues >= DBL_EPSILON unless its leading minors prove it SPD
 * (BatchedProjectSymPsd, mochi_core/.../utils/decomposition_utils_inl.h:1558) */
static void or_project_sym3(double S[9]) {
  const double m1 = S[0], m2 = S[0] * S[4] - S[1] * S[1];
  const double m3 = S[0] * (S[4] * S[8] - S[5] * S[5]) - S[1] * (S[1] * S[8] - S[5] * S[2]) +
                    S[2] * (S[1] * S[5] - S[4] * S[2]);
  if (m1 > 0.0 && m2 > 0.0 && m3 > 0.0) return;
  double A[9], V[9];
  memcpy(A, S, sizeof(A));
  jacobi_eig(3, A, V);
  double l[3];
  for (int i = 0; i < 3; ++i) l[i] = A[i * 4] > DBL_EPSILON ? A[i * 4] : DBL_EPSILON;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) S[a * 3 + b] = V[a * 3 + 0] * l[0] * V[b * 3 + 0] + V[a * 3 + 1] * l[1] * V[b * 3 + 1] +
                                               V[a * 3 + 2] * l[2] * V[b * 3 + 2];
}

void or_stress_damping(const double dN[12], double vol, const double u[12], const double uss[12], double kappa,
                       double lambda, double mu, int geometric, int project, double* energy, double res[12],
                       double K[144]) {
  static const int vi[6] = {0, 1, 2, 1, 0, 0}, vj[6] = {0, 1, 2, 2, 2, 1};
  double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Fs[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int f = 0; f < 4; ++f)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        F[r * 3 + c] += u[3 * f + r] * dN[3 * f + c];
        Fs[r * 3 + c] += uss[3 * f + r] * dN[3 * f + c];
      }
  double dE[6], Sv[6];
  for (int a = 0; a < 6; ++a) {
    double acc = 0.0;
    for (int p = 0; p < 3; ++p) acc += F[p * 3 + vi[a]] * F[p * 3 + vj[a]] - Fs[p * 3 + vi[a]] * Fs[p * 3 + vj[a]];
    dE[a] = a < 3 ? 0.5 * acc : acc; /* engineering shear */
  }
  const double tr = dE[0] + dE[1] + dE[2];
  for (int a = 0; a < 3; ++a) Sv[a] = kappa * lambda * tr + 2.0 * kappa * mu * dE[a];
  for (int a = 3; a < 6; ++a) Sv[a] = kappa * mu * dE[a];
  double S[9] = {Sv[0], Sv[5], Sv[4], Sv[5], Sv[1], Sv[3], Sv[4], Sv[3], Sv[2]};
  if (energy) {
    double psi = 0.0;
    for (int a = 0; a < 6; ++a) psi += Sv[a] * dE[a];
    *energy = 0.5 * psi * vol;
  }
  if (res) {
    for (int f = 0; f < 4; ++f)
      for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int c = 0; c < 3; ++c) {
          double pic = 0.0;
          for (int k = 0; k < 3; ++k) pic += F[i * 3 + k] * S[k * 3 + c];
          acc += pic * dN[3 * f + c];
        }
        res[3 * f + i] = vol * acc;
      }
  }
  if (!K) return;
  if (geometric && project) or_project_sym3(S);
  double FFt[9], a[4][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += F[i * 3 + k] * F[j * 3 + k];
      FFt[i * 3 + j] = v;
    }
  for (int f = 0; f < 4; ++f)
    for (int i = 0; i < 3; ++i)
      a[f][i] = F[i * 3 + 0] * dN[3 * f + 0] + F[i * 3 + 1] * dN[3 * f + 1] + F[i * 3 + 2] * dN[3 * f + 2];
  for (int f = 0; f < 4; ++f)
    for (int g = 0; g < 4; ++g) {
      const double dd = dN[3 * f] * dN[3 * g] + dN[3 * f + 1] * dN[3 * g + 1] + dN[3 * f + 2] * dN[3 * g + 2];
      double geo = 0.0;
      if (geometric)
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) geo += dN[3 * f + k] * S[k * 3 + l] * dN[3 * g + l];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double v = kappa * lambda * a[f][i] * a[g][j] + kappa * mu * (FFt[i * 3 + j] * dd + a[g][i] * a[f][j]);
          if (i == j) v += geo;
          K[(3 * f + i) * 12 + 3 * g + j] = vol * v;
        }
    }
}

/* Rotation-variant SVD F = U diag(s) V^T with det U = det V = +1 and s[2] < 0 iff det F < 0 (the
 * convention of BatchedRotationVariantSvd3x3, mochi_core/.../utils/decomposition_utils.h): V from the
 * eigenvectors of F^T F by decreasing eigenvalue, U from F V (normalised, Gram-Schmidt, u2 = u0 x u1),
 * s_k = u_k . F v_k. */
static void or_svd_rv(const double F[9], double U[9], double s[3], double V[9]) {
  double S[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += F[k * 3 + i] * F[k * 3 + j];
      S[i * 3 + j] = v;
    }
  jacobi_eig(3, S, V);
  int ord[3] = {0, 1, 2};
  for (int a = 0; a < 3; ++a)
    for (int b = a + 1; b < 3; ++b)
      if (S[ord[b] * 4] > S[ord[a] * 4]) {
        int t = ord[a];
        ord[a] = ord[b];
        ord[b] = t;
      }
  double Vs[9];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) Vs[r * 3 + k] = V[r * 3 + ord[k]];
  if (det3(Vs) < 0.0)
    for (int r = 0; r < 3; ++r) Vs[r * 3 + 2] = -Vs[r * 3 + 2];
  memcpy(V, Vs, sizeof(Vs));
  double fv[3][3];
  for (int k = 0; k < 3; ++k)
    for (int r = 0; r < 3; ++r) fv[k][r] = F[r * 3] * V[k] + F[r * 3 + 1] * V[3 + k] + F[r * 3 + 2] * V[6 + k];
  double u[3][3];
  const double n0 = sqrt(fv[0][0] * fv[0][0] + fv[0][1] * fv[0][1] + fv[0][2] * fv[0][2]);
  for (int r = 0; r < 3; ++r) u[0][r] = n0 > 0.0 ? fv[0][r] / n0 : (r == 0 ? 1.0 : 0.0);
  const double d01 = u[0][0] * fv[1][0] + u[0][1] * fv[1][1] + u[0][2] * fv[1][2];
  for (int r = 0; r < 3; ++r) u[1][r] = fv[1][r] - d01 * u[0][r];
  double n1 = sqrt(u[1][0] * u[1][0] + u[1][1] * u[1][1] + u[1][2] * u[1][2]);
  if (n1 <= 1e-12 * (n0 > 0.0 ? n0 : 1.0)) { /* rank < 2: any unit vector orthogonal to u0 */
    double a[3] = {fabs(u[0][0]) < 0.9 ? 1.0 : 0.0, fabs(u[0][0]) < 0.9 ? 0.0 : 1.0, 0.0};
    const double dd = a[0] * u[0][0] + a[1] * u[0][1] + a[2] * u[0][2];
    for (int r = 0; r < 3; ++r) u[1][r] = a[r] - dd * u[0][r];
    n1 = sqrt(u[1][0] * u[1][0] + u[1][1] * u[1][1] + u[1][2] * u[1][2]);
  }
  for (int r = 0; r < 3; ++r) u[1][r] /= n1;
  u[2][0] = u[0][1] * u[1][2] - u[0][2] * u[1][1];
  u[2][1] = u[0][2] * u[1][0] - u[0][0] * u[1][2];
  u[2][2] = u[0][0] * u[1][1] - u[0][1] * u[1][0];
  for (int k = 0; k < 3; ++k) {
    for (int r = 0; r < 3; ++r) U[r * 3 + k] = u[k][r];
    s[k] = u[k][0] * fv[k][0] + u[k][1] * fv[k][1] + u[k][2] * fv[k][2];
  }
}

void or_arap(double mu, const double F[9], int project, int psd_strategy, double min_eig, double* energy,
             double P[9], double C[81]) {
  /* batched_arap.cpp:29-136: energy 1/2 mu |s - 1|^2, PK1 mu (F - U V^T), tangent the exact Hessian
   * mu I - sum_n mu / (s_j + s_k) T_n (x) T_n over the twist modes T_n = u_k v_j^T - u_j v_k^T; the six
   * other eigenvalues are mu, so clamping the 9x9 spectrum equals the reference's twist-only clamp. */
  double U[9], s[3], V[9];
  or_svd_rv(F, U, s, V);
  if (energy) *energy = 0.5 * mu * ((s[0] - 1.0) * (s[0] - 1.0) + (s[1] - 1.0) * (s[1] - 1.0) +
                                    (s[2] - 1.0) * (s[2] - 1.0));
  if (P)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        P[i * 3 + j] = mu * (F[i * 3 + j] - (U[i * 3] * V[j * 3] + U[i * 3 + 1] * V[j * 3 + 1] + U[i * 3 + 2] * V[j * 3 + 2]));
  if (!C) return;
  memset(C, 0, sizeof(double) * 81);
  for (int a = 0; a < 9; ++a) C[a * 9 + a] = mu;
  static const int pj[3] = {1, 0, 0}, pk[3] = {2, 2, 1};
  for (int n = 0; n < 3; ++n) {
    const int j = pj[n], k = pk[n];
    const double lam = -mu / (s[j] + s[k]);
    double T[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) T[r * 3 + c] = U[r * 3 + k] * V[c * 3 + j] - U[r * 3 + j] * V[c * 3 + k];
    for (int a = 0; a < 9; ++a)
      for (int b = 0; b < 9; ++b) C[a * 9 + b] += lam * T[a] * T[b];
  }
  if (project && psd_strategy != OR_PSD_NONE) or_project_tangent(C, psd_strategy == OR_PSD_ABS_EIGEN, min_eig);
}

void or_material(int material, double mu, double lambda, const double F[9], int project, int psd_strategy,
                 double min_eig, double* energy, double P[9], double C[81]) {
  if (material == OR_MAT_STVK)
    or_stvk(mu, lambda, F, project, psd_strategy, min_eig, energy, P, C);
  else if (material == OR_MAT_LINEAR)
    or_linear_elastic(mu, lambda, F, energy, P, C);
  else if (material == OR_MAT_ARAP)
    or_arap(mu, F, project, psd_strategy, min_eig, energy, P, C);
  else
    or_smith_nh(mu, lambda, F, project, psd_strategy, min_eig, energy, P, C);
}

/* ------------------------------------------------------------------------------------------- */
/* contact                                                                                      */

void or_polyrelu(double x, double t, double shift, double* f, double* df, double* ddf) {
  /* activations.h:113-130 */
  x -= shift;
  int mask = (t <= 0.0) || (fabs(x) > t);
  if (mask) {
    *f = x > 0.0 ? x : 0.0;
    *df = x < 0.0 ? 0.0 : 1.0;
    *ddf = 0.0;
    return;
  }
  double xt = x / t, x2 = xt * xt, x3 = x2 * xt;
  double fv = (3.0 / 16.0) * t + (0.5 + (3.0 / 8.0) * xt - (1.0 / 16.0) * x3) * x;
  double dfv = 0.5 + 0.75 * xt - 0.25 * x3;
  double ddfv = 0.75 * (1.0 - x2) / t;
  *f = fv > 0.0 ? fv : 0.0;
  *df = dfv < 0.0 ? 0.0 : (dfv > 1.0 ? 1.0 : dfv);
  *ddf = ddfv > 0.0 ? ddfv : 0.0;
}

void or_penalty(double d, const double grad[3], double k, double t_half, double thr,
                double* energy, double force[3], double dforce[9]) {
  /* contact_utils.h:526-569: p = PolyReLU(-d; t, t - thr). */
  double p, dp, ddp;
  or_polyrelu(-d, t_half, t_half - thr, &p, &dp, &ddp);
  if (energy) *energy = 0.5 * k * p * p;
  double fn = k * p * dp;
  if (force)
    for (int i = 0; i < 3; ++i) force[i] = fn * grad[i];
  double dfn = -k * (dp * dp + p * ddp);
  if (dforce)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dforce[i * 3 + j] = dfn * grad[i] * grad[j];
}

/* Coulomb smoothing of the tangential displacement x >= 0 over the width t: value f, derivatives df,
 * ddf and df/x (finite at x = 0).
 * model 0, the C1 step of Incremental Potential Contact (Li et al. 2020): df rises as 2x/t - x^2/t^2
 * on [0, t) and is 1 above (mochi_core/.../utils/activations.h:150-168);
 * model 1, the C-infinity regularization f = sqrt(x^2 + t^2/4) - t/2 with t clamped to the machine
 * epsilon (activations.h:188-207). */
static void or_friction_smoother(int model, double x, double t, double* f, double* df, double* ddf,
                                 double* dfx) {
  if (model == 1) {
    const double e = t > DBL_EPSILON ? t : DBL_EPSILON;
    const double e2 = 0.25 * e * e;
    const double sq = sqrt(x * x + e2);
    *f = sq - 0.5 * e;
    *dfx = 1.0 / sq;
    *df = x / sq;
    *ddf = e2 / (sq * sq * sq);
    return;
  }
  const double r = x / t;
  if (x >= t) {
    *f = x - t / 3.0;
    *ddf = 0.0;
    *dfx = x == 0.0 ? 0.0 : 1.0 / x;
    *df = 1.0;
    return;
  }
  *f = x * r * (1.0 - r / 3.0);
  *ddf = 2.0 * (1.0 - r) / t;
  *dfx = (2.0 - r) / t;
  *df = x * *dfx;
}

static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

void or_collision_response(const or_contact_params* p, double d, const double grad[3], double d_ss,
                           const double grad_ss[3], const double n_col[3], const double pos[3],
                           const double pos_ss[3], double dt, int unit_grad, double* energy,
                           double force[3], double dforce[9]) {
  /* normals: the collider's (SDF gradient, stage-start with explicit normals) and the colliding
   * surface's; contact is masked when they are more aligned than max_align, and the dissipation's
   * normal force fades with the alignment (contact_utils.h:1058-1095) */
  const double* nc = p->explicit_normals ? grad_ss : grad;
  const int valid = n_col != NULL;
  const double align = valid ? dot3(nc, n_col) : -1.0;
  const int on = align <= p->max_align;
  const double afac = (p->fade && valid && p->max_align > -1.0) ? (p->max_align - align) / (p->max_align + 1.0)
                                                               : 1.0;
  /* penalty with the current distance and gradient (contact_utils.h:498-570) */
  double pv, dp, ddp;
  or_polyrelu(-d, p->t_half, p->t_half - p->thr, &pv, &dp, &ddp);
  if (!on) pv = dp = ddp = 0.0;
  double E = 0.5 * p->k * pv * pv;
  const double fn = p->k * pv * dp, dfn = -p->k * (dp * dp + pv * ddp);
  double F[3], D[9];
  for (int i = 0; i < 3; ++i) {
    F[i] = fn * grad[i];
    for (int j = 0; j < 3; ++j) D[3 * i + j] = dfn * grad[i] * grad[j];
  }
  const int diss = p->coulomb > 0.0 || p->viscous > 0.0 || p->normal_damping > 0.0;
  if (diss) {
    /* the dissipation's normal force: current (implicit) or at the stage-start distance, exact with
     * explicit normals, else estimated along the current gradient (contact_utils.h:1133-1175) */
    double fP;
    double prel[3];
    for (int i = 0; i < 3; ++i) prel[i] = pos[i] - pos_ss[i];
    if (p->implicit_normal_force) {
      fP = afac * fn;
    } else {
      const double dss = p->explicit_normals ? d_ss : d - dot3(grad, prel);
      double q, dq, ddq;
      or_polyrelu(-dss, p->t_half, p->t_half - p->thr, &q, &dq, &ddq);
      if (!on) q = dq = 0.0;
      fP = afac * p->k * q * dq;
    }
    /* friction plane normal (contact_utils.h:643-690) */
    double n[3];
    if (p->collider_normal || !valid) {
      for (int i = 0; i < 3; ++i) n[i] = nc[i];
      if (!unit_grad) {
        const double nl = sqrt(dot3(n, n));
        for (int i = 0; i < 3; ++i) n[i] /= nl;
        if (nl < 100.0 * 1e-6)
          for (int i = 0; i < 3; ++i) n[i] = valid ? -n_col[i] : 0.0;
      }
    } else {
      for (int i = 0; i < 3; ++i) n[i] = -n_col[i];
    }
    const double pn = dot3(prel, n);
    double pt[3];
    for (int i = 0; i < 3; ++i) pt[i] = prel[i] - pn * n[i];
    const double tn = sqrt(dot3(pt, pt));
    /* dforce = eigP (I - n n^T) + eigN n n^T [+ (eigT - eigP) t t^T]; energy = fP * factor
     * (contact_utils.h:700-960, GradTarget::Current) */
    double ef = 0.0, eigP = 0.0, eigN = 0.0, eigDT = 0.0, tg[3] = {0.0, 0.0, 0.0};
    if (p->coulomb > 0.0) {
      double f, df, ddf, dfx;
      or_friction_smoother(p->model, tn, p->falloff_vel * dt, &f, &df, &ddf, &dfx);
      ef = p->coulomb * f;
      const double c = p->coulomb * fP * dfx;
      for (int i = 0; i < 3; ++i) F[i] -= c * pt[i];
      eigP = -c;
      if (!p->fitted) {
        const double eigT = -p->coulomb * fP * ddf;
        const double inv = 1.0 / (tn + DBL_MIN);
        for (int i = 0; i < 3; ++i) tg[i] = pt[i] * inv;
        eigDT = tn > 1e-11 ? eigT - eigP : 0.0;
      }
    }
    if (p->viscous > 0.0) {
      const double cv = p->viscous / dt;
      ef += 0.5 * cv * tn * tn;
      for (int i = 0; i < 3; ++i) F[i] -= cv * fP * pt[i];
      eigP -= cv * fP;
    }
    if (p->normal_damping > 0.0) {
      const double cn = p->normal_damping / dt;
      ef += 0.5 * cn * pn * pn;
      for (int i = 0; i < 3; ++i) F[i] -= cn * fP * pn * n[i];
      eigN = -cn * fP;
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        D[3 * i + j] += (i == j ? eigP : 0.0) + (eigN - eigP) * n[i] * n[j];
        if (!p->fitted && p->coulomb > 0.0) D[3 * i + j] += eigDT * tg[i] * tg[j];
      }
    E += fP * ef;
  }
  if (energy) *energy = E;
  if (force)
    for (int i = 0; i < 3; ++i) force[i] = F[i];
  if (dforce)
    for (int i = 0; i < 9; ++i) dforce[i] = D[i];
}

/* Signed distance and gradient of a collider at time t. Plane: d = n.x - (o + (n.v) t).
 * Capsule: distance to the moving segment a(t) b(t) minus the radius (closed form). */
static void collider_sdf(const or_collider* c, const double x[3], double t, double* d,
                         double g[3]) {
  if (c->type == OR_COLLIDER_PLANE) {
    const double* n = c->p;
    double o = c->p[3] + (n[0] * c->vel[0] + n[1] * c->vel[1] + n[2] * c->vel[2]) * t;
    *d = n[0] * x[0] + n[1] * x[1] + n[2] * x[2] - o;
    g[0] = n[0];
    g[1] = n[1];
    g[2] = n[2];
    return;
  }
  double a[3], ab[3], ax[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = c->p[i] + c->vel[i] * t;
    ab[i] = c->p[3 + i] - c->p[i];
    ax[i] = x[i] - a[i];
  }
  double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
  double s = l2 > 0.0 ? (ax[0] * ab[0] + ax[1] * ab[1] + ax[2] * ab[2]) / l2 : 0.0;
  s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  double df[3];
  for (int i = 0; i < 3; ++i) df[i] = ax[i] - s * ab[i];
  double dist = sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
  *d = dist - c->radius;
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

/* ------------------------------------------------------------------------------------------- */
/* mesh / pattern                                                                               */

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* node -> incident tets CSR */
static void node_tets(int n_nodes, int n_tets, const int32_t* tets, int64_t** ptr_out,
                      int32_t** list_out) {
  int64_t* ptr = (int64_t*)calloc((size_t)n_nodes + 1, sizeof(int64_t));
  for (int64_t t = 0; t < n_tets; ++t)
    for (int k = 0; k < 4; ++k) ptr[tets[4 * t + k] + 1]++;
  for (int i = 0; i < n_nodes; ++i) ptr[i + 1] += ptr[i];
  int32_t* list = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ptr[n_nodes] ? ptr[n_nodes] : 1));
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n_nodes ? n_nodes : 1));
  memcpy(fill, ptr, sizeof(int64_t) * (size_t)n_nodes);
  for (int64_t t = 0; t < n_tets; ++t)
    for (int k = 0; k < 4; ++k) list[fill[tets[4 * t + k]]++] = (int32_t)t;
  free(fill);
  *ptr_out = ptr;
  *list_out = list;
}

static int node_neighbors(int i, const int32_t* tets, const int64_t* nt_ptr, const int32_t* nt,
                          int* buf) {
  int m = 0;
  buf[m++] = i;
  for (int64_t e = nt_ptr[i]; e < nt_ptr[i + 1]; ++e)
    for (int k = 0; k < 4; ++k) buf[m++] = tets[4 * (int64_t)nt[e] + k];
  qsort(buf, (size_t)m, sizeof(int), cmp_int);
  int u = 0;
  for (int k = 0; k < m; ++k)
    if (u == 0 || buf[k] != buf[u - 1]) buf[u++] = buf[k];
  return u;
}

int64_t or_pattern_nnzb(int n_nodes, int n_tets, const int32_t* tets) {
  int64_t* ptr;
  int32_t* nt;
  node_tets(n_nodes, n_tets, tets, &ptr, &nt);
  int maxdeg = 0;
  for (int i = 0; i < n_nodes; ++i)
    if (ptr[i + 1] - ptr[i] > maxdeg) maxdeg = (int)(ptr[i + 1] - ptr[i]);
  int* buf = (int*)malloc(sizeof(int) * (size_t)(4 * maxdeg + 1));
  int64_t total = 0;
  for (int i = 0; i < n_nodes; ++i) total += node_neighbors(i, tets, ptr, nt, buf);
  free(buf);
  free(ptr);
  free(nt);
  return total;
}

void or_pattern_fill(int n_nodes, int n_tets, const int32_t* tets, int64_t* row_ptr, int32_t* col) {
  int64_t* ptr;
  int32_t* nt;
  node_tets(n_nodes, n_tets, tets, &ptr, &nt);
  int maxdeg = 0;
  for (int i = 0; i < n_nodes; ++i)
    if (ptr[i + 1] - ptr[i] > maxdeg) maxdeg = (int)(ptr[i + 1] - ptr[i]);
  int* buf = (int*)malloc(sizeof(int) * (size_t)(4 * maxdeg + 1));
  row_ptr[0] = 0;
  for (int i = 0; i < n_nodes; ++i) {
    int m = node_neighbors(i, tets, ptr, nt, buf);
    for (int k = 0; k < m; ++k) col[row_ptr[i] + k] = buf[k];
    row_ptr[i + 1] = row_ptr[i] + m;
  }
  free(buf);
  free(ptr);
  free(nt);
}

int64_t or_pattern_find(const int64_t* row_ptr, const int32_t* col, int i, int j) {
  int64_t lo = row_ptr[i], hi = row_ptr[i + 1] - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) / 2;
    if (col[mid] == j) return mid;
    if (col[mid] < j)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return -1;
}

void or_rest_data(int n_tets, const int32_t* tets, const double* X, double* dN, double* vol) {
  /* finite_element.h:93-139 with 1-point quadrature: Dm = [x1-x0, x2-x0, x3-x0] (columns),
   * quadWeight = det(Dm)/6, dN_f = Dm^{-T} dN_f(param). */
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < n_tets; ++t) {
    const double* x0 = X + 3 * (int64_t)tets[4 * t + 0];
    double D[9];
    for (int k = 1; k <= 3; ++k) {
      const double* xk = X + 3 * (int64_t)tets[4 * t + k];
      for (int r = 0; r < 3; ++r) D[r * 3 + (k - 1)] = xk[r] - x0[r];
    }
    double det = det3(D);
    double cof[9];
    cof3(D, cof); /* D^{-T} = cof / det */
    double* d = dN + 12 * t;
    for (int f = 1; f <= 3; ++f)
      for (int c = 0; c < 3; ++c) d[3 * f + c] = cof[c * 3 + (f - 1)] / det;
    for (int c = 0; c < 3; ++c) d[c] = -(d[3 + c] + d[6 + c] + d[9 + c]);
    vol[t] = det / 6.0;
  }
}

/* Faces are numbered as TetFaces (mochi_core/.../elements/tetrahedral/simplex_quadrature.h:45-52):
 * 0:(0,1,2) 1:(0,1,3) 2:(0,2,3) 3:(1,2,3). */
static const int kFaceLocal[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
static const int kFaceOpp[4] = {3, 2, 1, 0};

typedef struct {
  int32_t a, b, c;
  int32_t tet, face;
} face_rec;

static int cmp_face(const void* p, const void* q) {
  const face_rec* x = (const face_rec*)p;
  const face_rec* y = (const face_rec*)q;
  if (x->a != y->a) return (x->a > y->a) - (x->a < y->a);
  if (x->b != y->b) return (x->b > y->b) - (x->b < y->b);
  if (x->c != y->c) return (x->c > y->c) - (x->c < y->c);
  if (x->tet != y->tet) return (x->tet > y->tet) - (x->tet < y->tet);
  return (x->face > y->face) - (x->face < y->face);
}

static int cmp_face_owner(const void* p, const void* q) {
  const face_rec* x = (const face_rec*)p;
  const face_rec* y = (const face_rec*)q;
  if (x->tet != y->tet) return (x->tet > y->tet) - (x->tet < y->tet);
  return (x->face > y->face) - (x->face < y->face);
}

int or_boundary_faces(int n_nodes, int n_tets, const int32_t* tets, const double* X,
                      int32_t* face_nodes, int32_t* face_tet, double* face_area) {
  (void)n_nodes;
  int64_t nf = 4 * (int64_t)n_tets;
  face_rec* r = (face_rec*)malloc(sizeof(face_rec) * (size_t)(nf ? nf : 1));
  for (int64_t t = 0; t < n_tets; ++t)
    for (int f = 0; f < 4; ++f) {
      int v[3];
      for (int k = 0; k < 3; ++k) v[k] = tets[4 * t + kFaceLocal[f][k]];
      qsort(v, 3, sizeof(int), cmp_int);
      face_rec* e = &r[4 * t + f];
      e->a = v[0];
      e->b = v[1];
      e->c = v[2];
      e->tet = (int32_t)t;
      e->face = f;
    }
  qsort(r, (size_t)nf, sizeof(face_rec), cmp_face);
  int64_t nb = 0;
  for (int64_t i = 0; i < nf;) {
    int64_t j = i + 1;
    while (j < nf && r[j].a == r[i].a && r[j].b == r[i].b && r[j].c == r[i].c) ++j;
    if (j - i == 1) r[nb++] = r[i];
    i = j;
  }
  /* canonical order: by owning tet, then local face */
  qsort(r, (size_t)nb, sizeof(face_rec), cmp_face_owner);
  if (face_nodes || face_tet || face_area) {
    for (int64_t k = 0; k < nb; ++k) {
      int64_t t = r[k].tet;
      int f = r[k].face;
      int32_t n0 = tets[4 * t + kFaceLocal[f][0]], n1 = tets[4 * t + kFaceLocal[f][1]],
              n2 = tets[4 * t + kFaceLocal[f][2]], no = tets[4 * t + kFaceOpp[f]];
      const double *x0 = X + 3 * (int64_t)n0, *x1 = X + 3 * (int64_t)n1, *x2 = X + 3 * (int64_t)n2,
                   *xo = X + 3 * (int64_t)no;
      double e1[3], e2[3], nrm[3], eo[3];
      for (int i = 0; i < 3; ++i) {
        e1[i] = x1[i] - x0[i];
        e2[i] = x2[i] - x0[i];
        eo[i] = xo[i] - x0[i];
      }
      nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
      nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
      nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
      double s = nrm[0] * eo[0] + nrm[1] * eo[1] + nrm[2] * eo[2];
      if (face_nodes) {
        face_nodes[3 * k + 0] = n0;
        /* outward: the normal (x1-x0)x(x2-x0) must point away from the opposite vertex */
        face_nodes[3 * k + 1] = s > 0.0 ? n2 : n1;
        face_nodes[3 * k + 2] = s > 0.0 ? n1 : n2;
      }
      if (face_tet) face_tet[k] = (int32_t)t;
      if (face_area)
        face_area[k] = 0.5 * sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    }
  }
  free(r);
  return (int)nb;
}

/* ------------------------------------------------------------------------------------------- */
/* assembly                                                                                     */

void or_mass_blocks(const or_scene* s, double* mass) {
  memset(mass, 0, sizeof(double) * (size_t)s->nnzb);
  for (int64_t t = 0; t < s->n_tets; ++t) {
    double m = s->rho[t] * s->vol[t] / 20.0;
    for (int f = 0; f < 4; ++f)
      for (int g = 0; g < 4; ++g) {
        int64_t slot = or_pattern_find(s->row_ptr, s->col, s->tets[4 * t + f], s->tets[4 * t + g]);
        mass[slot] += (f == g) ? 2.0 * m : m;
      }
  }
}

static inline void atomic_add(double* p, double v) {
#pragma omp atomic
  *p += v;
}

/* Quadrature points of the 3-point Dunavant rule on a face (triangular/simplex_quadrature.h:34-42). */
static const double kFaceW[3][3] = {{2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                                    {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0},
                                    {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0}};

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

/* Unit normal (x1 - x0) x (x2 - x0) of a deformed boundary face (zero for a degenerate face). */
static void face_normal(double xn[3][3], double nrm[3]) {
  double e1[3], e2[3];
  for (int r = 0; r < 3; ++r) {
    e1[r] = xn[1][r] - xn[0][r];
    e2[r] = xn[2][r] - xn[0][r];
  }
  nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
  nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
  nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
  const double nl = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
  for (int r = 0; r < 3; ++r) nrm[r] = nl > 0.0 ? nrm[r] / nl : 0.0;
}

int64_t or_assemble(const or_scene* s, const double* u, const double* ut, double t, int flags,
                    double* obj, double* g, double* H, int64_t* pair_out) {
  const int want_obj = flags & OR_ASM_OBJ, want_res = flags & OR_ASM_RES,
            want_hess = flags & OR_ASM_HESS;
  const int project = (flags & OR_ASM_PSD) != 0;
  const double dt = s->dt, dtfi2 = 1.0 / (dt * dt);
  const double dmp = s->mass_damping > 0.0 ? s->mass_damping / dt : 0.0; /* massDampingScale */
  double energy = 0.0;
  const int64_t N = s->n_nodes;
  if (want_res) memset(g, 0, sizeof(double) * 3 * (size_t)N);
  if (want_hess) {
    /* DRes <- massScale * M (mochi_physics/src/mochi_soft.cpp:249-262), massScale = 1/dt^2 + alpha/dt. */
    for (int64_t b = 0; b < s->nnzb; ++b) {
      double* blk = H + 9 * b;
      double m = s->mass[b] * (dtfi2 + dmp);
      for (int k = 0; k < 9; ++k) blk[k] = 0.0;
      blk[0] = blk[4] = blk[8] = m;
    }
  }

  /* Body terms: StressWork (fem_stress.h:107-262), GravityWork (fem_gravity.h:44-128),
   * InertiaWork (fem_inertia.h:55-137). */
#pragma omp parallel for schedule(static) reduction(+ : energy)
  for (int64_t e = 0; e < s->n_tets; ++e) {
    const int32_t* nd = s->tets + 4 * e;
    const double* dN = s->dN + 12 * e;
    const double w = s->vol[e];
    double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int f = 0; f < 4; ++f) {
      const double* uf = u + 3 * (int64_t)nd[f];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) F[r * 3 + c] += uf[r] * dN[3 * f + c];
    }
    double Psi, P[9], C[81];
    or_material(s->material, s->mu[e], s->lambda[e], F, project, s->psd_strategy, s->min_eig,
                want_obj ? &Psi : NULL, want_res ? P : NULL, want_hess ? C : NULL);
    const double rho = s->rho[e];
    /* inertia acceleration a_f = u_f - ut_f, consistent mass M_fg = rho w (1 + d_fg) / 20 */
    double a[4][3], asum[3] = {0, 0, 0};
    double dd[4][3], dsum[3] = {0, 0, 0}; /* mass damping: u - u_stage */
    for (int f = 0; f < 4; ++f)
      for (int r = 0; r < 3; ++r) {
        a[f][r] = u[3 * (int64_t)nd[f] + r] - ut[3 * (int64_t)nd[f] + r];
        asum[r] += a[f][r];
        dd[f][r] = (dmp > 0.0 && s->u_stage) ? u[3 * (int64_t)nd[f] + r] - s->u_stage[3 * (int64_t)nd[f] + r] : 0.0;
        dsum[r] += dd[f][r];
      }
    const double m = rho * w / 20.0;
    if (want_obj) {
      double xc[3] = {0, 0, 0};
      for (int f = 0; f < 4; ++f)
        for (int r = 0; r < 3; ++r)
          xc[r] += 0.25 * (s->X[3 * (int64_t)nd[f] + r] + u[3 * (int64_t)nd[f] + r]);
      double ein = 0.0, edm = 0.0;
      for (int r = 0; r < 3; ++r) {
        double sq = 0.0, sd = 0.0;
        for (int f = 0; f < 4; ++f) {
          sq += a[f][r] * a[f][r];
          sd += dd[f][r] * dd[f][r];
        }
        ein += m * (sq + asum[r] * asum[r]);
        edm += m * (sd + dsum[r] * dsum[r]);
      }
      energy += Psi * w - rho * w * (s->gravity[0] * xc[0] + s->gravity[1] * xc[1] +
                                     s->gravity[2] * xc[2]) +
                0.5 * dtfi2 * ein + 0.5 * dmp * edm;
    }
    if (want_res) {
      for (int f = 0; f < 4; ++f)
        for (int r = 0; r < 3; ++r) {
          double v = (P[r * 3 + 0] * dN[3 * f + 0] + P[r * 3 + 1] * dN[3 * f + 1] +
                      P[r * 3 + 2] * dN[3 * f + 2]) *
                     w;
          v -= rho * s->gravity[r] * w * 0.25;
          v += dtfi2 * m * (a[f][r] + asum[r]);
          v += dmp * m * (dd[f][r] + dsum[r]);
          atomic_add(&g[3 * (int64_t)nd[f] + r], v);
        }
    }
    /* Rayleigh stiffness damping (mochi_physics/src/mochi_soft.h:420-440): viscous stress about the
     * stage-start displacement, reference stiffness = the rest tangent = (lambda, mu) for these
     * isotropic materials */
    double dres[12], dK[144];
    const int sdamp = s->stiffness_damping > 0.0 && s->u_stage != NULL;
    if (sdamp) {
      double ue[12], us[12], de = 0.0;
      for (int f = 0; f < 4; ++f)
        for (int r = 0; r < 3; ++r) {
          ue[3 * f + r] = u[3 * (int64_t)nd[f] + r];
          us[3 * f + r] = s->u_stage[3 * (int64_t)nd[f] + r];
        }
      /* the reference stiffness (ComputeReferenceMaterialStiffnessVoigt): the tet's (lambda, mu), for
       * ARAP (0, mu / 2) */
      const double l0 = s->material == OR_MAT_ARAP ? 0.0 : s->lambda[e];
      const double m0 = s->material == OR_MAT_ARAP ? 0.5 * s->mu[e] : s->mu[e];
      or_stress_damping(dN, w, ue, us, s->stiffness_damping / dt, l0, m0,
                        s->stiffness_damping_geometric, project, want_obj ? &de : NULL, want_res ? dres : NULL,
                        want_hess ? dK : NULL);
      energy += de;
      if (want_res)
        for (int f = 0; f < 4; ++f)
          for (int r = 0; r < 3; ++r) atomic_add(&g[3 * (int64_t)nd[f] + r], dres[3 * f + r]);
    }
    if (want_hess) {
      for (int f = 0; f < 4; ++f)
        for (int gg = 0; gg < 4; ++gg) {
          int64_t slot = or_pattern_find(s->row_ptr, s->col, nd[f], nd[gg]);
          double* blk = H + 9 * slot;
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
              double k = 0.0;
              for (int j = 0; j < 3; ++j)
                for (int l = 0; l < 3; ++l)
                  k += dN[3 * f + j] * C[(r * 3 + j) * 9 + (c * 3 + l)] * dN[3 * gg + l];
              k *= w;
              if (sdamp) k += dK[(3 * f + r) * 12 + 3 * gg + c];
              atomic_add(&blk[r * 3 + c], k);
            }
        }
    }
  }

  /* Contact: boundary samples (P1Q3 trace elements) against kinematic colliders (rigid translations
   * with velocity vel), the penalty response with Coulomb / viscous friction and normal damping
   * (or_collision_response), integrated by TractionWork (fem_traction.h:58-178). The stage start is
   * u_stage at time t - dt (NULL: the current displacement). The contact set is the samples closer than
   * thr, plus with explicit normals those closer than thr at the stage start, which enter with d = thr
   * and the stage-start gradient (mochi_physics/src/mochi_stage_start_contact.cpp:205-318). */
  int64_t n_pairs = 0;
  int64_t cap = pair_out ? 3 * (int64_t)s->n_faces * (s->n_colliders > 0 ? s->n_colliders : 1) : 0;
  int64_t* pairs = pair_out ? (int64_t*)malloc(sizeof(int64_t) * (size_t)(cap ? cap : 1)) : NULL;
  if (s->n_colliders > 0) {
    or_contact_params cp;
    cp.k = s->k_contact;
    cp.t_half = s->t_half;
    cp.thr = s->thr;
    cp.max_align = s->max_align;
    cp.coulomb = s->coulomb;
    cp.falloff_vel = s->falloff_vel;
    cp.viscous = s->viscous;
    cp.normal_damping = s->normal_damping;
    cp.collider_normal = s->collider_normal;
    cp.explicit_normals = s->explicit_normals;
    cp.fade = s->fade;
    cp.implicit_normal_force = s->implicit_normal_force;
    cp.fitted = s->fitted;
    cp.model = s->friction_model;
    const int diss = cp.coulomb > 0.0 || cp.viscous > 0.0 || cp.normal_damping > 0.0;
    const int need_ss = diss || cp.explicit_normals;
    const double* us = s->u_stage ? s->u_stage : u;
    const double t0 = t - s->dt;
#pragma omp parallel for schedule(static) reduction(+ : energy)
    for (int64_t f = 0; f < s->n_faces; ++f) {
      const int32_t* fn = s->face_nodes + 3 * f;
      double xn[3][3], xn0[3][3], nrm[3], nrm0[3];
      for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) {
          xn[k][r] = s->X[3 * (int64_t)fn[k] + r] + u[3 * (int64_t)fn[k] + r];
          xn0[k][r] = s->X[3 * (int64_t)fn[k] + r] + us[3 * (int64_t)fn[k] + r];
        }
      face_normal(xn, nrm);
      face_normal(xn0, nrm0);
      const double wq = s->face_area[f] / 3.0;
      for (int q = 0; q < 3; ++q) {
        double xs[3], xs0[3];
        for (int r = 0; r < 3; ++r) {
          xs[r] = kFaceW[q][0] * xn[0][r] + kFaceW[q][1] * xn[1][r] + kFaceW[q][2] * xn[2][r];
          xs0[r] = kFaceW[q][0] * xn0[0][r] + kFaceW[q][1] * xn0[1][r] + kFaceW[q][2] * xn0[2][r];
        }
        for (int c = 0; c < s->n_colliders; ++c) {
          const or_collider* col = &s->colliders[c];
          double d, gr[3], d0 = 0.0, gr0[3] = {0.0, 0.0, 0.0};
          collider_sdf(col, xs, t, &d, gr);
          if (need_ss) collider_sdf(col, xs0, t0, &d0, gr0);
          const int cur = d < s->thr;
          const int ss = cp.explicit_normals && d0 < s->thr;
          if (!cur && !ss) continue;
          if (!cur) { /* in contact at the stage start only */
            d = s->thr;
            for (int r = 0; r < 3; ++r) gr[r] = gr0[r];
          }
          const double* ncol = cp.explicit_normals ? nrm0 : nrm;
          const double* nc = cp.explicit_normals ? gr0 : gr;
          if (nc[0] * ncol[0] + nc[1] * ncol[1] + nc[2] * ncol[2] > s->max_align) continue; /* masked */
          if (pairs) {
            int64_t slot;
#pragma omp atomic capture
            slot = n_pairs++;
            pairs[slot] = (3 * f + q) * (int64_t)s->n_colliders + c;
          } else {
#pragma omp atomic
            n_pairs++;
          }
          /* sample positions in the collider frame, now and at the stage start */
          double pos[3], pos0[3];
          for (int r = 0; r < 3; ++r) {
            pos[r] = xs[r] - col->vel[r] * t;
            pos0[r] = xs0[r] - col->vel[r] * t0;
          }
          double E, force[3], dforce[9];
          or_collision_response(&cp, d, gr, d0, gr0, ncol, pos, pos0, s->dt, 1, &E, force, dforce);
          if (want_obj) energy += E * wq;
          if (want_res)
            for (int k = 0; k < 3; ++k)
              for (int r = 0; r < 3; ++r)
                atomic_add(&g[3 * (int64_t)fn[k] + r], -force[r] * kFaceW[q][k] * wq);
          if (want_hess)
            for (int k = 0; k < 3; ++k)
              for (int l = 0; l < 3; ++l) {
                int64_t slot = or_pattern_find(s->row_ptr, s->col, fn[k], fn[l]);
                double wkl = kFaceW[q][k] * kFaceW[q][l] * wq;
                for (int r = 0; r < 3; ++r)
                  for (int cc = 0; cc < 3; ++cc)
                    atomic_add(&H[9 * slot + r * 3 + cc], -dforce[r * 3 + cc] * wkl);
              }
        }
      }
    }
  }
  if (pair_out) {
    qsort(pairs, (size_t)n_pairs, sizeof(int64_t), cmp_i64);
    memcpy(pair_out, pairs, sizeof(int64_t) * (size_t)n_pairs);
    free(pairs);
  }

  /* Dirichlet conditions (mochi_physics/src/mochi_solve.cpp:337-396). */
  for (int64_t i = 0; i < N; ++i) {
    if (!s->pin[i]) continue;
    for (int r = 0; r < 3; ++r)
      if (want_res && (s->pin[i] >> r & 1)) g[3 * i + r] = 0.0;
  }
  if (want_hess) {
    for (int64_t i = 0; i < N; ++i)
      for (int64_t b = s->row_ptr[i]; b < s->row_ptr[i + 1]; ++b) {
        int j = s->col[b];
        if (!s->pin[i] && !s->pin[j]) continue;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c)
            if ((s->pin[i] >> r & 1) || (s->pin[j] >> c & 1))
              H[9 * b + r * 3 + c] = (i == j && r == c) ? 1.0 : 0.0;
      }
  }
  if (obj) *obj = energy;
  return n_pairs;
}

/* ------------------------------------------------------------------------------------------- */
/* linear solver                                                                                */

void or_bsr_apply(int n, const int64_t* row_ptr, const int32_t* col, const double* H,
                  const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int64_t b = row_ptr[i]; b < row_ptr[i + 1]; ++b) {
      const double* h = H + 9 * b;
      const double* xj = x + 3 * (int64_t)col[b];
      s0 += h[0] * xj[0] + h[1] * xj[1] + h[2] * xj[2];
      s1 += h[3] * xj[0] + h[4] * xj[1] + h[5] * xj[2];
      s2 += h[6] * xj[0] + h[7] * xj[1] + h[8] * xj[2];
    }
    y[3 * i] = s0;
    y[3 * i + 1] = s1;
    y[3 * i + 2] = s2;
  }
}

static double dotv(int64_t n, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* Preconditioner setup: Jacobi (BlockJacobiPrec<1>) inverts the scalar diagonal; block Jacobi
 * inverts each 3x3 diagonal block (block_jacobi_prec.h:35-151). */
static void prec_setup(int n, const int64_t* row_ptr, const int32_t* col, const double* H, int kind,
                       double* P) {
  for (int64_t i = 0; i < n; ++i) {
    int64_t b = or_pattern_find(row_ptr, col, (int)i, (int)i);
    const double* d = H + 9 * b;
    if (kind == 1) {
      for (int r = 0; r < 3; ++r) P[3 * i + r] = 1.0 / d[r * 3 + r];
    } else if (kind == 2) {
      double c[9];
      cof3(d, c);
      double det = det3(d);
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) P[9 * i + r * 3 + cc] = c[cc * 3 + r] / det;
    }
  }
}

static void prec_apply(int n, int kind, const double* P, const double* r, double* z) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (kind == 0) {
      for (int k = 0; k < 3; ++k) z[3 * i + k] = r[3 * i + k];
    } else if (kind == 1) {
      for (int k = 0; k < 3; ++k) z[3 * i + k] = P[3 * i + k] * r[3 * i + k];
    } else {
      const double* B = P + 9 * i;
      for (int k = 0; k < 3; ++k)
        z[3 * i + k] = B[3 * k] * r[3 * i] + B[3 * k + 1] * r[3 * i + 1] + B[3 * k + 2] * r[3 * i + 2];
    }
  }
}

int or_stop_status(double rr, double bb, double rel_tol, double abs_tol, double rel_div_tol) {
  const double div = (bb * rel_div_tol) * rel_div_tol;
  const double conv = fmax(abs_tol * abs_tol, (bb * rel_tol) * rel_tol);
  if (!isfinite(rr) || rr > div || rr < -conv) return 3;
  if (rr < 0.0) rr = 0.0;
  if (rr <= conv) return rr <= abs_tol * abs_tol ? 2 : 1;
  return 0;
}

or_pcg_status or_pcg(int n, const int64_t* row_ptr, const int32_t* col, const double* H,
                     const double* b, double* x, const or_pcg_params* prm) {
  const int64_t m = 3 * (int64_t)n;
  double* r = (double*)malloc(sizeof(double) * (size_t)m);
  double* q = (double*)malloc(sizeof(double) * (size_t)m);
  double* p = (double*)malloc(sizeof(double) * (size_t)m);
  double* z = (double*)malloc(sizeof(double) * (size_t)m);
  double* P = (double*)malloc(sizeof(double) * (size_t)(9 * n > 0 ? 9 * n : 1));
  prec_setup(n, row_ptr, col, H, prm->precond, P);
  or_pcg_status st = {0, 0.0, 0.0, 0};
  memcpy(r, b, sizeof(double) * (size_t)m);
  /* StatusResidualL2::SetScaling: scale = |b|^2 (stopping_criterion.h:140-144, 92-98). */
  const double bb = dotv(m, b, b);
  /* thresholds: or_stop_status */
  if (!prm->zero_guess) {
    or_bsr_apply(n, row_ptr, col, H, x, q);
    for (int64_t i = 0; i < m; ++i) r[i] -= q[i];
  }
  double rr = dotv(m, r, r);
#define OR_CHECK(it_)                                                                      \
  do {                                                                                     \
    st.res_norm = sqrt(rr < 0 ? 0 : rr);                                                   \
    st.rel_res_norm = bb == 0.0 ? 0.0 : sqrt((rr < 0 ? 0 : rr) / bb);                      \
    const int cls_ = or_stop_status(rr, bb, prm->rel_tol, prm->abs_tol, prm->rel_div_tol); \
    if (cls_ != 0) {                                                                       \
      st.num_iter = (it_);                                                                 \
      st.convergence = cls_ == 3 ? 3 : 1;                                                  \
      goto done;                                                                           \
    }                                                                                      \
  } while (0)
  OR_CHECK(0);
  prec_apply(n, prm->precond, P, r, z);
  memcpy(p, z, sizeof(double) * (size_t)m);
  double rz = dotv(m, r, z);
  for (int it = 1; it <= prm->max_iter; ++it) {
    or_bsr_apply(n, row_ptr, col, H, p, q);
    double pq = dotv(m, p, q);
    double alpha = rz / pq;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rr = dotv(m, r, r);
    OR_CHECK(it);
    double beta_pr = 0.0;
    if (prm->polak_ribiere && it > 1) beta_pr = dotv(m, r, z);
    prec_apply(n, prm->precond, P, r, z);
    double rz_old = rz;
    rz = dotv(m, r, z);
    if (rz == 0.0) {
      st.num_iter = it;
      st.convergence = 3;
      goto done;
    }
    double beta = (rz - beta_pr) / rz_old;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) p[i] = z[i] + beta * p[i];
  }
  st.num_iter = prm->max_iter;
  st.convergence = 2;
done:
#undef OR_CHECK
  free(r);
  free(q);
  free(p);
  free(z);
  free(P);
  return st;
}

/* ------------------------------------------------------------------------------------------- */
/* Newton step                                                                                  */

void or_default_newton_params(or_newton_params* p) {
  /* nonlinear_solver_params.h:338-457 with maxIter raised for convergence to relTol. */
  p->max_iter = 50;
  p->rel_tol = 1e-6;
  p->abs_tol = 1e-3;
  p->rel_step_tol = 10.0 * DBL_EPSILON;
  p->ls_max_iter = 4;
  p->ls_alpha = 0.5;
  p->ew_forcing = 0;
  p->rel_div_tol = 1e4;
  p->abs_div_tol = 1e9;
  p->lin.rel_tol = 1e-6;
  p->lin.abs_tol = 1e-9;
  p->lin.rel_div_tol = 1e10;
  p->lin.max_iter = 10000;
  p->lin.precond = 1;
  p->lin.polak_ribiere = 1;
  p->lin.zero_guess = 1;
}

static double norm2(int64_t n, const double* a) { return sqrt(dotv(n, a, a)); }

or_newton_status or_step(const or_scene* s_in, double* u, double* v, double t,
                         const or_newton_params* prm, const double* warm) {
  const int64_t m = 3 * (int64_t)s_in->n_nodes;
  double* u0 = (double*)malloc(sizeof(double) * (size_t)m);
  double* ut = (double*)malloc(sizeof(double) * (size_t)m);
  double* g = (double*)malloc(sizeof(double) * (size_t)m);
  double* dx = (double*)malloc(sizeof(double) * (size_t)m);
  double* ubase = (double*)malloc(sizeof(double) * (size_t)m);
  double* H = (double*)malloc(sizeof(double) * 9 * (size_t)s_in->nnzb);
  memcpy(u0, u, sizeof(double) * (size_t)m);
  or_scene sl = *s_in; /* the stage-start displacement of mass damping is this step's start */
  sl.u_stage = u0;
  const or_scene* s = &sl;
  /* x~ = x0 + dt v0 (GatherPredTarget, batched_element_utils.h:90-123) */
  for (int64_t i = 0; i < m; ++i) ut[i] = u0[i] + s->dt * v[i];
  or_newton_status st;
  memset(&st, 0, sizeof(st));
  or_pcg_params lin = prm->lin;
  double res_prev = 0.0, lin_res = 0.0;
  double dxnorm = 0.0;
  int have_g = 0;
  for (;;) {
    const int first = st.newton_iters == 0;
    /* newton_solver.cpp:650-668: residual always; DRes together with it on the first pass. */
    if (!have_g || first) {
      st.n_contacts = or_assemble(s, u, ut, t, OR_ASM_RES | (first ? (OR_ASM_HESS | OR_ASM_PSD) : 0),
                                  NULL, g, H, NULL);
    }
    double res = norm2(m, g);
    if (first) st.res_norm0 = res;
    st.res_norm = res;
    /* stop criteria in the reference order (newton_solver.cpp:303-313) */
    if (res <= prm->abs_tol || (!first && res <= prm->rel_tol * st.res_norm0)) {
      st.convergence = 1;
      break;
    }
    if (st.newton_iters >= prm->max_iter) {
      st.convergence = 2;
      break;
    }
    if (!first && dxnorm <= prm->rel_step_tol * norm2(m, u)) {
      st.convergence = 2;
      break;
    }
    /* Eisenstat-Walker choice 2 (newton_solver.cpp:452-468) */
    if (prm->ew_forcing == 2) {
      const double kMax = 0.01, kSafe = 0.01, kMin = 100.0 * DBL_EPSILON;
      double eta;
      if (first) {
        eta = kMax;
      } else {
        double a = 0.5 + 0.5 * sqrt(5.0), gam = 0.9;
        double safe = gam * pow(lin.rel_tol, a);
        eta = gam * pow(res / res_prev, a);
        if (safe > kSafe) eta = fmax(eta, safe);
        eta = fmin(fmax(eta, kMin), kMax);
      }
      lin.rel_tol = eta;
    }
    (void)lin_res;
    res_prev = res;
    st.newton_iters++;
    if (!first)
      or_assemble(s, u, ut, t, OR_ASM_HESS | OR_ASM_PSD, NULL, NULL, H, NULL);
    /* linear solve H dx = g from zero (newton_solver.cpp:746-752) or from the supplied guess */
    if (warm) {
      memcpy(dx, warm, sizeof(double) * (size_t)m);
      lin.zero_guess = 0;
    } else {
      memset(dx, 0, sizeof(double) * (size_t)m);
      lin.zero_guess = 1;
    }
    or_pcg_status ls = or_pcg(s->n_nodes, s->row_ptr, s->col, H, g, dx, &lin);
    st.cg_iters += ls.num_iter;
    lin_res = ls.res_norm;
    dxnorm = norm2(m, dx);
    /* ResidualNorm line search along -dx (line_search.h:300-336); without improvement the final
     * iterate is kept (the reference's retry re-assembles an identical Hessian for this model). */
    memcpy(ubase, u, sizeof(double) * (size_t)m);
    double scale = 1.0;
    for (int it = 0; it < prm->ls_max_iter; ++it) {
      if (it > 0) scale *= prm->ls_alpha;
      for (int64_t i = 0; i < m; ++i) u[i] = ubase[i] - scale * dx[i];
      st.n_contacts = or_assemble(s, u, ut, t, OR_ASM_RES, NULL, g, NULL, NULL);
      st.ls_iters++;
      if (norm2(m, g) <= res) break;
    }
    have_g = 1;
    /* explosion control (newton_solver.cpp:841-874) */
    double rn = norm2(m, g);
    if (rn > prm->rel_div_tol * st.res_norm0 || rn > prm->abs_div_tol || !isfinite(rn)) {
      st.res_norm = rn;
      st.convergence = 3;
      break;
    }
  }
  /* backward Euler velocity update */
  for (int64_t i = 0; i < m; ++i) v[i] = (u[i] - u0[i]) / s->dt;
  free(u0);
  free(ut);
  free(g);
  free(dx);
  free(ubase);
  free(H);
  return st;
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void or_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
