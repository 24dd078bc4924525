// ref_shim.cpp — C entry points over the REFERENCE's own code, compiled from its sources in the
// build container by oracle/build_ref.sh into oracle/_ref/libsdx_ref.so (test infrastructure only).
//
// Each entry point calls the reference function named beside it, unmodified, in its FP64 build
// (MOCHI_USE_DOUBLE_PRECISION=1). The shim itself only marshals plain arrays in and out; it is used
// to pin the C restatement in oracle/sdx_oracle.c and as the CPU "reference" baseline kernels.
#include <mochi_core/contact/contact_params.h>
#include <mochi_core/contact/contact_utils.h>
#include <mochi_core/element_operations/fem_stress.h>
#include <mochi_core/element_operations/fem_stress_damping.h>
#include <mochi_core/materials/reference_material_stiffness.h>
#include <mochi_core/elements/tetrahedral/finite_element.h>
#include <mochi_core/linear_algebra/block_sparse_matrix.h>
#include <mochi_core/linear_algebra/krylov/block_jacobi_prec.h>
#include <mochi_core/linear_algebra/krylov/pcg.h>
#include <mochi_core/linear_algebra/matrix.h>
#include <mochi_core/materials/batched_arap.h>
#include <mochi_core/materials/batched_linear_elastic.h>
#include <mochi_core/materials/batched_smith_neo_hookean.h>
#include <mochi_core/materials/batched_st_venant_kirchhoff.h>
#include <mochi_core/solvers/krylov_solver.h>
#include <mochi_core/utils/activations.h>

#include <cstdint>
#include <cstring>

using namespace mochi;

namespace {
MaterialPsdStrategy ToStrategy(int s) {
  switch (s) {
    case 0:
      return MaterialPsdStrategy::None;
    case 2:
      return MaterialPsdStrategy::AbsEigenProjection;
    case 3:
      return MaterialPsdStrategy::Fast;
    default:
      return MaterialPsdStrategy::Projection;
  }
}
} // namespace

extern "C" {

// BatchedSmithNeoHookeanConstitutiveResponse<1> (mochi_core/src/materials/batched_smith_neo_hookean.cpp:29).
// oracle: 0 None, 1 Correct, 2 Conservative (MaterialPsdOracle).
void ref_smith_nh(double mu, double lambda, const double* F9, int project, int psd_strategy,
                  int oracle, double* energy, double* P9, double* C81) {
  materials::BatchLameParams<1> p;
  p.mu = BatchReal<1>{mu};
  p.lambda = BatchReal<1>{lambda};
  p.psdStrategy = ToStrategy(psd_strategy);
  BatchReal3x3<1> F{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) F[i][j] = BatchReal<1>{F9[i * 3 + j]};
  BatchDouble<1> e{};
  BatchReal3x3<1> pk1{};
  NdArray<BatchReal3x3<1>, 3, 3> C{};
  materials::BatchedSmithNeoHookeanConstitutiveResponse<1>(
      p, F, &e, &pk1, &C, project != 0, static_cast<materials::MaterialPsdOracle>(oracle));
  if (energy) *energy = Get0(e);
  if (P9)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) P9[i * 3 + j] = Get0(pk1[i][j]);
  if (C81)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) C81[(i * 3 + j) * 9 + k * 3 + l] = Get0(C[i][j][k][l]);
}

// BatchedStVenantKirchhoffConstitutiveResponse<1> (mochi_core/src/materials/batched_st_venant_kirchhoff.cpp:29),
// BatchedLinearElasticConstitutiveResponse<1> (batched_linear_elastic.cpp:27) and
// BatchedArapConstitutiveResponse<1> (batched_arap.cpp:29, stiffness = mu); material 1 / 2 / 5 as in
// SoftMaterialType.
void ref_material(int material, double mu, double lambda, const double* F9, int project, int psd_strategy,
                  double* energy, double* P9, double* C81) {
  materials::BatchLameParams<1> p;
  p.mu = BatchReal<1>{mu};
  p.lambda = BatchReal<1>{lambda};
  p.psdStrategy = ToStrategy(psd_strategy);
  BatchReal3x3<1> F{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) F[i][j] = BatchReal<1>{F9[i * 3 + j]};
  BatchDouble<1> e{};
  BatchReal3x3<1> pk1{};
  NdArray<BatchReal3x3<1>, 3, 3> C{};
  if (material == 1) {
    materials::BatchedStVenantKirchhoffConstitutiveResponse<1>(p, F, &e, &pk1, &C, project != 0);
  } else if (material == 5) {
    materials::BatchArapParams<1> a;
    a.stiffness = BatchReal<1>{mu};
    a.psdStrategy = ToStrategy(psd_strategy);
    materials::BatchedArapConstitutiveResponse<1>(a, F, &e, &pk1, &C, project != 0);
  } else {
    materials::BatchedLinearElasticConstitutiveResponse<1>(p, F, &e, &pk1, &C, project != 0);
  }
  if (energy) *energy = Get0(e);
  if (P9)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) P9[i * 3 + j] = Get0(pk1[i][j]);
  if (C81)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) C81[(i * 3 + j) * 9 + k * 3 + l] = Get0(C[i][j][k][l]);
}

// fem::StressDampingWork<1> on one P1 tet (mochi_core/.../element_operations/fem_stress_damping.h:29-501),
// isotropic reference stiffness C0 = (lambda0, mu0) in Voigt form, stiffness damping factor kappa.
void ref_stress_damping(const double* X12, const double* u12, const double* uss12, double kappa,
                        double lambda0, double mu0, int geometric, int project, double* energy,
                        double* res12, double* K144) {
  Real3 coords[4];
  for (int i = 0; i < 4; ++i) coords[i] = Real3{X12[3 * i], X12[3 * i + 1], X12[3 * i + 2]};
  Int4 conn[1] = {Int4{0, 1, 2, 3}};
  using Elem = tetrahedral::Pk3DElement<1, 1>;
  Elem elem(0, Span<Real3 const>(coords, 4), Span<Int4 const>(conn, 1));
  NdArray<int, 1> idx{0};
  fem::BatchElementVector<1, Elem> disp{}, ss{};
  for (int i = 0; i < 12; ++i) {
    disp[i] = BatchReal<1>{u12[i]};
    ss[i] = BatchReal<1>{uss12[i]};
  }
  NdArray<BatchReal<1>, 6, 6> c0{};
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) {
      double v = 0.0;
      if (a < 3 && b < 3) v = lambda0 + (a == b ? 2.0 * mu0 : 0.0);
      if (a >= 3 && a == b) v = mu0;
      c0[a][b] = BatchReal<1>{v};
    }
  BatchDouble<1> e{0.0};
  fem::BatchElementVector<1, Elem> res{};
  fem::BatchElementMatrix<1, Elem> K{};
  fem::StressDampingWork<1>(idx, Span<Elem const>(&elem, 1), disp, ss, &e, &res, &K, project != 0,
                            geometric != 0, kappa, c0, /*materialIsIsotropic*/ true);
  *energy = Get0(e);
  for (int i = 0; i < 12; ++i) res12[i] = Get0(res[i]);
  for (int i = 0; i < 144; ++i) K144[i] = Get0(K[i]);
}

// ComputeReferenceMaterialStiffnessVoigt<1> (mochi_core/.../materials/reference_material_stiffness.h:67)
// of material 0 (Smith Neo-Hookean), 1 (StVK) or 2 (linear elastic).
void ref_reference_stiffness(int material, double mu, double lambda, double* c0v36) {
  auto response = [&](NdArray<int, 1> const&, auto const& F, auto* en, auto* pk1, auto* tan, bool psd) {
    materials::BatchLameParams<1> p;
    p.mu = BatchReal<1>{mu};
    p.lambda = BatchReal<1>{lambda};
    p.psdStrategy = MaterialPsdStrategy::None;
    if (material == 1) {
      materials::BatchedStVenantKirchhoffConstitutiveResponse<1>(p, F, en, pk1, tan, psd);
    } else if (material == 5) {
      materials::BatchArapParams<1> a;
      a.stiffness = BatchReal<1>{mu};
      a.psdStrategy = MaterialPsdStrategy::None;
      materials::BatchedArapConstitutiveResponse<1>(a, F, en, pk1, tan, psd);
    } else if (material == 2)
      materials::BatchedLinearElasticConstitutiveResponse<1>(p, F, en, pk1, tan, psd);
    else
      materials::BatchedSmithNeoHookeanConstitutiveResponse<1>(p, F, en, pk1, tan, psd,
                                                               materials::MaterialPsdOracle::Correct);
  };
  auto c0 = materials::ComputeReferenceMaterialStiffnessVoigt<1>(NdArray<int, 1>{0}, response);
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) c0v36[a * 6 + b] = Get0(c0[a][b]);
}

// PolyReLU (mochi_core/include/mochi_core/utils/activations.h:113).
void ref_polyrelu(double x, double t, double shift, double* f, double* df, double* ddf) {
  PolyReLU<double>(x, t, shift, *f, *df, *ddf);
}

// ComputeBatchContactPenaltyForceDForce<1> (mochi_core/include/mochi_core/contact/contact_utils.h:498).
// dforce6 = (xx, yy, zz, xy, xz, yz).
void ref_penalty(double d, const double* grad3, double k, double t_half, double thr, double* energy,
                 double* force3, double* dforce6) {
  ContactParams params;
  params.penaltyCoefficient = k;
  params.penaltySmoothingHalfDistance = t_half;
  params.penaltyThresholdDefault = thr;
  params.penaltyThresholdExtraPadding = 0;
  ContactEvalConfig config{};
  config.addPadding = false;
  BatchDouble<1> e{};
  BatchReal3<1> f{};
  BatchReal6<1> df{};
  BatchReal<1> fn{};
  BatchReal3<1> g{BatchReal<1>{grad3[0]}, BatchReal<1>{grad3[1]}, BatchReal<1>{grad3[2]}};
  ComputeBatchContactPenaltyForceDForce<1>(
      e, f, df, fn, BatchReal<1>{d}, g, ~SimdZero<BatchReal<1>>(), BatchReal<1>{1.0}, params,
      config, true, true, true, false);
  *energy = Get0(e);
  for (int i = 0; i < 3; ++i) force3[i] = Get0(f[i]);
  for (int i = 0; i < 6; ++i) dforce6[i] = Get0(df[i]);
}

// ComputeBatchCollisionForceDForce<1, GradTarget::Current> (mochi_core/include/mochi_core/contact/
// contact_utils.h:1003-1230): the penalty response plus Coulomb / viscous friction and normal viscous
// damping (ComputeBatchContactDissipationForceDForce, contact_utils.h:627-960) of one sample, every
// vector in the collider frame. d, grad: implicit SDF value and gradient; d_ss, grad_ss: stage-start
// ones (read only with explicit normals); n_col: the colliding surface normal; p, p_ss: the sample's
// current and stage-start positions. model: 0 C1Regularized, 1 CinfRegularized. dforce9 row-major.
void ref_collision_response(double d, const double* grad3, double d_ss, const double* grad_ss3,
                            const double* n_col3, const double* p3, const double* p_ss3, double k,
                            double t_half, double thr, double max_align, double coulomb,
                            double falloff_vel, double viscous, double normal_damping,
                            int collider_normal, int valid_colliding_normals, int explicit_normals,
                            int fade, int implicit_normal_force, int fitted, int model, double dt,
                            int unit_grad, double* energy, double* force3, double* dforce9) {
  ContactParams params;
  params.penaltyCoefficient = k;
  params.penaltySmoothingHalfDistance = t_half;
  params.penaltyThresholdDefault = thr;
  params.penaltyThresholdExtraPadding = 0;
  params.maxAlignmentNormals = max_align;
  params.coulombFrictionCoefficient = coulomb;
  params.frictionFalloffVel = falloff_vel;
  params.viscousFrictionCoefficient = viscous;
  params.normalViscousDampingCoefficient = normal_damping;
  params.frictionWithColliderNormal = collider_normal != 0;
  ContactEvalConfig config{};
  config.addPadding = false;
  config.validCollidingNormals = valid_colliding_normals != 0;
  config.explicitNormals = explicit_normals != 0;
  config.fadeFriction = fade != 0;
  config.implicitNormalForceForDissipation = implicit_normal_force != 0;
  config.useFittedHessian = fitted != 0;
  config.frictionModel = model == 1 ? CoulombFrictionModel::CinfRegularized : CoulombFrictionModel::C1Regularized;
  double e[1] = {0.0};
  Real3 f[1];
  VMatrix3x3r df[1];
  real dist[1] = {d}, dist_ss[1] = {d_ss};
  Real3 g[1] = {Real3{grad3[0], grad3[1], grad3[2]}};
  Real3 g_ss[1] = {Real3{grad_ss3[0], grad_ss3[1], grad_ss3[2]}};
  Real3 nc[1] = {Real3{n_col3[0], n_col3[1], n_col3[2]}};
  Real3 pc[1] = {Real3{p3[0], p3[1], p3[2]}};
  Real3 pss[1] = {Real3{p_ss3[0], p_ss3[1], p_ss3[2]}};
  ComputeBatchCollisionForceDForce<1, GradTarget::Current>(
      Span<double>(e, 1), Span<Real3>(f, 1), Span<VMatrix3x3r>(df, 1), Span<real const>(dist, 1),
      Span<Real3 const>(g, 1), Span<real const>(dist_ss, 1), Span<Real3 const>(g_ss, 1),
      Span<Real3 const>(nc, 1), Span<Real3 const>(pc, 1), Span<Real3 const>(pss, 1), params, config, dt,
      true, true, true, unit_grad != 0);
  *energy = e[0];
  for (int i = 0; i < 3; ++i) force3[i] = f[0][i];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) dforce9[3 * i + j] = df[0][i][j];
}

// fem::StressWork<1> over one Pk3DElement<1,1> built from rest coordinates (mochi_core/include/
// mochi_core/element_operations/fem_stress.h:107), Smith Neo-Hookean response, PSD oracle Correct.
// X12 = 4 rest nodes, u12 = 4 nodal displacements. res12 / K144 are overwritten.
void ref_stress_work(const double* X12, const double* u12, double mu, double lambda, int project,
                     int psd_strategy, double* energy, double* res12, double* K144) {
  Real3 coords[4];
  for (int i = 0; i < 4; ++i) coords[i] = Real3{X12[3 * i], X12[3 * i + 1], X12[3 * i + 2]};
  Int4 conn[1] = {Int4{0, 1, 2, 3}};
  using Elem = tetrahedral::Pk3DElement<1, 1>;
  Elem elem(0, Span<Real3 const>(coords, 4), Span<Int4 const>(conn, 1));
  NdArray<int, 1> idx{0};
  fem::BatchElementVector<1, Elem> disp{};
  for (int i = 0; i < 12; ++i) disp[i] = BatchReal<1>{u12[i]};
  BatchDouble<1> e{0.0};
  fem::BatchElementVector<1, Elem> res{};
  fem::BatchElementMatrix<1, Elem> K{};
  auto constitutive = [&](NdArray<int, 1> const&, auto const& F, auto* en, auto* pk1, auto* tan,
                          bool psd) {
    materials::BatchLameParams<1> p;
    p.mu = BatchReal<1>{mu};
    p.lambda = BatchReal<1>{lambda};
    p.psdStrategy = ToStrategy(psd_strategy);
    materials::BatchedSmithNeoHookeanConstitutiveResponse<1>(
        p, F, en, pk1, tan, psd, materials::MaterialPsdOracle::Correct);
  };
  fem::StressWork<1>(idx, Span<Elem const>(&elem, 1), disp, &e, &res, &K, project != 0,
                     constitutive);
  *energy = Get0(e);
  for (int i = 0; i < 12; ++i) res12[i] = Get0(res[i]);
  for (int i = 0; i < 144; ++i) K144[i] = Get0(K[i]);
}

// krylov::PCG (mochi_core/include/mochi_core/linear_algebra/krylov/pcg.h:70) with the residual-L2
// stop test (stopping_criterion.h:110), operator = scalar CSR matrix, preconditioner = Jacobi (the
// inverse diagonal) or identity. Returns the iteration count; writes x, |r|, |r|/|b|, status.
int ref_pcg_csr(int n, const int64_t* row_ptr, const int32_t* col, const double* val,
                const double* b, double* x, double rel_tol, double abs_tol, double rel_div_tol,
                int max_iter, int jacobi, int polak_ribiere, int zero_guess, double* res_norm,
                double* rel_res_norm, int* convergence) {
  ColumnVector<double> bv(n), xv(n), dinv(n);
  for (int i = 0; i < n; ++i) {
    bv[i] = b[i];
    xv[i] = x[i];
    double d = 0.0;
    for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
      if (col[k] == i) d = val[k];
    dinv[i] = jacobi ? 1.0 / d : 1.0;
  }
  auto opA = [&](auto const& in, auto& out) {
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += val[k] * in[col[k]];
      out[i] = s;
    }
  };
  auto opP = [&](auto const& in, auto& out) {
    for (int i = 0; i < n; ++i) out[i] = dinv[i] * in[i];
  };
  krylov::StatusResidualL2<krylov::UsualDot, double> stop{rel_tol, abs_tol, rel_div_tol};
  auto st = krylov::PCG(opA, bv, xv, opP, max_iter, stop, false, VerbosityLevel::Silent,
                        polak_ribiere != 0,
                        zero_guess ? InitialGuessHint::Zero : InitialGuessHint::Unknown);
  for (int i = 0; i < n; ++i) x[i] = xv[i];
  *res_norm = st.residualNorm;
  *rel_res_norm = st.relativeResidualNorm;
  *convergence = static_cast<int>(st.convergence);
  return st.numIterDone;
}

// krylov::PCG as ref_pcg_csr, in the build's own precision mochi::real (mochi_config.h:110-116): matrix
// values, vectors, dot products and the stop test in float when the shim is compiled with
// MOCHI_USE_DOUBLE_PRECISION=0 (the reference's FP32 mode), in double otherwise.
int ref_pcg_csr_real(int n, const int64_t* row_ptr, const int32_t* col, const double* val,
                     const double* b, double* x, double rel_tol, double abs_tol, double rel_div_tol,
                     int max_iter, int jacobi, int polak_ribiere, int zero_guess, double* res_norm,
                     double* rel_res_norm, int* convergence) {
  ColumnVector<real> bv(n), xv(n), dinv(n);
  const int64_t nnz = row_ptr[n];
  DynamicArray<real> v(nnz);
  for (int64_t k = 0; k < nnz; ++k) v[k] = static_cast<real>(val[k]);
  for (int i = 0; i < n; ++i) {
    bv[i] = static_cast<real>(b[i]);
    xv[i] = static_cast<real>(x[i]);
    real d = 0;
    for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
      if (col[k] == i) d = v[k];
    dinv[i] = jacobi ? real(1) / d : real(1);
  }
  auto opA = [&](auto const& in, auto& out) {
    for (int i = 0; i < n; ++i) {
      real s = 0;
      for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += v[k] * in[col[k]];
      out[i] = s;
    }
  };
  auto opP = [&](auto const& in, auto& out) {
    for (int i = 0; i < n; ++i) out[i] = dinv[i] * in[i];
  };
  krylov::StatusResidualL2<krylov::UsualDot, real> stop{static_cast<real>(rel_tol), static_cast<real>(abs_tol),
                                                        static_cast<real>(rel_div_tol)};
  auto st = krylov::PCG(opA, bv, xv, opP, max_iter, stop, false, VerbosityLevel::Silent, polak_ribiere != 0,
                        zero_guess ? InitialGuessHint::Zero : InitialGuessHint::Unknown);
  for (int i = 0; i < n; ++i) x[i] = xv[i];
  *res_norm = st.residualNorm;
  *rel_res_norm = st.relativeResidualNorm;
  *convergence = static_cast<int>(st.convergence);
  return st.numIterDone;
}

// the build's floating-point mode: 8 (double) or 4 (float) bytes per mochi::real
int ref_real_size(void) { return static_cast<int>(sizeof(real)); }

// mochi::BlockSparseMatrix<double, 3> (mochi_core/include/mochi_core/linear_algebra/block_sparse_matrix.h:63)
// on the block pattern (ptr, idx), every scalar entry written through its own SetValue (:230-238, which
// places it by FindValueIndex, :459-475); copies out Values(), i.e. the values in the reference's storage
// layout. blocks: 9 row-major values per block.
void ref_bsr3_values(int n_block_rows, const int32_t* ptr, const int32_t* idx, const double* blocks,
                     double* values_out) {
  const int nnzb = ptr[n_block_rows];
  DynamicArray<int> p(ptr, ptr + n_block_rows + 1), ix(idx, idx + nnzb);
  DynamicArray<double> v(9 * (size_t)nnzb);
  BlockSparseMatrix<double, 3> A(n_block_rows, std::move(p), std::move(ix), std::move(v));
  A.SetZero();
  for (int br = 0; br < n_block_rows; ++br)
    for (int k = ptr[br]; k < ptr[br + 1]; ++k)
      for (int e = 0; e < 9; ++e) A.SetValue(3 * br + e / 3, 3 * idx[k] + e % 3, blocks[9 * (size_t)k + e]);
  auto const V = A.Values();
  for (size_t i = 0; i < V.size(); ++i) values_out[i] = V[i];
}

// krylov::PCG (pcg.h:70) on a mochi::BlockSparseMatrix<double, 3> holding `values` as its Values() (the
// reference's layout), applied by the matrix's own Apply (block_sparse_matrix.h:1134), with the
// reference's BlockJacobiPrec (block_jacobi_prec.h:35): precond 1 = Jacobi (block size 1), 2 = block
// Jacobi (3x3), 0 = none; residual-L2 stop test. Returns the iteration count.
int ref_bsr3_pcg(int n_block_rows, const int32_t* ptr, const int32_t* idx, const double* values,
                 const double* b, double* x, double rel_tol, double abs_tol, double rel_div_tol, int max_iter,
                 int precond, int polak_ribiere, int zero_guess, double* res_norm, double* rel_res_norm,
                 int* convergence) {
  const int nnzb = ptr[n_block_rows];
  const int n = 3 * n_block_rows;
  DynamicArray<int> p(ptr, ptr + n_block_rows + 1), ix(idx, idx + nnzb);
  DynamicArray<double> v(values, values + 9 * (size_t)nnzb);
  BlockSparseMatrix<double, 3> A(n_block_rows, std::move(p), std::move(ix), std::move(v));
  ColumnVector<double> bv(n), xv(n);
  for (int i = 0; i < n; ++i) {
    bv[i] = b[i];
    xv[i] = x[i];
  }
  krylov::StatusResidualL2<krylov::UsualDot, double> stop{rel_tol, abs_tol, rel_div_tol};
  auto const hint = zero_guess ? InitialGuessHint::Zero : InitialGuessHint::Unknown;
  LinearSolverStatus st;
  if (precond == 1) {
    krylov::BlockJacobiPrec<double, 1> P(A);
    st = krylov::PCG(A, bv, xv, P, max_iter, stop, false, VerbosityLevel::Silent, polak_ribiere != 0, hint);
  } else if (precond == 2) {
    krylov::BlockJacobiPrec<double, 3> P(A);
    st = krylov::PCG(A, bv, xv, P, max_iter, stop, false, VerbosityLevel::Silent, polak_ribiere != 0, hint);
  } else {
    auto opP = [&](auto const& in, auto& out) {
      for (int i = 0; i < n; ++i) out[i] = in[i];
    };
    st = krylov::PCG(A, bv, xv, opP, max_iter, stop, false, VerbosityLevel::Silent, polak_ribiere != 0, hint);
  }
  for (int i = 0; i < n; ++i) x[i] = xv[i];
  *res_norm = st.residualNorm;
  *rel_res_norm = st.relativeResidualNorm;
  *convergence = static_cast<int>(st.convergence);
  return st.numIterDone;
}

} // extern "C"
