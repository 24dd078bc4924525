/*
 * sdx_oracle.h — CPU oracle (test infrastructure only) for the implicit soft-body step.
 *
 * This is a plain-C, FP64 restatement of the reference's algorithm for the soft-body hot
 * path. It is the CHECKER used by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline leg. It is never part of the product path: the CUDA library fails loudly
 * when its extension is missing and never calls into this file.
 *
 * Parity pins (see tests/test_oracle_golden.py):
 *   - Smith Neo-Hookean energy / PK1 / tangent: golden vectors of the reference test suite
 *     (mochi_core/test/data/material_test_data.h, smith block, E = 1, nu = 0.4) and, in the
 *     build container, the reference's own BatchedSmithNeoHookeanConstitutiveResponse compiled
 *     from source into oracle/_ref (projected tangents included).
 *   - Jacobi-PCG: the reference's 100x100 SPD golden system (krylov_solver_test_data.h) and
 *     the inline 64x64 tridiagonal system (krylov_solver_test_helpers.h:55-120).
 *   - PolyReLU / penalty response: the reference's header-only functions in oracle/_ref.
 *
 * All reference citations are paths inside superdex_physics/libraries/mochi/.
 */
#ifndef SDX_ORACLE_H
#define SDX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PSD strategies, same meaning as MaterialPsdStrategy (mochi_core/.../materials/material_types.h:52). */
enum { OR_PSD_NONE = 0, OR_PSD_PROJECTION = 1, OR_PSD_ABS_EIGEN = 2, OR_PSD_FAST = 3 };

/* Smith et al. 2018 stable Neo-Hookean response.
 * Follows mochi_core/src/materials/batched_smith_neo_hookean.cpp:29-269 (PSD oracle "Correct").
 * F, P row-major 3x3; C is the 9x9 tangent dP_ij/dF_kl with index 3*i+j (row) and 3*k+l (col).
 * Any output pointer may be NULL. min_eig is the projection floor (kMinProjectedEigenvalue). */
void or_smith_nh(double mu, double lambda, const double F[9], int project, int psd_strategy,
                 double min_eig, double* energy, double P[9], double C[81]);

/* Soft materials, same values as SoftMaterialType (mochi_core/.../materials/material_types.h:148-172). */
enum { OR_MAT_NEO_HOOKEAN = 0, OR_MAT_STVK = 1, OR_MAT_LINEAR = 2, OR_MAT_ARAP = 5 };

/* St. Venant-Kirchhoff: psi = mu |G|^2 + lambda/2 tr(G)^2 with G = (F^T F - I)/2; P = F S,
 * S = 2 mu G + lambda tr(G) I. Follows mochi_core/src/materials/batched_st_venant_kirchhoff.cpp:29-203:
 * Projection / AbsEigenProjection clamp the 9 tangent eigenvalues (always: no definiteness test); Fast
 * keeps only the non-negative stretches of G (no shear) inside the tangent's S. Same layout as
 * or_smith_nh. */
void or_stvk(double mu, double lambda, const double F[9], int project, int psd_strategy, double min_eig,
             double* energy, double P[9], double C[81]);

/* Linear elasticity: eps = (F + F^T)/2 - I, psi = mu eps:eps + lambda/2 tr(eps)^2,
 * P = 2 mu eps + lambda tr(eps) I, constant PSD tangent (no projection).
 * mochi_core/src/materials/batched_linear_elastic.cpp:25-97. */
void or_linear_elastic(double mu, double lambda, const double F[9], double* energy, double P[9], double C[81]);

/* As-rigid-as-possible material with stiffness mu (mochi_core/src/materials/batched_arap.cpp:29-136):
 * energy 1/2 mu |sigma - 1|^2 over the rotation-variant singular values, PK1 mu (F - U V^T), tangent with
 * the twist-mode eigenvalues clamped under projection. */
void or_arap(double mu, const double F[9], int project, int psd_strategy, double min_eig, double* energy,
             double P[9], double C[81]);

/* Dispatch on OR_MAT_* (ARAP takes mu as its stiffness). */
void or_material(int material, double mu, double lambda, const double F[9], int project, int psd_strategy,
                 double min_eig, double* energy, double P[9], double C[81]);

/* Rayleigh stiffness damping of one P1 tet (viscous stress), isotropic reference stiffness (lambda, mu):
 * dE = E(F) - E(F_stage) (Green strains, Voigt with engineering shear), S = kappa (lambda tr(dE) I +
 * 2 mu dE), energy 1/2 S : dE vol, residual (F S) dN vol, Hessian the Gauss-Newton part
 * kappa B^T C0 B plus, if geometric, the (PSD-projected when project) S term.
 * Follows mochi_core/.../element_operations/fem_stress_damping.h:29-501 (isotropic path); kappa is the
 * damping coefficient / dt. dN: 4x3 shape-function gradients; u, uss: 12 displacements. res: 12, K: 144
 * (row (f,i), column (g,j)); any output may be NULL. */
void or_stress_damping(const double dN[12], double vol, const double u[12], const double uss[12], double kappa,
                       double lambda, double mu, int geometric, int project, double* energy, double res[12],
                       double K[144]);

/* (E, nu) -> (lambda, mu). mochi_core/.../materials/material_utils.h:331-339. */
void or_lame(double E, double nu, double* lambda, double* mu);

/* PolyReLU(x; t, shift) with first and second derivative. mochi_core/.../utils/activations.h:113-130. */
void or_polyrelu(double x, double t, double shift, double* f, double* df, double* ddf);

/* Penalty contact response for one sample (frictionless, alignment mask applied by caller).
 * mochi_core/.../contact/contact_utils.h:498-570. force = k p p' grad, dforce = -k(p'^2+p p'') grad grad^T. */
void or_penalty(double d, const double grad[3], double k, double t_half, double thr,
                double* energy, double force[3], double dforce[9]);

/* Contact response parameters (ContactParams, ContactEvalConfig; mochi_core/.../contact/
 * contact_params.h:80-260, contact_utils.h:459-490). */
typedef struct {
  double k, t_half, thr, max_align;       /* penalty stiffness, smoothing half distance, threshold,
                                             maxAlignmentNormals */
  double coulomb, falloff_vel;            /* coulombFrictionCoefficient, frictionFalloffVel [m/s] */
  double viscous, normal_damping;         /* viscousFrictionCoefficient, normalViscousDampingCoefficient [s/m] */
  int collider_normal;                    /* frictionWithColliderNormal */
  int explicit_normals;                   /* explicitNormals */
  int fade;                               /* fadeFriction */
  int implicit_normal_force;              /* implicitNormalForceForDissipation */
  int fitted;                             /* fittedSaturationHessian.contactFriction */
  int model;                              /* CoulombFrictionModel: 0 C1Regularized, 1 CinfRegularized */
} or_contact_params;

/* Contact response of one sample in the collider frame: penalty plus Coulomb / viscous friction and
 * normal viscous damping, GradTarget::Current. mochi_core/.../contact/contact_utils.h:1003-1230
 * (ComputeBatchCollisionForceDForce) and 627-960 (ComputeBatchContactDissipationForceDForce).
 * d, grad: current SDF value and gradient; d_ss, grad_ss: at the stage start (read with explicit
 * normals); n_col: colliding surface normal (NULL: not valid); pos, pos_ss: current and stage-start
 * sample positions; dt: the stage's dtFactor. dforce (row-major) is d force / d pos. */
void or_collision_response(const or_contact_params* p, double d, const double grad[3], double d_ss,
                           const double grad_ss[3], const double n_col[3], const double pos[3],
                           const double pos_ss[3], double dt, int unit_grad, double* energy,
                           double force[3], double dforce[9]);

/* ---- mesh / pattern ---------------------------------------------------------------- */

/* Number of nonzero 3x3 blocks of the node-node adjacency induced by the tets (diagonal included). */
int64_t or_pattern_nnzb(int n_nodes, int n_tets, const int32_t* tets);
/* Fill a CSR block pattern with sorted column indices. row_ptr has n_nodes+1 entries. */
void or_pattern_fill(int n_nodes, int n_tets, const int32_t* tets, int64_t* row_ptr, int32_t* col);
/* Position of block (i, j) in the pattern, or -1. */
int64_t or_pattern_find(const int64_t* row_ptr, const int32_t* col, int i, int j);

/* Per-tet rest data of a P1 tet with 1-point quadrature (mochi_core/.../elements/tetrahedral/
 * finite_element.h:93-139): dN[t*12 + 3*f + c] = dN_f/dX_c, vol[t] = quadWeights[0] (signed). */
void or_rest_data(int n_tets, const int32_t* tets, const double* X, double* dN, double* vol);

/* Boundary faces (faces owned by exactly one tet), outward oriented, with rest area.
 * Returns the count; face_nodes/face_tet/face_area may be NULL for a count-only call. */
int or_boundary_faces(int n_nodes, int n_tets, const int32_t* tets, const double* X,
                      int32_t* face_nodes, int32_t* face_tet, double* face_area);

/* ---- scene description --------------------------------------------------------------- */

enum { OR_COLLIDER_PLANE = 0, OR_COLLIDER_CAPSULE = 1 };

typedef struct {
  int type;          /* OR_COLLIDER_* */
  double p[6];       /* plane: normal n[3], offset o (d = n.x - o); capsule: a[3], b[3] */
  double radius;     /* capsule radius */
  double vel[3];     /* linear velocity of the collider [m/s] */
} or_collider;

typedef struct {
  /* mesh */
  int n_nodes, n_tets, n_faces;
  const double* X;          /* 3N rest positions */
  const int32_t* tets;      /* 4T */
  const double* mu;         /* T */
  const double* lambda;     /* T */
  const double* rho;        /* T */
  const uint8_t* pin;       /* N, bit c set -> DoF c pinned */
  const int32_t* face_nodes;/* 3F */
  const int32_t* face_tet;  /* F */
  const double* face_area;  /* F */
  /* derived data (filled by or_scene_prepare) */
  const double* dN;         /* 12T */
  const double* vol;        /* T */
  const int64_t* row_ptr;   /* N+1 */
  const int32_t* col;       /* nnzb */
  int64_t nnzb;
  const double* mass;       /* nnzb scalar consistent-mass couplings m_ij */
  /* physics */
  double gravity[3];
  double dt;
  int psd_strategy;
  double min_eig;
  /* contact */
  int n_colliders;
  const or_collider* colliders;
  double k_contact, t_half, thr, max_align;
  /* material (OR_MAT_*) of every tet of the body */
  int material;
  /* Rayleigh mass damping alpha [1/s] about the stage-start displacement u_stage (3N; or_step sets it;
   * NULL: the inertia-free terms are skipped) — mochi_physics/src/mochi_soft.h:274-290, 408-420 */
  double mass_damping;
  const double* u_stage;
  /* Rayleigh stiffness damping coefficient beta [s] (stiffnessDampingCoefficient; kappa = beta / dt)
   * and its geometric term (stiffnessDampingIncludeGeometricTerm) */
  double stiffness_damping;
  int stiffness_damping_geometric;
  /* contact dissipation and evaluation settings (or_contact_params; k, t_half, thr, max_align above) */
  double coulomb, falloff_vel, viscous, normal_damping;
  int collider_normal, explicit_normals, fade, implicit_normal_force, fitted, friction_model;
} or_scene;

/* Consistent P1 mass coupling per block (Q4 quadrature, exact for P1): m_ij = sum_t rho V (1+d_ij)/20.
 * mochi_core/.../element_operations/fem_inertia.h:199-239 + mochi_physics/src/mochi_soft.cpp:883-936. */
void or_mass_blocks(const or_scene* s, double* mass);

/* Flags for or_assemble. */
enum { OR_ASM_OBJ = 1, OR_ASM_RES = 2, OR_ASM_HESS = 4, OR_ASM_PSD = 8 };

/* Assemble objective, gradient g (3N) and Hessian H (9*nnzb, block row-major) of the backward-Euler
 * incremental potential at displacement u, inertia target ut = u0 + dt*v0, colliders at time t.
 * Dirichlet rows/cols are zeroed with unit diagonal (mochi_physics/src/mochi_solve.cpp:337-396).
 * Contact statistics: number of active (sample, collider) pairs is returned. If pair_out is not
 * NULL, the active pairs are written as (sample_index * n_colliders + collider) in ascending order. */
int64_t or_assemble(const or_scene* s, const double* u, const double* ut, double t, int flags,
                    double* obj, double* g, double* H, int64_t* pair_out);

/* ---- linear solver ------------------------------------------------------------------ */

typedef struct {
  double rel_tol, abs_tol, rel_div_tol;
  int max_iter;
  int precond;        /* 0 none, 1 Jacobi, 2 block Jacobi */
  int polak_ribiere;  /* 1 -> Polak-Ribiere beta (reference default) */
  int zero_guess;     /* 1 -> x is known to be zero (InitialGuessHint::Zero) */
} or_pcg_params;

typedef struct {
  int num_iter;
  double res_norm, rel_res_norm;
  int convergence;    /* 0 none, 1 converged, 2 stopped, 3 diverged (LinearSolverConvergenceStatus) */
} or_pcg_status;

/* StopTest::CheckStatus with SetScaling(bb) (stopping_criterion.h:65-78, 92-98): the classification of a
 * squared residual norm rr: 0 active, 1 converged (relative), 2 converged (absolute), 3 diverged. A negative
 * rr within the convergence threshold is round-off and counts as 0; a more negative one diverges. */
int or_stop_status(double rr, double bb, double rel_tol, double abs_tol, double rel_div_tol);

/* Left-preconditioned CG with the residual-L2 stop test.
 * mochi_core/.../linear_algebra/krylov/pcg.h:70-238, stopping_criterion.h:31-166. */
or_pcg_status or_pcg(int n_rows_blk, const int64_t* row_ptr, const int32_t* col, const double* H,
                     const double* b, double* x, const or_pcg_params* p);

/* y = H x for a 3x3-block CSR matrix. */
void or_bsr_apply(int n_rows_blk, const int64_t* row_ptr, const int32_t* col, const double* H,
                  const double* x, double* y);

/* ---- Newton step ---------------------------------------------------------------------- */

typedef struct {
  int max_iter;            /* Newton iterations */
  double rel_tol, abs_tol; /* residual norm stop test (newton_solver.cpp:187-195) */
  double rel_step_tol;     /* |dx| <= tol*|x| stop */
  int ls_max_iter;         /* ResidualNorm line search iterations */
  double ls_alpha;         /* backtracking factor */
  int ew_forcing;          /* 0 constant linear tolerance, 2 Eisenstat-Walker choice 2 */
  double rel_div_tol, abs_div_tol;
  or_pcg_params lin;
} or_newton_params;

typedef struct {
  int newton_iters;
  int cg_iters;
  int ls_iters;
  double res_norm0, res_norm;
  int convergence;         /* 1 converged, 2 stopped, 3 diverged */
  int64_t n_contacts;      /* active pairs at the last assembly */
} or_newton_status;

/* One backward-Euler step. u, v are updated in place; t is the end-of-step time at which colliders
 * are evaluated. warm (optional, 3N) is an initial guess for each Newton linear solve (NULL -> 0).
 * Follows mochi_core/src/solvers/newton_solver.cpp:603-876 with the ResidualNorm line search
 * (mochi_core/.../solvers/line_search.h:300-336). */
or_newton_status or_step(const or_scene* s, double* u, double* v, double t,
                         const or_newton_params* p, const double* warm);

/* Default parameters matching the reference defaults used on this path. */
void or_default_newton_params(or_newton_params* p);

int or_num_threads(void);
void or_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
