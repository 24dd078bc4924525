/*
 * sdx_b200.h — C-ABI of the B200 implicit soft-body step (libsdx_b200.so).
 *
 * Plain pointers and sizes only. Every entry point returns an int status (SDX_OK == 0); the text of
 * the last error on the calling thread is available from sdx_last_error(). Handles own their device
 * buffers; a handle is not re-entrant, distinct handles are independent (one per thread is fine).
 *
 * Reference interfaces replaced (paths inside superdex_physics/libraries/mochi/):
 *   - mochi::LinearSolver<T>::Solve / CudaIterativeSolve
 *       mochi_core/include/mochi_core/solvers/linear_solver.h:265-271, 321-496, 614-662
 *     with KrylovSolverParams (mochi_core/include/mochi_core/solvers/krylov_solver.h:43-82) and
 *     LinearSolverStatus (krylov_solver.h:85-116)                       -> sdx_pcg_solve
 *   - the FEM-body assembly AssembleObjResDRes + soft::MakeBatchedBodyOp
 *       mochi_core/include/mochi_core/element_operations/element_assembler.h:230-236,
 *       mochi_physics/src/mochi_soft.h:314-420, mochi_physics/src/mochi_soft.cpp:202-318
 *     plus the async contact response mochi_physics/src/mochi_soft.cpp:386-474 -> sdx_assemble
 *   - the island Newton step solver::StepIslandNewtonAsync / NewtonSolver<T>::Solve
 *       mochi_physics/src/mochi_solve.cpp:1090, mochi_core/src/solvers/newton_solver.cpp:603-876
 *                                                                         -> sdx_step
 *   - Scene state access (displacements / velocities of soft actors)
 *       mochi_physics/src/mochi_soft.cpp:476-495 (EntityGetSolution)      -> sdx_get/set_state
 */
#ifndef SDX_B200_H
#define SDX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------------- */
#define SDX_OK 0
#define SDX_ERR_INVALID_ARGUMENT -1
#define SDX_ERR_CUDA -2
#define SDX_ERR_NOT_READY -3      /* call order: bodies must be uploaded first */
#define SDX_ERR_DEVICE_TIMEOUT -4 /* a bounded device-side wait gave up (grid barrier); the context stays
                                     usable. The environment variable SDX_DEBUG_SPIN_LIMIT, read at each
                                     solve, lowers the bound of the PCG grid barriers (tests use it to
                                     make the wait run out) */
#define SDX_ERR_OUT_OF_MEMORY -5
#define SDX_ERR_UNSUPPORTED -6

/* ---- enums (values match the reference enums where one exists) --------------------------------- */
/* PreconditionerType subset (mochi_core/.../solvers/linear_solver_params.h) */
#define SDX_PREC_NONE 0
#define SDX_PREC_JACOBI 1
#define SDX_PREC_BLOCK_JACOBI 2
/* LinearSolverConvergenceStatus (krylov_solver.h:85-116) */
#define SDX_LINEAR_NONE 0
#define SDX_LINEAR_CONVERGED 1
#define SDX_LINEAR_STOPPED 2
#define SDX_LINEAR_DIVERGED 3
/* InitialGuessHint (linear_solver.h) */
#define SDX_GUESS_UNKNOWN 0
#define SDX_GUESS_ZERO 1
/* MaterialPsdStrategy (mochi_core/.../materials/material_types.h:52) */
#define SDX_PSD_NONE 0
#define SDX_PSD_PROJECTION 1
#define SDX_PSD_ABS_EIGEN 2
#define SDX_PSD_FAST 3
/* value types of host matrices */
#define SDX_F32 0
#define SDX_F64 1
/* collider types (plane, capsule) */
#define SDX_COLLIDER_PLANE 0
#define SDX_COLLIDER_CAPSULE 1
/* assembly flags (AssemblyParams: assemObj / assemRes / assemDRes / psdDRes) */
#define SDX_ASM_OBJ 1
#define SDX_ASM_RES 2
#define SDX_ASM_HESS 4
#define SDX_ASM_PSD 8
/* warm start of each Newton linear solve */
#define SDX_WARM_ZERO 0     /* reference behaviour: dx0 = 0 (newton_solver.cpp:746) */
#define SDX_WARM_PREVIOUS 1 /* dx0 = the previous solve's dx of the same env */
#define SDX_WARM_LEARNED 2  /* dx0 = per-vertex MLP prediction (sdx_mlp_*) */
#define SDX_WARM_TEMPORAL 3 /* dx0 = the previous step's dx of the same Newton iteration (first 4) */

/* Value layouts of a host 3x3 block CSR matrix (sdx_linear_params.value_layout).
 * ROW_STRIPS is the reference's own storage, BlockSparseMatrix<T,3>::Values(): each block row br with
 * nb = row_ptr[br+1] - row_ptr[br] blocks is one row-major 3 x (3 nb) strip, so entry (lr, lc) of its
 * k-th block sits at 9 row_ptr[br] + 3 (lr nb + k) + lc (FindValueIndex,
 * mochi_core/include/mochi_core/linear_algebra/block_sparse_matrix.h:459-475). BLOCKS is 9 contiguous
 * row-major values per block, the layout cuSPARSE BSR takes and ConvertCsrToBsr produces
 * (mochi_core/src/linear_algebra/cuda/cuda_bsr_matrix.cu:22-47). */
#define SDX_BSR_ROW_STRIPS 0
#define SDX_BSR_BLOCKS 1

/* Mirrors KrylovSolverParams (krylov_solver.h:43-82). Only the residual-L2 norm is supported. */
typedef struct {
  double rel_tol;       /* ||r|| <= max(abs_tol, rel_tol ||b||) */
  double abs_tol;
  double rel_div_tol;   /* diverged when ||r|| > rel_div_tol ||b|| */
  int max_iter;
  int preconditioner;   /* SDX_PREC_* */
  int abort_if_not_spd; /* stop with DIVERGED on p.Ap <= 0 */
  int polak_ribiere;    /* 1: Polak-Ribiere beta (reference default) */
  int replace_every;    /* FP64 true-residual replacement period in iterations (0: default 32) */
  int value_layout;     /* SDX_BSR_* of the values passed to the sdx_pcg_solve* entry points
                           (default SDX_BSR_ROW_STRIPS, the reference's layout) */
  /* Mixed-precision iterative refinement (no counterpart in the reference; 0 = off): when > 0, the solve
   * runs as passes of the PCG to this relative tolerance of each pass's right-hand side. Pass 0 solves
   * A x = b from the initial guess (warm starts included); each later pass computes r = b - A x in FP64,
   * stops the env when ||r|| meets rel_tol / abs_tol, else solves A d = r from zero and adds d to x. The
   * iteration count is the sum over the passes; max_iter bounds each pass. */
  double refine_inner_rel_tol;
  int refine_max_passes;  /* passes after pass 0 (default 8); an env still above tolerance then stops */
} sdx_linear_params;

/* Coulomb friction smoothing (CoulombFrictionModel, contact_params.h:307-327) */
#define SDX_FRICTION_C1 0
#define SDX_FRICTION_CINF 1

/* Mirrors LinearSolverStatus (krylov_solver.h:85-116). */
typedef struct {
  int num_iter;
  double residual_norm;
  double relative_residual_norm;
  int convergence; /* SDX_LINEAR_* */
} sdx_linear_status;

/* Newton / physics parameters of a step (NonLinearSolverParams, nonlinear_solver_params.h:327-466;
 * ContactParams, contact_params.h:85-183). */
typedef struct {
  double dt;
  double gravity[3];
  int psd_strategy;            /* SDX_PSD_* (default projection) */
  double k_contact;            /* penaltyCoefficient [Pa/m] */
  double t_half;               /* penaltySmoothingHalfDistance [m] */
  double thr;                  /* penaltyThresholdDefault [m] */
  double max_align;            /* maxAlignmentNormals */
  int newton_max_iter;
  double newton_rel_tol, newton_abs_tol, newton_rel_step_tol;
  int ls_max_iter;
  double ls_alpha;
  int ew_forcing;              /* 0 constant linear tolerance, 2 Eisenstat-Walker choice 2 */
  double rel_div_tol, abs_div_tol;
  int warm_start;              /* SDX_WARM_* */
  sdx_linear_params linear;
  double mass_damping;         /* Rayleigh mass damping coefficient alpha [1/s] (massDampingCoefficient):
                                  adds alpha/dt * M (u - u_stage) to the residual and alpha/dt * M to the
                                  Hessian (ComputeSoftDampingScales, mochi_physics/src/mochi_soft.h:274-290) */
  double stiffness_damping;    /* Rayleigh stiffness damping coefficient beta [s] (stiffnessDampingCoefficient):
                                  viscous stress kappa C0 (E(F) - E(F_stage)), kappa = beta / dt
                                  (fem::StressDampingWork, fem_stress_damping.h:29-501) */
  int stiffness_damping_geometric; /* stiffnessDampingIncludeGeometricTerm: add the viscous-stress term to
                                      the Hessian (PSD-projected with the material's projection) */
  /* Contact dissipation (ComputeBatchContactDissipationForceDForce, contact_utils.h:627-960): Coulomb and
   * viscous friction and normal viscous damping of each contact sample, driven by the sample's
   * displacement relative to the collider over the step and by the normal force at the stage start
   * (ContactParams, contact_params.h:150-230; ContactEvalConfig, contact_utils.h:459-490). */
  double friction_coulomb;         /* coulombFrictionCoefficient (the reference's default is 0.5; 0 here) */
  double friction_falloff_vel;     /* frictionFalloffVel [m/s] (default 0.01) */
  double friction_viscous;         /* viscousFrictionCoefficient [s/m] (default 0) */
  double contact_normal_damping;   /* normalViscousDampingCoefficient [s/m] (default 0) */
  int friction_model;              /* SDX_FRICTION_* (CoulombFrictionModel, default C1) */
  int friction_fitted_hessian;     /* fittedSaturationHessian.contactFriction (default 1) */
  int friction_fade;               /* fadeFriction (default 1) */
  int friction_collider_normal;    /* frictionWithColliderNormal (default 1) */
  int contact_explicit_normals;    /* explicitNormals (default 0): alignment, friction plane and the
                                      dissipation's normal force from the stage start; pairs in contact at
                                      the stage start stay in the contact set */
  int contact_implicit_normal_force; /* implicitNormalForceForDissipation (default 0; not together with
                                        explicit normals) */
  int newton_graph;  /* no counterpart in the reference (default 0). 1: each step is one CUDA graph launch;
                        the Newton loop and the ResidualNorm line search are conditional while-nodes whose
                        conditions device kernels set from the same stop tests, so the step takes no host
                        round trip. Zero, previous or temporal warm start with the constant or Eisenstat-Walker linear
                        tolerance; the PCG runs on the grid kernel over the upload's partition (no
                        re-partitioning, no cluster kernel) and per-kernel profiling records nothing. The
                        graph is built on the first such step and rebuilt when the parameters or the bodies
                        change; the launch-shape tuners only run in host-driven steps. */
} sdx_step_params;

/* Per-env statistics of the last step (StageSolverStats, mochi_physics/src/mochi_solve.cpp:1144). */
typedef struct {
  int newton_iters;
  int cg_iters;
  int ls_iters;
  int convergence;             /* 1 converged, 2 stopped, 3 diverged */
  double res_norm0, res_norm;
  int64_t n_contacts;          /* active (sample, collider) pairs at the last assembly */
} sdx_env_stats;

typedef struct sdx_context sdx_context;

const char* sdx_last_error(void);
int sdx_version(void);
/* Fill `p` with the defaults of this path (reference defaults, Newton to rel 1e-6, CG rel 1e-6). */
void sdx_default_step_params(sdx_step_params* p);
void sdx_default_linear_params(sdx_linear_params* p);

/* ---- linear solver boundary (LinearSolver<T>::Solve with solverType CudaCG) -------------------- */

/* Solve A x = b, A symmetric positive definite in 3x3 block CSR (block_rows rows, nnzb blocks,
 * row_ptr / col as BlockSparseMatrix<T,3>::Pointers() / Indices(), widened to int64 row pointers).
 * values: 9*nnzb of SDX_F32 or SDX_F64 in params->value_layout (SDX_BSR_ROW_STRIPS: the reference's
 * BlockSparseMatrix::Values() as it is). b, x: host FP64 vectors of 3*block_rows; x is the initial guess
 * on entry (ignored when hint == SDX_GUESS_ZERO) and the solution on exit. The matrix is stored on the
 * device in FP32; dot products and x, r accumulate in FP64. */
int sdx_pcg_solve(int block_rows, int64_t nnzb, const int64_t* row_ptr, const int32_t* col,
                  const void* values, int value_type, const double* b, double* x, int hint,
                  const sdx_linear_params* params, sdx_linear_status* status);

/* Same, with an explicit context whose device workspace and launch tuning are reused. */
int sdx_pcg_solve_ctx(sdx_context* ctx, int block_rows, int64_t nnzb, const int64_t* row_ptr,
                      const int32_t* col, const void* values, int value_type, const double* b,
                      double* x, int hint, const sdx_linear_params* params,
                      sdx_linear_status* status);

/* No counterpart in the reference. A Jacobi-PCG solve for callers that cannot allocate GPU memory
 * when they need the solve — an engine whose pool allocator owns all device memory and forbids
 * cudaMalloc/cudaFree inside its step callbacks, or a real-time loop that must not take allocator
 * locks. Same algorithm, parameters and status as sdx_pcg_solve, but every pointer is a DEVICE pointer
 * owned by the caller (BSR with FP32 values in params->value_layout, FP64 b and x) and nothing is
 * allocated: the work vectors live in one fixed array inside the library, held by every GPU that loads
 * it until the process exits. Limits: at most SDX_NOALLOC_MAX_BLOCK_ROWS block rows (larger systems
 * return SDX_ERR_INVALID_ARGUMENT). A row_ptr that is not monotone, does not start at 0 or does not end
 * at nnzb, or a column index out of range, returns SDX_ERR_INVALID_ARGUMENT (checked on the device; no
 * access leaves the caller's arrays). All calls on a device share that array: calls whose GPU work
 * overlaps (unordered streams or threads) race and must be serialized by the caller. The first call on
 * a device performs a one-time set-up (it looks up the array's device address). Every call
 * synchronizes `stream` and copies the status to pageable host memory, so it cannot be made while
 * that stream (or the device) is being captured into a CUDA graph. `stream` is a cudaStream_t (NULL:
 * legacy default stream); the call returns after the solve has finished on that stream. */
#define SDX_NOALLOC_MAX_BLOCK_ROWS 65536
int sdx_pcg_solve_device_noalloc(int block_rows, int64_t nnzb, const int64_t* row_ptr, const int32_t* col,
                                 const float* values, const double* b, double* x, int hint,
                                 const sdx_linear_params* params, sdx_linear_status* status,
                                 void* stream);

/* ---- context / FEM bodies ----------------------------------------------------------------------- */

sdx_context* sdx_create(int device);
int sdx_destroy(sdx_context* ctx);

/* Upload n_envs independent soft bodies in the CSR-of-environments layout: env e owns nodes
 * [node_offsets[e], node_offsets[e+1]) and tets [tet_offsets[e], tet_offsets[e+1]); tets hold GLOBAL
 * node ids (4 per tet, positive orientation). X: 3 doubles per node. lambda, mu, rho: per tet.
 * pin: per node, bit c set pins DoF c (Dirichlet). Builds the block pattern, the 3x3 sliced-ELL
 * matrix layout, boundary faces (P1Q3 contact samples), mass couplings and per-tet scatter slots. */
int sdx_upload_bodies(sdx_context* ctx, int n_envs, const int64_t* node_offsets,
                      const int64_t* tet_offsets, const double* X, const int32_t* tets,
                      const double* lambda, const double* mu, const double* rho, const uint8_t* pin);

/* Kinematic colliders. rows: 11 doubles per collider = (type, p[6], radius, vel[3]);
 * plane p = (n[3], o) with d = n.x - o; capsule p = (a[3], b[3]). env: owning env of each collider,
 * non-decreasing. */
int sdx_set_colliders(sdx_context* ctx, int n_colliders, const int32_t* env, const double* rows);

/* Soft material of each env, values as SoftMaterialType (mochi_core/.../materials/material_types.h:
 * 148-172): the constitutive response of BatchedSmithNeoHookean (batched_smith_neo_hookean.cpp:29),
 * BatchedStVenantKirchhoff (batched_st_venant_kirchhoff.cpp:29) or BatchedLinearElastic
 * (batched_linear_elastic.cpp:27) with the body's per-tet Lame parameters. Default: all Neo-Hookean. */
#define SDX_MAT_NEO_HOOKEAN 0
#define SDX_MAT_ST_VENANT_KIRCHHOFF 1
#define SDX_MAT_LINEAR_ELASTIC 2
#define SDX_MAT_ARAP 5  /* BatchedArap (batched_arap.cpp:29), stiffness = the tet's mu; not with SDX_PSD_FAST */
int sdx_set_materials(sdx_context* ctx, int n_envs, const int32_t* material);

int sdx_set_params(sdx_context* ctx, const sdx_step_params* params);

/* State in user node order (3 doubles per node): displacement u and velocity v. */
int sdx_set_state(sdx_context* ctx, const double* u, const double* v, double time);
int sdx_get_state(sdx_context* ctx, double* u, double* v, double* time);

/* Masked state write (SceneBatchExecutorV2::WriteState, mochi_physics/pybind/src/scene_batch_executor_v2.cpp:
 * 459-540): in user node order, DoF i of u / v is written where its mask byte is nonzero (a NULL mask
 * writes every DoF; NULL values leave the vector as it is). The host buffers may be reused on return. */
int sdx_write_state_masked(sdx_context* ctx, const double* u, const double* v, const uint8_t* u_mask,
                           const uint8_t* v_mask);

/* State snapshots (Scene::CaptureState / RestoreState / ReleaseState / ReleaseAllStates / IsEqualState /
 * CaptureStateToBytes / RestoreStateFromBytes, mochi_physics/include/mochi_physics/cpp_api/mochi_scene.h:
 * 79-93; mochi_physics/src/mochi_scene.cpp:739-840). A snapshot holds everything a later step reads: the
 * displacement, velocity and clock, the warm-start vectors of the last solves and the temporal history,
 * and the per-env statistics; stepping on from a restored snapshot repeats the original steps (up to the
 * rounding order of the assembly's atomic accumulation). Handles refer to device-resident copies (no host round trip; captures are ordered on the
 * context's stream). env_mask (n_envs bytes, NULL: all) restores only the selected envs and keeps the
 * clock. A handle of another context, or one already released, is refused by sdx_restore_state;
 * releasing an unknown handle is a no-op. The bytes format is little-endian, versioned, carries a
 * fingerprint of the uploaded bodies and a checksum; out = NULL asks for the size. */
int sdx_capture_state(sdx_context* ctx, uint64_t* handle);
int sdx_restore_state(sdx_context* ctx, uint64_t handle, int release_immediately, const uint8_t* env_mask);
int sdx_release_state(sdx_context* ctx, uint64_t handle);
int sdx_release_all_states(sdx_context* ctx);
int sdx_is_equal_state(sdx_context* ctx, uint64_t a, uint64_t b, int* equal);
int sdx_capture_state_to_bytes(sdx_context* ctx, uint8_t* out, int64_t capacity, int64_t* size);
int sdx_restore_state_from_bytes(sdx_context* ctx, const uint8_t* data, int64_t size);

/* Sizes of the uploaded problem. */
int sdx_get_sizes(sdx_context* ctx, int64_t* n_nodes, int64_t* n_tets, int64_t* nnzb,
                  int64_t* n_faces);
/* Block pattern in user node order (row_ptr: n_nodes+1, col: nnzb), sorted columns. */
int sdx_get_pattern(sdx_context* ctx, int64_t* row_ptr, int32_t* col);
/* Boundary faces: 3 user node ids per face (outward), owning tet, rest area. */
int sdx_get_faces(sdx_context* ctx, int32_t* face_nodes, int32_t* face_tet, double* face_area);

/* Assemble at displacement u (host, user order; NULL = current state) with inertia target
 * ut = u_state + dt v_state and colliders at time t. Outputs (any may be NULL): obj per env (FP64),
 * gradient g (FP64, user order), Hessian values (FP32, 9 per block in sdx_get_pattern order),
 * active contact pairs per env. Dirichlet rows/cols are applied. */
int sdx_assemble(sdx_context* ctx, const double* u, double t, int flags, double* obj, double* g,
                 float* hess, int64_t* n_pairs);

/* Active contact pairs of the last assembly as sample*max_colliders_per_env + local collider, per
 * env ascending (deterministic prefix-sum compaction). pairs_cap bounds the output. */
int sdx_get_contact_pairs(sdx_context* ctx, int64_t* pairs, int64_t pairs_cap, int64_t* n_pairs);

/* Advance every env n_steps backward-Euler steps from the current state (device resident). */
int sdx_step(sdx_context* ctx, int n_steps);
int sdx_get_stats(sdx_context* ctx, sdx_env_stats* per_env);

/* ---- external linear solver (no counterpart in the reference's soft-body path) -----------------
 * sdx_step solves each Newton system with this library's PCG. A caller may hand those solves to its own
 * solver instead, e.g. a restatement of the reference's CUDA path (krylov::CudaPCG, cuSPARSE bsrmv and
 * cuBLAS, mochi_core/src/linear_algebra/cuda/cuda_pcg.cpp:243-525) run as a comparison arm. The hook
 * gets every env's Newton system on the device in user node order: the sdx_get_pattern block pattern
 * with FP32 values in SDX_BSR_BLOCKS layout (Dirichlet rows and columns applied), b = the Newton
 * gradient and x = the update (initial guess in, solution out), both FP64. It solves the envs with
 * env_mask[e] != 0, writes their CG iteration counts to iters[e] and returns SDX_OK; any other value
 * stops the step with that status. */
typedef struct {
  int n_envs;
  const int64_t* node_offsets; /* host, n_envs + 1: env e owns nodes [node_offsets[e], node_offsets[e+1]) */
  const uint8_t* env_mask;     /* host, n_envs */
  int64_t n_nodes, nnzb;
  const int64_t* row_ptr;      /* device, n_nodes + 1 (global node ids, columns stay inside the env) */
  const int32_t* col;          /* device, nnzb */
  const float* values;         /* device, 9 * nnzb */
  const double* b;             /* device, 3 * n_nodes */
  double* x;                   /* device, 3 * n_nodes */
  int zero_guess;              /* 1: x holds no initial guess (start from zero) */
  void* stream;                /* cudaStream_t the hook must order its work on */
} sdx_device_system;
typedef int (*sdx_linear_solve_fn)(void* user, const sdx_device_system* sys, const sdx_linear_params* params,
                                   int* iters);
/* fn = NULL restores this library's PCG. */
int sdx_set_linear_solver(sdx_context* ctx, sdx_linear_solve_fn fn, void* user);

/* ---- learned CG warm start (no counterpart in the reference) -------------------------------------
 * A per-vertex MLP (15 -> 128 -> 128 -> 128 -> 3, GELU; BF16 weights / activations, FP32 accumulate;
 * forward on the tensor cores) maps 1-ring-averaged displacement, dt * velocity, the last Newton
 * update, the previous step's update at the same Newton iteration and the Jacobi-preconditioned Newton
 * gradient (each group divided by the env's RMS of it)
 * to the Newton update in the same units. With warm_start = SDX_WARM_LEARNED its prediction is the
 * initial guess of every Newton linear solve; the converged residual still decides the solution. */
#define SDX_MLP_PARAMS 37264
int sdx_mlp_init(sdx_context* ctx, uint64_t seed);
int sdx_mlp_set_params(sdx_context* ctx, const float* params, int n);
int sdx_mlp_get_params(sdx_context* ctx, float* params, int n);
/* Y (n x 3) = MLP(X (n x 16, column 15 ignored)); host arrays. */
int sdx_mlp_forward(sdx_context* ctx, const float* X, int n, float* Y);
/* Gradient of the mean-squared error against targets T (n x 3) w.r.t. all parameters, and the loss. */
int sdx_mlp_gradients(sdx_context* ctx, const float* X, const float* T, int n, float* grad, double* loss);
/* Adam (lr) over `epochs` shuffled passes of minibatches of `batch` samples; epoch_loss[epochs]. */
int sdx_mlp_train(sdx_context* ctx, const float* X, const float* T, int64_t n, int batch, int epochs, float lr,
                  uint64_t seed, double* epoch_loss);
/* While stepping, record (features, normalized solution) of samples_per_solve random nodes of every
 * Newton linear solve, up to `capacity` samples (0 disables). */
int sdx_collect_training(sdx_context* ctx, int samples_per_solve, int64_t capacity, uint64_t seed);
int sdx_get_training_data(sdx_context* ctx, float* X, float* T, int64_t cap, int64_t* n);

/* Kernel-level entry points used by the benchmark: y = A x on the context's last assembled matrix
 * (device resident, FP32), repeated `reps` times; returns the average time per SpMV in ms. */
int sdx_bench_spmv(sdx_context* ctx, int reps, double* ms_per_spmv, double* bytes_per_spmv);
/* Count of kernel launches issued by this context since creation (for launch accounting). */
int64_t sdx_kernel_launches(sdx_context* ctx);

/* The CUDA stream (cudaStream_t) all work of this context is issued on, for event timing by callers. */
int sdx_get_stream(sdx_context* ctx, void** stream);

/* Opt-in per-kernel device timing (CUDA events on the context stream around each launch). */
typedef struct {
  double pcg_ms;            /* persistent PCG launches */
  int64_t pcg_launches;
  int64_t pcg_iters;        /* sum over launches of the largest iteration count of the batch */
  double asm_hess_ms;       /* element kernel launches that assemble the Hessian */
  int64_t asm_hess_launches;
  double asm_res_ms;        /* element kernel launches that assemble the residual only */
  int64_t asm_res_launches;
  double contact_ms;
  int64_t contact_launches;
  double seed_ms;           /* Hessian seeding with the scaled mass matrix */
  int64_t seed_launches;
  double pcg_bytes;         /* algorithmic HBM bytes of the PCG launches: per env, its CG iterations x
                               (40 B per block + 4 B per row pointer + 228 B per row, 156 B per row when
                               z carries r and an FP32 increment carries x between true-residual
                               replacements) */
  int64_t pcg_relaunches;   /* re-partitioned PCG relaunches (batches whose slow envs got all CTAs) */
  int64_t pcg_threads;      /* threads per CTA of the PCG launch shape in use (autotuned or default) */
  double warm_ms;           /* learned warm start: features, MLP inference and the start-vector kernel */
  int64_t warm_launches;
  int64_t pcg_cluster_solves; /* PCG solves that ran on the cluster kernel (a batch of small envs, one
                                 thread-block cluster per env at a time) instead of the grid kernel */
  int64_t pcg_cluster_size;   /* cluster size the autotuner picked for this batch (0: chosen by occupancy;
                                 -1: the grid kernel won, long queues stay on it) */
  double tune_grid_us;        /* autotuner: best grid-kernel time of its 24-iteration solve (0: not tuned) */
  double tune_cluster_us;     /* autotuner: best cluster-kernel time of the same solve (0: none timed) */
  int64_t elem_threads;       /* element kernel CTA size of Hessian assemblies (autotuned or 128) */
  int64_t elem_res_threads;   /* element kernel CTA size of residual-only assemblies */
  int64_t elem_aggregated;    /* 1: Hessian blocks are warp-aggregated before their reductions */
  int64_t contact_threads;    /* contact kernel CTA size */
  double tune_elem_us;        /* assembly tuner: fastest Hessian element launch (0: not tuned) */
  double tune_elem_default_us;/* the same launch with the default shape (128 threads, plain scatter) */
  double pcg_cluster_ms;      /* the share of pcg_ms spent in cluster-kernel solves */
  double pcg_cluster_bytes;   /* the share of pcg_bytes of those solves */
} sdx_profile;
/* enable: 0 off, 1 per-kernel event timing, 2 also the per-CTA PCG phase timers (sdx_get_pcg_cta_profile) */
int sdx_set_profiling(sdx_context* ctx, int enable);
int sdx_get_profile(sdx_context* ctx, sdx_profile* out);

/* Launch shape the cluster PCG uses on the current device for a queue of n_envs envs: how many
   thread-block clusters of how many CTAs (one 512-thread CTA per SM). No reference counterpart (the
   reference solves one env at a time). SDX_ERR_UNSUPPORTED when no cluster shape fits; batches then stay
   on the grid kernel. */
int sdx_pcg_cluster_shape(int n_envs, int* n_clusters, int* cluster_size);
/* Per-CTA phase times of the persistent PCG (no reference counterpart), recorded while profiling at level 2
 * (sdx_set_profiling(ctx, 2)): 4 values per CTA, SM clock cycles summed since then: SpMV phase, wait at the
 * barrier after it, update phase, wait at the barrier after it. */
int sdx_get_pcg_cta_profile(sdx_context* ctx, int n_cta, double* out);

#ifdef __cplusplus
}
#endif
#endif
