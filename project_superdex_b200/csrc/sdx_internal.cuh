// sdx_internal.cuh — kernel argument blocks and launch wrappers shared by the host runtime and the
// kernels of libsdx_b200.so.
//
// HBM layout (all envs of a batch live in one set of arrays, CSR-of-environments):
//   * rows: each env's nodes occupy a contiguous range of "rows" padded to a multiple of 32, so a
//     32-row slice belongs to exactly one env. Vectors are indexed by row (3 components per row).
//   * matrix: 3x3 sliced-ELL ("SELL-32 of 3x3 blocks"). Slice s covers rows [32s, 32s+32) and has
//     width w_s = the longest block row in it. Block position p = slice_ptr[s] + 32k + lane holds the
//     k-th block of row 32s+lane; its column is col[p] (padding: row | 0x80000000). The 9 values of
//     the 32 blocks of one (slice, k) group occupy 1152 contiguous bytes starting at G = (p - lane) * 9
//     floats, split 4 + 4 + 1: entries e = 0..3 of lane l at G + 4l + e, entries 4..7 at
//     G + 128 + 4l + (e - 4), entry 8 at G + 256 + l (e = 3r + c). A warp loads a group with two
//     fully coalesced 128-bit loads and one 32-bit load per lane.
//   * per tet: int4 rows, 4 float4 rest records (dN 12, vol, mu, lambda, rho) stored as 4 separate
//     float4 arrays (coalesced), 4 int4 records of the 16 block positions its 4x4 blocks scatter to.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sdx {

constexpr int kSlice = 32;
constexpr int kPadBit = 0x80000000;
constexpr int kPcgMaxEnvsPerCta = 32;
// cluster PCG: the largest env it takes (rows); the queue length, in envs per co-resident cluster, from
// which it runs a whole batch; the envs (at most kClusterTailEnvs, each at most kClusterLatencyRows rows)
// it takes at the end of a batch's Newton iterations. Per CG iteration on two-env batches the cluster
// kernel measured 9.0 us against the grid kernel's 11.9 us at 2,197 rows per env, but 15.3 against 12.2
// at 9,261 and 24.7 against 13.9 at 24,389 (the grid kernel spreads a small env over every SM), so the
// tail rule is kept to tiny envs.
constexpr int64_t kClusterMaxRows = 131072;
constexpr int kClusterQueueFactor = 4;
constexpr int kClusterTailEnvs = 4;
constexpr int64_t kClusterLatencyRows = 4096;
constexpr int kPcgNq = 11;  // partial sums per (CTA, env) and phase (11: the two-vector start)

__host__ __device__ __forceinline__ size_t val_index(int64_t p, int e) {
  const size_t g = (size_t)(p - (p & 31)) * 9;
  const size_t l = (size_t)(p & 31);
  return e < 4 ? g + 4 * l + e : (e < 8 ? g + 128 + 4 * l + (e - 4) : g + 256 + l);
}

struct Matrix {
  int n_slices;
  const int* slice_ptr;  // n_slices + 1, in block positions
  const int* slice_w;
  const int* slice_env;
  const int* col;
  float* val;
};

// largest CTA size of the element kernel (the shape tuner picks 64, 128 or 256)
constexpr int kElemMaxThreads = 256;

struct ElemArgs {
  int64_t n_tets;
  const int4* tets;
  const float4* rest0;
  const float4* rest1;
  const float4* rest2;
  const float4* rest3;
  const int4* slots0;
  const int4* slots1;
  const int4* slots2;
  const int4* slots3;
  const int* slice_env;
  const uint8_t* env_mask;      // NULL = all
  const uint8_t* env_material;  // per env: 0 Smith Neo-Hookean, 1 St. Venant-Kirchhoff, 2 linear (NULL: 0)
  const double* u;
  const double* ut;
  const double* u0;  // stage-start displacement (mass damping)
  const double* X;
  const uint8_t* pin;
  double* g;
  float* val;
  double* obj;  // per env
  double dtfi2;
  double mdamp;  // mass damping scale alpha / dt (0: none)
  double kdamp;  // stiffness damping factor kappa = beta / dt (0: none)
  int kdamp_geo; // include the geometric (stress) term of the stiffness damping Hessian
  double grav[3];
  float min_eig;
  int psd;
  int flags;
  int has_arap;  // some env uses ARAP (launch the variant that evaluates it)
  int threads;   // CTA size: 64, 128 or 256 (anything else: 128)
  int aggregate; // Hessian launches: warp-aggregated block scatter
};

struct ContactArgs {
  int64_t n_samples;
  const int4* faces;  // 3 rows + env
  const double* face_area;
  const int* face_slots;  // 9 per face
  const double* colliders;  // 11 per collider
  const int* coll_off;      // per env
  const uint8_t* env_mask;
  const double* u;
  const double* X;
  const uint8_t* pin;
  double* g;
  float* val;
  double* obj;
  unsigned* pair_mask;      // per sample (NULL: not recorded)
  unsigned long long* n_pairs;  // per env
  double t, k, t_half, thr, max_align;
  int flags;
  // contact dissipation and evaluation settings (ContactParams, ContactEvalConfig)
  const double* u0;   // stage-start displacement (time t0); read when dissipative or explicit normals
  double t0;          // stage-start time
  double coulomb;     // coulombFrictionCoefficient
  double falloff;     // frictionFalloffVel * dt: the smoothing width in displacement
  double viscous, normal_damping;  // viscousFrictionCoefficient / dt, normalViscousDampingCoefficient / dt
  int cflags;         // kContact* bits
  int threads;        // CTA size: 64, 128 or 256 (anything else: 128)
  const double* t_dev;  // evaluation time in device memory (NULL: t); the stage start is then t_dev - (t - t0)
};

// ContactArgs::cflags
constexpr int kContactColliderNormal = 1;  // frictionWithColliderNormal
constexpr int kContactExplicit = 2;        // explicitNormals
constexpr int kContactFade = 4;            // fadeFriction
constexpr int kContactImplicitFn = 8;      // implicitNormalForceForDissipation
constexpr int kContactFitted = 16;         // fittedSaturationHessian.contactFriction
constexpr int kContactCinf = 32;           // CoulombFrictionModel::CinfRegularized

// CG scalars of one env carried across a re-partitioning relaunch
struct EnvSave {
  double rz, beta, bb, conv_thr, div_thr, rr;
  int first, status;
};

struct PcgArgs {
  Matrix A;
  int n_envs;
  int precond;  // 0 none, 1 Jacobi, 2 block Jacobi
  const int* diag_pos;
  const double* b;
  double* x;
  const double* x2;  // second start vector (learned correction): Galerkin start on span{x, x2} (NULL: none)
  double* gal;       // 3 per row: A x2 kept by the Galerkin start (needed with x2)
  double* r;
  float* p;
  float* q;
  float4* z;
  float* dinv;  // 3 per row (Jacobi) or 9 per row (block Jacobi)
  const int* cta_slice;   // CTA c covers entries [cta_slice[c], cta_slice[c+1]) of the slice list
  const int* slice_list;  // ascending slice ids (NULL: entry i is slice i)
  const int* cta_eoff;    // CTA c's envs: cta_envs[cta_eoff[c] .. cta_eoff[c+1]), ascending
  const int* cta_envs;
  const int* env_cta0;
  const int* env_cta1;
  const int* env_poff;  // partials of env e live at [env_poff[e], env_poff[e] + env_cta1[e] - env_cta0[e]]
  double* part;
  const uint8_t* env_mask;
  const double* env_rel_tol;  // per-env relative tolerance (NULL: rel_tol)
  double rel_tol, abs_tol, rel_div_tol;
  int max_iter;
  int polak_ribiere;
  int replace_every;
  int zero_guess;
  const int* zero_guess_dev;  // zero_guess read from device memory at launch start (NULL: zero_guess)
  int scale_guess;  // non-zero guess: replace x0 by alpha x0, alpha = (x0.b)/(x0.A x0) (energy-optimal)
  int abort_spd;
  int* out_iters;
  double* out_res;
  double* out_relres;
  int* out_conv;
  unsigned* sync;  // [0] barrier arrivals (monotonic), [1] unused, [2] error, [3] active envs,
                   // [4] verify_iter, [5] active rows, [6] resume iteration, [7] repartition exit
  long long spin_limit;
  int r_in_z;    // Jacobi / no preconditioner: r is carried by z between true-residual replacements
                 // (r = z / d, FP32 precision) and x by its FP64 value at the last replacement plus the FP32
                 // increment xi, so the update phase reads and writes no FP64 vector
  float* xi;     // FP32 increment of x since the last true-residual replacement (r_in_z)
  int stage_update;  // cluster PCG, Jacobi, z carrying r: the update phase's operands of a warp's next
                     // stage_update (2..4; 0: off) slices are brought into shared memory by bulk asynchronous
                     // copies (one mbarrier per buffer)
  int prefetch;  // bulk L2 prefetch of each warp's next slices (0: none): the update phase's distance in
                 // slices (the matrix of the next slice in the SpMV phase whenever it is set); set when the
                 // CG vectors cannot stay in L2, so every operand comes from HBM
  // Re-partitioning: once the rows of the envs still iterating fall to repart_rows (0: never), the
  // kernel saves every env's CG scalars in es[] and exits after the iteration; the host re-partitions
  // the remaining envs over all CTAs and relaunches with resume = 1 from iteration it0.
  const int* env_nrows;  // rows per env (counted off sync[5] as envs finish)
  long long repart_rows;
  int resume;
  int it0;
  EnvSave* es;
  // per-CTA phase timing (NULL: off), SM clock cycles accumulated over the launch's iterations:
  // [4 c + 0] SpMV phase, [4 c + 1] wait at the barrier after it, [4 c + 2] update phase, [4 c + 3] wait
  unsigned long long* cta_ns;
  // slots per warp in the shared partial sums: the most envs any CTA of the partition covers (0: the
  // maximum, kPcgMaxEnvsPerCta). A single-env partition keeps 1 slot, so the CTA's shared memory stays
  // small and the L1 share of the SM's unified memory, which the SpMV's z gathers use, stays large.
  int wstride;
  // cluster PCG (k_pcg_cluster): the envs to solve, largest first (taken in order through sync[1]), and
  // each env's slice range [env_soff[e], env_soff[e + 1])
  const int* cl_envs;
  int cl_n;
  const int* env_soff;
  int cl_skip_masked;  // the queue holds every env: skip those whose env_mask byte is 0
};

// Device-resident Newton state of a step run as one CUDA graph (the Newton loop and the line search as
// conditional while-nodes): per env the stop-test state of NewtonSolver<T>::Solve, the masks the kernels
// read, and the control words the decision kernels write.
struct NewtonDev {
  int n_envs;
  int* status;      // 0 iterating, 1 converged, 2 stopped, 3 diverged
  int* iters;       // Newton iterations
  int* cg;          // CG iterations summed over the step
  int* lsi;         // line-search evaluations
  double* res0;     // residual norm at the first iteration
  double* res;      // current residual norm
  double* res_prev; // at the previous iteration (Eisenstat-Walker)
  double* dxn;      // ||dx|| of the last update
  double* eta;      // per-env linear tolerance (Eisenstat-Walker), read by the PCG
  uint8_t* mask;    // envs of the current Newton pass (the kernels' env mask)
  uint8_t* lsmask;  // envs still in the line search
  double* scale;    // line-search step per env
  double* nrm;      // per-env sums of squares written by k_env_dot
  double* unorm;    // per-env ||u||^2
  int* ctl;         // [0] envs in the pass, [1] line-search envs left, [2] Newton pass, [3] line-search trial,
                    // [4] zero-start flag of the PCG, [5] error bits (1: PCG barrier timed out), [6] first control,
                    // [7] line-search trials of the step
  int* hist_valid;  // per Newton pass: the temporal history holds that pass's update
  int* pcg_iters;         // CG iterations of the last solve, per env
  unsigned* pcg_sync;     // the PCG's control words (reset before each solve; [2] its error word)
  int* pcg_conv;
  const int* env_nrows;   // rows per env
  // PCG kernel choice per pass (a switch node): branch b is taken for the first b whose threshold the envs of
  // the pass reach (min_envs[b] > 0), else the last branch (the grid kernel); 0 when there is no choice
  int n_branch;
  int min_envs[4];
};

// Newton stop-test constants (NonLinearSolverParams)
struct NewtonConsts {
  double abs_tol, rel_tol, rel_step_tol, rel_div_tol, abs_div_tol, lin_rel_tol, ls_alpha;
  int max_iter, ls_max_iter, ew_forcing;
};

cudaError_t launch_pcg_captured(const PcgArgs& a, int n_cta, int threads, cudaStream_t st);
void launch_nt_begin(const NewtonDev& d, const NewtonConsts& k, cudaStream_t st);
void launch_nt_control(const NewtonDev& d, const NewtonConsts& k, cudaGraphConditionalHandle loop,
                       cudaStream_t st);
void launch_nt_pcg_prepare(const NewtonDev& d, cudaGraphConditionalHandle pick, cudaStream_t st);
void launch_nt_temporal(const NewtonDev& d, int n_slices, const int* slice_env, int hist_len, const double* hist,
                        double* dx, cudaStream_t st);
void launch_nt_keep_hist(const NewtonDev& d, int n_slices, const int* slice_env, int hist_len, const double* dx,
                         double* hist, cudaStream_t st);
void launch_nt_after_solve(const NewtonDev& d, int ls_max_iter, cudaGraphConditionalHandle ls, cudaStream_t st);
void launch_nt_ls_scale(const NewtonDev& d, double alpha, cudaStream_t st);
void launch_nt_ls_check(const NewtonDev& d, int ls_max_iter, cudaGraphConditionalHandle ls, cudaStream_t st);

struct ClusterShape {
  int n_clusters, size;
  int last_error;  // cudaError_t of the last failed occupancy query (0: none)
};


// kernels launched by the host runtime (sdx_kernels.cu)
void launch_mass_accum(int64_t n_tets, const int4* slots[4], const float4* rest3, float* mass,
                       cudaStream_t st);
void launch_seed_hessian(const Matrix& A, const float* mass, const uint8_t* pin, const uint8_t* env_mask,
                         float mass_scale, cudaStream_t st);
void launch_element(const ElemArgs& a, cudaStream_t st);
void launch_contact(const ContactArgs& a, cudaStream_t st);
void launch_env_dot(int n_slices, const int* slice_env, const uint8_t* env_mask, const double* a,
                    const double* b, double* out, cudaStream_t st);
void launch_zero_rows(int n_slices, const int* slice_env, const uint8_t* env_mask, double* v,
                      cudaStream_t st);
void launch_pred(int64_t n3, const double* u, const double* v, double dt, double* ut, double* u0,
                 cudaStream_t st);
void launch_ls_candidate(int n_slices, const int* slice_env, const uint8_t* env_mask,
                         const double* ubase, const double* dx, const double* scale, double* u,
                         cudaStream_t st);
void launch_residual64(const Matrix& A, const uint8_t* env_mask, const double* x, const double* b, double* r,
                       cudaStream_t st);
void launch_add_rows(int n_slices, const int* slice_env, const uint8_t* env_mask, const double* d, double* x,
                     cudaStream_t st);
void launch_copy_rows(int n_slices, const int* slice_env, const uint8_t* env_mask, const double* src,
                      double* dst, cudaStream_t st);
void launch_velocity(int64_t n3, const double* u, const double* u0, double dt, double* v,
                     cudaStream_t st);
cudaError_t launch_pcg(const PcgArgs& a, int n_cta, int threads, cudaStream_t st);
// want_size > 0 asks for that cluster size (when it fits); SDX_PCG_CLUSTER_SIZE overrides both
ClusterShape pcg_cluster_shape(int n_envs, int want_size = 0);
cudaError_t launch_pcg_cluster(const PcgArgs& a, ClusterShape shape, cudaStream_t st);
void launch_spmv(const Matrix& A, const float4* x, float* y, int threads, cudaStream_t st);
void launch_bsr_to_sell(int n_rows, const int64_t* row_ptr, const int32_t* bcol, const float* bval, bool strips,
                        const int* slice_ptr, int* col, float* val, int* diag_pos, cudaStream_t st);
void launch_pack_z(int64_t n_rows, const double* x, float4* z, cudaStream_t st);
int pcg_shared_bytes(int threads, int wstride = kPcgMaxEnvsPerCta);
int pcg_max_ctas_per_sm(int threads);

}  // namespace sdx
