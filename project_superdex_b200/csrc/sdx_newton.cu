// sdx_newton.cu — the decision kernels of a backward-Euler step captured as one CUDA graph.
//
// The host-driven step (step_once in sdx_host.cu) reads per-env norms back after every Newton pass and
// line-search trial to take the stop tests of NewtonSolver<T>::Solve (newton_solver.cpp:303-313, 452-468,
// 841-874) and the ResidualNorm line search (line_search.h:300-336). Here the same decisions run on the
// device, in single-CTA kernels over the envs, so that the whole step is one graph launch: the Newton loop
// and the line search are conditional while-nodes whose conditions these kernels set
// (cudaGraphSetConditional), and every other kernel reads the masks and step lengths they write.
#include "sdx_internal.cuh"

namespace sdx {

constexpr int kNtThreads = 1024;

// number of threads of the CTA with flag set, returned to every thread
__device__ __forceinline__ int block_count(bool flag) {
  __shared__ int s_count;
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(&s_count, __popc(m));
  __syncthreads();
  const int n = s_count;
  __syncthreads();
  return n;
}

__global__ void __launch_bounds__(kNtThreads) k_nt_begin(NewtonDev d, double lin_rel_tol) {
  for (int e = threadIdx.x; e < d.n_envs; e += blockDim.x) {
    d.status[e] = 0;
    d.iters[e] = 0;
    d.cg[e] = 0;
    d.lsi[e] = 0;
    d.res0[e] = d.res[e] = d.res_prev[e] = d.dxn[e] = 0.0;
    d.eta[e] = lin_rel_tol;
    d.mask[e] = 1;  // the first assembly covers every env
    d.lsmask[e] = 0;
  }
  if (threadIdx.x == 0) {
    d.ctl[0] = d.n_envs;
    d.ctl[1] = 0;
    d.ctl[2] = 0;
    d.ctl[3] = 0;
    d.ctl[4] = 1;
    d.ctl[5] = 0;
    d.ctl[6] = 1;
    d.ctl[7] = 0;
  }
}

// Stop tests at the top of a Newton pass, in the reference's order; on every pass after the first, the
// explosion control of the pass before (on the envs it iterated) comes first. Sets the pass mask, the
// Eisenstat-Walker tolerances and the loop condition (some env iterates).
__global__ void __launch_bounds__(kNtThreads) k_nt_control(NewtonDev d, NewtonConsts k,
                                                           cudaGraphConditionalHandle loop) {
  const bool first = d.ctl[6] != 0;
  const int E = d.n_envs;
  bool any = false;
  for (int e0 = 0; e0 < E; e0 += blockDim.x) {
    const int e = e0 + threadIdx.x;
    bool active = false;
    if (e < E) {
      if (first) {
        d.res[e] = sqrt(fmax(d.nrm[e], 0.0));
      } else if (d.mask[e]) {
        const double r = d.res[e];
        if (r > k.rel_div_tol * d.res0[e] || r > k.abs_div_tol || !isfinite(r)) d.status[e] = 3;
      }
      d.mask[e] = 0;
      if (d.status[e] == 0) {
        const int it = d.iters[e];
        const double r = d.res[e];
        if (it == 0) d.res0[e] = r;
        if (r <= k.abs_tol || (it > 0 && r <= k.rel_tol * d.res0[e])) {
          d.status[e] = 1;
        } else if (it >= k.max_iter) {
          d.status[e] = 2;
        } else if (it > 0 && d.dxn[e] <= k.rel_step_tol * sqrt(fmax(d.unorm[e], 0.0))) {
          d.status[e] = 2;
        } else {
          if (k.ew_forcing == 2) {  // Eisenstat-Walker choice 2
            const double kMax = 0.01, kSafe = 0.01, kMin = 100.0 * 2.220446049250313e-16;
            double eta;
            if (it == 0) {
              eta = kMax;
            } else {
              const double al = 0.5 + 0.5 * sqrt(5.0), gam = 0.9;
              const double safe = gam * pow(d.eta[e], al);
              double v = gam * pow(r / d.res_prev[e], al);
              if (safe > kSafe) v = fmax(v, safe);
              eta = fmin(fmax(v, kMin), kMax);
            }
            d.eta[e] = eta;
          }
          d.res_prev[e] = r;
          d.iters[e] = it + 1;
          d.mask[e] = 1;
          active = true;
        }
      }
    }
    const int n = block_count(active);
    if (threadIdx.x == 0) d.ctl[0] = (e0 == 0 ? 0 : d.ctl[0]) + n;
    any = any || n > 0;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    d.ctl[6] = 0;
    // passes are bounded by the Newton iteration cap: every env in a pass has its count raised
    cudaGraphSetConditional(loop, any ? 1u : 0u);
  }
}

// The PCG's control words and outputs before a solve of the pass's envs (what run_pcg writes from the host),
// and the PCG kernel for the pass (the host loop's routing: the cluster kernel while the queue keeps its
// clusters busy, the grid kernel for short queues).
__global__ void __launch_bounds__(kNtThreads) k_nt_pcg_prepare(NewtonDev d, cudaGraphConditionalHandle pick) {
  __shared__ unsigned long long s_rows;
  if (threadIdx.x == 0) s_rows = 0ull;
  __syncthreads();
  unsigned long long rows = 0ull;
  for (int e = threadIdx.x; e < d.n_envs; e += blockDim.x) {
    if (d.mask[e]) rows += (unsigned long long)d.env_nrows[e];
    d.pcg_iters[e] = 0;
    d.pcg_conv[e] = 0;
  }
  atomicAdd(&s_rows, rows);
  __syncthreads();
  if (threadIdx.x == 0) {
    d.pcg_sync[0] = 0u;
    d.pcg_sync[1] = 0u;
    d.pcg_sync[2] = 0u;
    d.pcg_sync[3] = (unsigned)d.ctl[0];
    d.pcg_sync[4] = 0u;
    d.pcg_sync[5] = (unsigned)s_rows;
    d.pcg_sync[6] = 0u;
    d.pcg_sync[7] = 0u;
    if (d.n_branch > 0) {
      int b = d.n_branch - 1;
      for (int k = d.n_branch - 2; k >= 0; --k)
        if (d.min_envs[k] > 0 && d.ctl[0] >= d.min_envs[k]) b = k;
      cudaGraphSetConditional(pick, (unsigned)b);
    }
  }
}

// Temporal start: this pass's update of the previous step into dx for the pass's envs, when it exists;
// the PCG's zero-start flag otherwise.
__global__ void k_nt_temporal(NewtonDev d, int n_slices, const int* __restrict__ slice_env, int hist_len,
                              const double* __restrict__ hist, double* dx) {
  const int pass = d.ctl[2];
  const bool valid = pass < hist_len && d.hist_valid[pass] != 0;
  const int64_t n3 = (int64_t)n_slices * kSlice * 3;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) d.ctl[4] = valid ? 0 : 1;
  if (!valid || i >= n3 || !d.mask[slice_env[i / (kSlice * 3)]]) return;
  dx[i] = hist[(int64_t)pass * n3 + i];
}

__global__ void k_nt_keep_hist(NewtonDev d, int n_slices, const int* __restrict__ slice_env, int hist_len,
                               const double* __restrict__ dx, double* hist) {
  const int pass = d.ctl[2];
  if (pass >= hist_len) return;
  const int64_t n3 = (int64_t)n_slices * kSlice * 3;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) d.hist_valid[pass] = 1;
  if (i >= n3 || !d.mask[slice_env[i / (kSlice * 3)]]) return;
  hist[(int64_t)pass * n3 + i] = dx[i];
}

// After the pass's solve: CG counts, ||dx|| (from the norms just reduced), the line-search start (every env
// of the pass at step 1), the next pass number, the PCG's error word, and the line-search loop condition.
__global__ void __launch_bounds__(kNtThreads) k_nt_after_solve(NewtonDev d, int ls_max_iter,
                                                                cudaGraphConditionalHandle ls) {
  for (int e = threadIdx.x; e < d.n_envs; e += blockDim.x) {
    const bool in = d.mask[e] != 0;
    if (in) {
      d.cg[e] += d.pcg_iters[e];
      d.dxn[e] = sqrt(fmax(d.nrm[e], 0.0));
      d.scale[e] = 1.0;
    }
    d.lsmask[e] = in ? 1 : 0;
  }
  if (threadIdx.x == 0) {
    if (d.pcg_sync[2] != 0u) d.ctl[5] |= 1;
    d.ctl[1] = d.ctl[0];
    d.ctl[2] += 1;
    d.ctl[3] = 0;
    cudaGraphSetConditional(ls, (d.ctl[0] > 0 && ls_max_iter > 0) ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(kNtThreads) k_nt_ls_scale(NewtonDev d, double alpha) {
  if (d.ctl[3] == 0) return;
  for (int e = threadIdx.x; e < d.n_envs; e += blockDim.x)
    if (d.lsmask[e]) d.scale[e] *= alpha;
}

// One line-search trial's verdict per env: accept when the residual norm did not grow; the last trial keeps
// its evaluated norm (explosion control then judges it). Continues while envs are left and trials remain.
__global__ void __launch_bounds__(kNtThreads) k_nt_ls_check(NewtonDev d, int ls_max_iter,
                                                            cudaGraphConditionalHandle ls) {
  const int it = d.ctl[3];
  int left_total = 0;
  for (int e0 = 0; e0 < d.n_envs; e0 += blockDim.x) {
    const int e = e0 + threadIdx.x;
    bool left = false;
    if (e < d.n_envs && d.lsmask[e]) {
      d.lsi[e]++;
      const double rn = sqrt(fmax(d.nrm[e], 0.0));
      const double r = d.res[e];
      if (rn <= r) {
        d.lsmask[e] = 0;
      } else {
        left = true;
      }
      d.res[e] = (rn <= r) ? rn : r;
      if (it == ls_max_iter - 1 && left) d.res[e] = rn;
    }
    left_total += block_count(left);
  }
  if (threadIdx.x == 0) {
    d.ctl[1] = left_total;
    d.ctl[3] = it + 1;
    d.ctl[7] += 1;
    cudaGraphSetConditional(ls, (left_total > 0 && it + 1 < ls_max_iter) ? 1u : 0u);
  }
}

void launch_nt_begin(const NewtonDev& d, const NewtonConsts& k, cudaStream_t st) {
  k_nt_begin<<<1, kNtThreads, 0, st>>>(d, k.lin_rel_tol);
}

void launch_nt_control(const NewtonDev& d, const NewtonConsts& k, cudaGraphConditionalHandle loop,
                       cudaStream_t st) {
  k_nt_control<<<1, kNtThreads, 0, st>>>(d, k, loop);
}

void launch_nt_pcg_prepare(const NewtonDev& d, cudaGraphConditionalHandle pick, cudaStream_t st) {
  k_nt_pcg_prepare<<<1, kNtThreads, 0, st>>>(d, pick);
}

void launch_nt_temporal(const NewtonDev& d, int n_slices, const int* slice_env, int hist_len, const double* hist,
                        double* dx, cudaStream_t st) {
  const int64_t n3 = (int64_t)n_slices * kSlice * 3;
  k_nt_temporal<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(d, n_slices, slice_env, hist_len, hist, dx);
}

void launch_nt_keep_hist(const NewtonDev& d, int n_slices, const int* slice_env, int hist_len, const double* dx,
                         double* hist, cudaStream_t st) {
  const int64_t n3 = (int64_t)n_slices * kSlice * 3;
  k_nt_keep_hist<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(d, n_slices, slice_env, hist_len, dx, hist);
}

void launch_nt_after_solve(const NewtonDev& d, int ls_max_iter, cudaGraphConditionalHandle ls, cudaStream_t st) {
  k_nt_after_solve<<<1, kNtThreads, 0, st>>>(d, ls_max_iter, ls);
}

void launch_nt_ls_scale(const NewtonDev& d, double alpha, cudaStream_t st) {
  k_nt_ls_scale<<<1, kNtThreads, 0, st>>>(d, alpha);
}

void launch_nt_ls_check(const NewtonDev& d, int ls_max_iter, cudaGraphConditionalHandle ls, cudaStream_t st) {
  k_nt_ls_check<<<1, kNtThreads, 0, st>>>(d, ls_max_iter, ls);
}

}  // namespace sdx
