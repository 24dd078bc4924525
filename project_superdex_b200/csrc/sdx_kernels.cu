// sdx_kernels.cu — sm_100a kernels of the implicit soft-body step.
//
// Element assembly follows fem::StressWork / GravityWork / InertiaWork
// (mochi_core/include/mochi_core/element_operations/fem_stress.h:107-262, fem_gravity.h:44-128,
// fem_inertia.h:55-137) with the DRes seeded by the scaled mass matrix
// (mochi_physics/src/mochi_soft.cpp:249-262). Contact follows the penalty response
// (mochi_core/include/mochi_core/contact/contact_utils.h:498-570) integrated by TractionWork
// (fem_traction.h:58-178). The linear solve is the reference's left-preconditioned CG with the
// residual-L2 stop test (mochi_core/include/mochi_core/linear_algebra/krylov/pcg.h:70-238), fused
// into one persistent cooperative launch per solve.
#include <array>
#include <cooperative_groups.h>

#include "sdx_device.cuh"
#include "sdx_internal.cuh"

namespace sdx {

// ------------------------------------------------------------------------------------------------
// mass couplings and Hessian seeding

__global__ void k_mass_accum(int64_t n_tets, const int4* __restrict__ s0, const int4* __restrict__ s1,
                             const int4* __restrict__ s2, const int4* __restrict__ s3,
                             const float4* __restrict__ rest3, float* mass) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tets) return;
  const float4 r3 = rest3[t];
  const float m = r3.w * r3.x / 20.0f;  // rho * vol / 20: P1 consistent mass (Q4 exact)
  const int4 sl[4] = {s0[t], s1[t], s2[t], s3[t]};
  const int* sp = reinterpret_cast<const int*>(sl);
#pragma unroll
  for (int f = 0; f < 4; ++f)
#pragma unroll
    for (int g = 0; g < 4; ++g) atomicAdd(mass + sp[f * 4 + g], f == g ? 2.0f * m : m);
}

void launch_mass_accum(int64_t n_tets, const int4* slots[4], const float4* rest3, float* mass,
                       cudaStream_t st) {
  if (n_tets == 0) return;
  const int th = 256;
  k_mass_accum<<<(unsigned)((n_tets + th - 1) / th), th, 0, st>>>(n_tets, slots[0], slots[1], slots[2],
                                                                   slots[3], rest3, mass);
}

// One warp per slice: DRes <- mass_scale * M with Dirichlet rows/cols (unit diagonal).
__global__ void k_seed_hessian(Matrix A, const float* __restrict__ mass, const uint8_t* __restrict__ pin,
                               const uint8_t* __restrict__ env_mask, float mass_scale) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= A.n_slices) return;
  const int s = warp;
  if (env_mask && !env_mask[A.slice_env[s]]) return;
  const int row = s * kSlice + lane;
  const int base = A.slice_ptr[s], w = A.slice_w[s];
  const int pr = pin[row];
  for (int k = 0; k < w; ++k) {
    const int p = base + k * kSlice + lane;
    const int cj = A.col[p];
    if (cj & kPadBit) {
#pragma unroll
      for (int e = 0; e < 9; ++e) A.val[val_index(p, e)] = 0.0f;
      continue;
    }
    const int pc = pin[cj];
    const float m = mass[p] * mass_scale;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float v = (r == c) ? m : 0.0f;
        if (((pr >> r) & 1) || ((pc >> c) & 1)) v = (cj == row && r == c) ? 1.0f : 0.0f;
        A.val[val_index(p, r * 3 + c)] = v;
      }
  }
}

void launch_seed_hessian(const Matrix& A, const float* mass, const uint8_t* pin, const uint8_t* env_mask,
                         float mass_scale, cudaStream_t st) {
  if (A.n_slices == 0) return;
  const int th = 256;
  const int64_t threads = (int64_t)A.n_slices * 32;
  k_seed_hessian<<<(unsigned)((threads + th - 1) / th), th, 0, st>>>(A, mass, pin, env_mask, mass_scale);
}

// ------------------------------------------------------------------------------------------------
// per-tet element kernel

__device__ __forceinline__ void warp_env_add(double* obj, int env, double v) {
  // aggregate lanes of the same env before one atomic
  // (the shuffles name only the lanes of this env, which all run the same number of them)
  const unsigned mask = __activemask();
  const unsigned same = __match_any_sync(mask, env);
  const int leader = __ffs(same) - 1;
  double s = 0.0;
  for (unsigned m = same; m; m &= m - 1) {
    const int l = __ffs(m) - 1;
    s += __shfl_sync(same, v, l);
  }
  if ((int)(threadIdx.x & 31) == leader) atomicAdd(obj + env, s);
}

// One 3x3 block into the sliced-ELL values: entries 0-3 and 4-7 are 16-byte-aligned runs, so two float4
// reductions and one scalar one. kAgg: the lanes of the warp (those converged here) that hold a block for
// the same position p first add their blocks in the group's lowest lane, which alone writes. On the
// Freudenthal split of a tet grid a warp's 32 tets share the hex diagonals, so the diagonal blocks of
// nodes 0 and 3 (and the off-diagonal pair between them) repeat up to 6 times per warp instruction.
template <bool kAgg>
__device__ __forceinline__ void scatter_block(float* val, int p, const float kb[9]) {
  if (kAgg) {
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, p);
    const int lane = (int)(threadIdx.x & 31);
    if (peers != (1u << lane)) {
      float s[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) s[i] = 0.0f;
      for (unsigned m = peers; m; m &= m - 1) {  // every lane of the group runs the same shuffles
        const int l = __ffs(m) - 1;
#pragma unroll
        for (int i = 0; i < 9; ++i) s[i] += __shfl_sync(peers, kb[i], l);
      }
      if (lane != __ffs(peers) - 1) return;
      atomicAdd(reinterpret_cast<float4*>(val + val_index(p, 0)), make_float4(s[0], s[1], s[2], s[3]));
      atomicAdd(reinterpret_cast<float4*>(val + val_index(p, 4)), make_float4(s[4], s[5], s[6], s[7]));
      atomicAdd(val + val_index(p, 8), s[8]);
      return;
    }
  }
  atomicAdd(reinterpret_cast<float4*>(val + val_index(p, 0)), make_float4(kb[0], kb[1], kb[2], kb[3]));
  atomicAdd(reinterpret_cast<float4*>(val + val_index(p, 4)), make_float4(kb[4], kb[5], kb[6], kb[7]));
  atomicAdd(val + val_index(p, 8), kb[8]);
}

// kArap: the variant that also evaluates ARAP envs (SVD-based, more registers); launched only when some
// env uses ARAP, so the other materials keep the lean variant. kDamp: the variant with Rayleigh stiffness
// damping (viscous stress, its residual, energy and Hessian terms), launched only when it is on. kAgg:
// warp-aggregated block scatter (scatter_block). The lean variant fits 128 registers, so 512 threads share
// an SM whatever the CTA size (64, 128 or 256 threads, a launch-time choice of the shape tuner).
template <bool kArap, bool kDamp, bool kAgg>
__global__ void __launch_bounds__(kElemMaxThreads, (kArap || kDamp) ? 1 : 2) k_element(ElemArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_tets) return;
  const int4 nd = a.tets[t];
  const int env = a.slice_env[nd.x >> 5];
  if (a.env_mask && !a.env_mask[env]) return;
  const int mat = a.env_material ? a.env_material[env] : 0;
  const float4 R0 = a.rest0[t], R1 = a.rest1[t], R2 = a.rest2[t], R3 = a.rest3[t];
  const float dN[12] = {R0.x, R0.y, R0.z, R0.w, R1.x, R1.y, R1.z, R1.w, R2.x, R2.y, R2.z, R2.w};
  const float vol = R3.x, mu = R3.y, lam = R3.z, rho = R3.w;
  const int rows[4] = {nd.x, nd.y, nd.z, nd.w};
  double uf[4][3];
#pragma unroll
  for (int f = 0; f < 4; ++f)
#pragma unroll
    for (int r = 0; r < 3; ++r) uf[f][r] = a.u[3 * (int64_t)rows[f] + r];
  double F[9] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};
#pragma unroll
  for (int f = 0; f < 4; ++f)
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) F[r * 3 + c] = fma(uf[f][r], (double)dN[3 * f + c], F[r * 3 + c]);

  const bool want_res = a.flags & 2, want_obj = a.flags & 1, want_hess = a.flags & 4;
  // Rayleigh stiffness damping: viscous stress about the stage-start displacement
  // (fem_stress_damping.h:29-501; reference stiffness = the tet's lambda, mu)
  double Sv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, dE[6];
  if (kDamp && a.kdamp > 0.0) {
    double Fs[9] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double us = a.u0[3 * (int64_t)rows[f] + r];
#pragma unroll
        for (int c = 0; c < 3; ++c) Fs[r * 3 + c] = fma(us, (double)dN[3 * f + c], Fs[r * 3 + c]);
      }
    // reference stiffness (ComputeReferenceMaterialStiffnessVoigt): (lambda, mu), for ARAP (0, mu / 2)
    const bool arap = kArap && mat == 5;
    const double l0 = arap ? 0.0 : (double)lam, m0 = arap ? 0.5 * (double)mu : (double)mu;
    visc_stress_f64(F, Fs, a.kdamp * l0, a.kdamp * m0, dE, Sv);
  }
  if (want_res || want_obj) {
    const SnhConsts kc = snh_consts((double)mu, (double)lam);
    const double w = (double)vol;
    const double m = (double)rho * w / 20.0;
    // inertia about the target ut and mass damping about the stage start u0 (mochi_physics/src/mochi_soft.h:
    // 408-420), P1Q4 consistent mass m (1 + delta_fg): per component the node sums, and for the energy the
    // squares; the per-node differences are formed again where they are used (the targets come from L1)
    double asum[3] = {0.0, 0.0, 0.0}, dsum[3] = {0.0, 0.0, 0.0}, ein = 0.0, edm = 0.0;
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double d_in = uf[f][r] - a.ut[3 * (int64_t)rows[f] + r];
        asum[r] += d_in;
        ein += d_in * d_in;
        if (a.mdamp > 0.0) {
          const double d_dm = uf[f][r] - a.u0[3 * (int64_t)rows[f] + r];
          dsum[r] += d_dm;
          edm += d_dm * d_dm;
        }
      }
    if (want_res) {
      double P[9];
      if (mat == 1)
        stvk_energy_pk1_f64((double)mu, (double)lam, F, nullptr, P);
      else if (mat == 2)
        linear_energy_pk1_f64((double)mu, (double)lam, F, nullptr, P);
      else if (kArap && mat == 5)
        arap_energy_pk1_f64((double)mu, F, nullptr, P);
      else
        snh_pk1_f64(kc, F, P);
      if (kDamp && a.kdamp > 0.0) {  // + F S_visc
        const double S[9] = {Sv[0], Sv[5], Sv[4], Sv[5], Sv[1], Sv[3], Sv[4], Sv[3], Sv[2]};
        double FS[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            FS[r * 3 + c] = F[r * 3 + 0] * S[c] + F[r * 3 + 1] * S[3 + c] + F[r * 3 + 2] * S[6 + c];
#pragma unroll
        for (int i = 0; i < 9; ++i) P[i] += FS[i];
      }
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int pf = a.pin[rows[f]];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          if ((pf >> r) & 1) continue;
          const int64_t idx = 3 * (int64_t)rows[f] + r;
          double v = (P[r * 3 + 0] * dN[3 * f + 0] + P[r * 3 + 1] * dN[3 * f + 1] +
                      P[r * 3 + 2] * dN[3 * f + 2]) * w;
          v -= (double)rho * a.grav[r] * w * 0.25;
          v += a.dtfi2 * m * ((uf[f][r] - a.ut[idx]) + asum[r]);
          if (a.mdamp > 0.0) v += a.mdamp * m * ((uf[f][r] - a.u0[idx]) + dsum[r]);
          atomicAdd(a.g + idx, v);
        }
      }
    }
    if (want_obj) {
      double xc[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int r = 0; r < 3; ++r) xc[r] += 0.25 * (a.X[3 * (int64_t)rows[f] + r] + uf[f][r]);
      ein = m * (ein + asum[0] * asum[0] + asum[1] * asum[1] + asum[2] * asum[2]);
      edm = m * (edm + dsum[0] * dsum[0] + dsum[1] * dsum[1] + dsum[2] * dsum[2]);
      double psi;
      if (mat == 1)
        stvk_energy_pk1_f64((double)mu, (double)lam, F, &psi, nullptr);
      else if (mat == 2)
        linear_energy_pk1_f64((double)mu, (double)lam, F, &psi, nullptr);
      else if (kArap && mat == 5)
        arap_energy_pk1_f64((double)mu, F, &psi, nullptr);
      else
        psi = snh_energy_f64(kc, F);
      if (kDamp && a.kdamp > 0.0) psi += 0.5 * (Sv[0] * dE[0] + Sv[1] * dE[1] + Sv[2] * dE[2] + Sv[3] * dE[3] +
                                       Sv[4] * dE[4] + Sv[5] * dE[5]);
      const double e = psi * w -
                       (double)rho * w * (a.grav[0] * xc[0] + a.grav[1] * xc[1] + a.grav[2] * xc[2]) +
                       0.5 * a.dtfi2 * ein + 0.5 * a.mdamp * edm;
      warp_env_add(a.obj, env, e);
    }
  }

  if (want_hess) {
    float Ff[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Ff[i] = (float)F[i];
    TanForm T;
    if (mat == 1)
      stvk_tanform(mu, lam, Ff, (a.flags & 8) != 0, a.psd, a.min_eig, T);
    else if (mat == 2)
      linear_tanform(mu, lam, T);
    else if (kArap && mat == 5)
      arap_tanform(mu, Ff, (a.flags & 8) != 0, a.psd, a.min_eig, T);
    else
      snh_tanform(mu, lam, Ff, (a.flags & 8) != 0, a.psd, a.min_eig, T);
    const int4 S0 = a.slots0[t], S1 = a.slots1[t], S2 = a.slots2[t], S3 = a.slots3[t];
    const int slot[16] = {S0.x, S0.y, S0.z, S0.w, S1.x, S1.y, S1.z, S1.w,
                          S2.x, S2.y, S2.z, S2.w, S3.x, S3.y, S3.z, S3.w};
    int pins[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) pins[f] = a.pin[rows[f]];
    // stiffness damping: Gauss-Newton part kappa B^T C0 B and the (projected) geometric part
    const bool kd = kDamp && a.kdamp > 0.0;
    float aF[4][3], FFt[9], Sg[9];
    const bool arap_h = kArap && mat == 5;
    const float kl = arap_h ? 0.0f : (float)(a.kdamp * (double)lam);
    const float km = (float)(a.kdamp * (arap_h ? 0.5 * (double)mu : (double)mu));
    if (kd) {
#pragma unroll
      for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int i = 0; i < 3; ++i)
          aF[f][i] = Ff[i * 3 + 0] * dN[3 * f + 0] + Ff[i * 3 + 1] * dN[3 * f + 1] + Ff[i * 3 + 2] * dN[3 * f + 2];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          FFt[i * 3 + j] = Ff[i * 3 + 0] * Ff[j * 3 + 0] + Ff[i * 3 + 1] * Ff[j * 3 + 1] + Ff[i * 3 + 2] * Ff[j * 3 + 2];
      const float s6[6] = {(float)Sv[0], (float)Sv[1], (float)Sv[2], (float)Sv[3], (float)Sv[4], (float)Sv[5]};
      Sg[0] = s6[0]; Sg[4] = s6[1]; Sg[8] = s6[2];
      Sg[5] = Sg[7] = s6[3];
      Sg[2] = Sg[6] = s6[4];
      Sg[1] = Sg[3] = s6[5];
      if (a.kdamp_geo && (a.flags & 8)) project_sym3_f32(Sg);
    }
    // Blocks K_fg = vol B_f^T C B_g (fem_stress.h:218-241) from the factored tangent, for f <= g; K_gf is the
    // transpose (C and the damping terms are symmetric). Pinned rows and columns stay zero. A block is
    // scattered whole: entries 0-3 and 4-7 are 16-byte aligned runs in the sliced-ELL value layout, so it
    // takes two float4 reductions and one scalar one.
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
#pragma unroll 1
      for (int g = f; g < 4; ++g) {
        const float df[3] = {dN[3 * f], dN[3 * f + 1], dN[3 * f + 2]};
        const float dg[3] = {dN[3 * g], dN[3 * g + 1], dN[3 * g + 2]};
        float kb[9];
        tan_block(T, df, dg, kb);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float k = vol * kb[3 * r + c];
            if (kd) {
              const float dd = df[0] * dg[0] + df[1] * dg[1] + df[2] * dg[2];
              float v = kl * aF[f][r] * aF[g][c] + km * (FFt[r * 3 + c] * dd + aF[g][r] * aF[f][c]);
              if (a.kdamp_geo && r == c) {
                float geo = 0.0f;
#pragma unroll
                for (int kk = 0; kk < 3; ++kk)
                  geo += df[kk] * (Sg[kk * 3 + 0] * dg[0] + Sg[kk * 3 + 1] * dg[1] + Sg[kk * 3 + 2] * dg[2]);
                v += geo;
              }
              k += vol * v;
            }
            kb[3 * r + c] = k;
          }
        float kt[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            kt[3 * c + r] = (((pins[g] >> c) & 1) || ((pins[f] >> r) & 1)) ? 0.0f : kb[3 * r + c];
            if (((pins[f] >> r) & 1) || ((pins[g] >> c) & 1)) kb[3 * r + c] = 0.0f;
          }
        scatter_block<kAgg>(a.val, slot[f * 4 + g], kb);
        if (g != f) scatter_block<kAgg>(a.val, slot[g * 4 + f], kt);
      }
    }
  }
}

template <bool kAgg>
static void launch_element_t(const ElemArgs& a, unsigned nb, int th, cudaStream_t st) {
  const bool damp = a.kdamp > 0.0;
  if (a.has_arap && damp)
    k_element<true, true, kAgg><<<nb, th, 0, st>>>(a);
  else if (a.has_arap)
    k_element<true, false, kAgg><<<nb, th, 0, st>>>(a);
  else if (damp)
    k_element<false, true, kAgg><<<nb, th, 0, st>>>(a);
  else
    k_element<false, false, kAgg><<<nb, th, 0, st>>>(a);
}

void launch_element(const ElemArgs& a, cudaStream_t st) {
  if (a.n_tets == 0) return;
  const int th = (a.threads == 64 || a.threads == 256) ? a.threads : 128;
  const unsigned nb = (unsigned)((a.n_tets + th - 1) / th);
  // the aggregated scatter only changes the Hessian's scatter; a residual-only launch takes the plain code
  if (a.aggregate && (a.flags & 4))
    launch_element_t<true>(a, nb, th, st);
  else
    launch_element_t<false>(a, nb, th, st);
}

// ------------------------------------------------------------------------------------------------
// contact: one thread per boundary sample (face, quadrature point)

__constant__ double c_face_w[3][3] = {{2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                                      {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0},
                                      {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0}};

__device__ __forceinline__ void face_normal(const double xn[3][3], double nrm[3]) {
  double e1[3], e2[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    e1[r] = xn[1][r] - xn[0][r];
    e2[r] = xn[2][r] - xn[0][r];
  }
  nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
  nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
  nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
  const double nl = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
#pragma unroll
  for (int r = 0; r < 3; ++r) nrm[r] = nl > 0.0 ? nrm[r] / nl : 0.0;
}

// Per (sample, collider) pair: the penalty response (contact_utils.h:498-570) with the alignment mask
// and, when dissipative, Coulomb / viscous friction and normal damping driven by the sample's displacement
// relative to the collider since the stage start (u0 at t0) and by the normal force at the stage-start
// distance (contact_utils.h:1003-1230). Colliders are rigid translations, so the collider frame is the
// world frame moved by vel t. With explicit normals the alignment, the friction plane and the normal
// force come from the stage start, and pairs in contact only at the stage start enter with d = thr.
__global__ void __launch_bounds__(256) k_contact(ContactArgs a) {
  const int64_t sidx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (sidx >= a.n_samples) return;
  const int64_t f = sidx / 3;
  const int q = (int)(sidx - 3 * f);
  const int4 fr = a.faces[f];
  const int env = fr.w;
  // the evaluation time: a launch captured once into a graph reads it from device memory
  const double t_now = a.t_dev ? *a.t_dev : a.t;
  const double t_stage = t_now - (a.t - a.t0);
  unsigned bits = 0;
  if (!a.env_mask || a.env_mask[env]) {
    const int rows[3] = {fr.x, fr.y, fr.z};
    const bool diss = a.coulomb > 0.0 || a.viscous > 0.0 || a.normal_damping > 0.0;
    const bool expl = (a.cflags & kContactExplicit) != 0;
    const bool need_ss = (diss || expl) && a.u0 != nullptr;
    double xn[3][3], xs[3], nrm[3], xs0[3], nrm0[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int r = 0; r < 3; ++r) xn[k][r] = a.X[3 * (int64_t)rows[k] + r] + a.u[3 * (int64_t)rows[k] + r];
    face_normal(xn, nrm);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      xs[r] = c_face_w[q][0] * xn[0][r] + c_face_w[q][1] * xn[1][r] + c_face_w[q][2] * xn[2][r];
    if (need_ss) {
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int r = 0; r < 3; ++r) xn[k][r] = a.X[3 * (int64_t)rows[k] + r] + a.u0[3 * (int64_t)rows[k] + r];
      face_normal(xn, nrm0);
#pragma unroll
      for (int r = 0; r < 3; ++r)
        xs0[r] = c_face_w[q][0] * xn[0][r] + c_face_w[q][1] * xn[1][r] + c_face_w[q][2] * xn[2][r];
    } else {
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        nrm0[r] = nrm[r];
        xs0[r] = xs[r];
      }
    }
    const double wq = a.face_area[f] / 3.0;
    const int c0 = a.coll_off[env], c1 = a.coll_off[env + 1];
    double energy = 0.0;
    for (int c = c0; c < c1; ++c) {
      const double* crow = a.colliders + 11 * (int64_t)c;
      double d, gr[3], d0 = 0.0, gr0[3] = {0.0, 0.0, 0.0};
      collider_sdf(crow, xs, t_now, d, gr);
      if (need_ss) collider_sdf(crow, xs0, t_stage, d0, gr0);
      const bool cur = d < a.thr;
      if (!cur && !(expl && d0 < a.thr)) continue;
      if (!cur) {  // in contact at the stage start only
        d = a.thr;
#pragma unroll
        for (int r = 0; r < 3; ++r) gr[r] = gr0[r];
      }
      const double* nc = expl ? gr0 : gr;
      const double* ncol = expl ? nrm0 : nrm;
      const double align = nc[0] * ncol[0] + nc[1] * ncol[1] + nc[2] * ncol[2];
      if (align > a.max_align) continue;  // masked: no energy, force or dforce
      bits |= 1u << (c - c0);
      double pv, dp, ddp;
      polyrelu(-d, a.t_half, a.t_half - a.thr, pv, dp, ddp);
      double E = 0.5 * a.k * pv * pv;
      const double fn = a.k * pv * dp, dfn = -a.k * (dp * dp + pv * ddp);
      double F[3], D[6];
#pragma unroll
      for (int r = 0; r < 3; ++r) F[r] = fn * gr[r];
      D[0] = dfn * gr[0] * gr[0];
      D[1] = dfn * gr[1] * gr[1];
      D[2] = dfn * gr[2] * gr[2];
      D[3] = dfn * gr[0] * gr[1];
      D[4] = dfn * gr[0] * gr[2];
      D[5] = dfn * gr[1] * gr[2];
      if (diss) {
        const double afac = ((a.cflags & kContactFade) && a.max_align > -1.0)
                                ? (a.max_align - align) / (a.max_align + 1.0)
                                : 1.0;
        double prel[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) prel[r] = (xs[r] - crow[8 + r] * t_now) - (xs0[r] - crow[8 + r] * t_stage);
        double fP;
        if (a.cflags & kContactImplicitFn) {
          fP = afac * fn;
        } else {
          const double dss = expl ? d0 : d - (gr[0] * prel[0] + gr[1] * prel[1] + gr[2] * prel[2]);
          double qv, dq, ddq;
          polyrelu(-dss, a.t_half, a.t_half - a.thr, qv, dq, ddq);
          fP = afac * a.k * qv * dq;
        }
        // the collider's normal (unit SDF gradient) or the colliding surface's, flipped
        double n[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) n[r] = (a.cflags & kContactColliderNormal) ? nc[r] : -ncol[r];
        dissipation_response(a.coulomb, a.falloff, a.viscous, a.normal_damping, (a.cflags & kContactFitted) != 0,
                             (a.cflags & kContactCinf) != 0, fP, n, prel, E, F, D);
      }
      energy += E * wq;
      if (a.flags & 2) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int pk = a.pin[rows[k]];
#pragma unroll
          for (int r = 0; r < 3; ++r)
            if (!((pk >> r) & 1)) atomicAdd(a.g + 3 * (int64_t)rows[k] + r, -F[r] * c_face_w[q][k] * wq);
        }
      }
      if (a.flags & 4) {
        // symmetric index of (r, cc) in D
        constexpr int kSym[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int pk = a.pin[rows[k]];
#pragma unroll
          for (int l = 0; l < 3; ++l) {
            const int pl = a.pin[rows[l]];
            const int p = a.face_slots[9 * f + 3 * k + l];
            const double wkl = c_face_w[q][k] * c_face_w[q][l] * wq;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
              for (int cc = 0; cc < 3; ++cc) {
                if (((pk >> r) & 1) || ((pl >> cc) & 1)) continue;
                atomicAdd(a.val + val_index(p, 3 * r + cc), (float)(-D[kSym[3 * r + cc]] * wkl));
              }
          }
        }
      }
    }
    if (a.flags & 1) {
      if (energy != 0.0) atomicAdd(a.obj + env, energy);
    }
    if (bits) atomicAdd(a.n_pairs + env, (unsigned long long)__popc(bits));
  }
  if (a.pair_mask) a.pair_mask[sidx] = bits;
}

void launch_contact(const ContactArgs& a, cudaStream_t st) {
  if (a.n_samples == 0) return;
  const int th = (a.threads == 64 || a.threads == 256) ? a.threads : 128;
  k_contact<<<(unsigned)((a.n_samples + th - 1) / th), th, 0, st>>>(a);
}

// ------------------------------------------------------------------------------------------------
// per-env reductions and row-wise vector kernels (one warp per slice)

__global__ void k_env_dot(int n_slices, const int* __restrict__ slice_env, const uint8_t* __restrict__ env_mask,
                          const double* __restrict__ a, const double* __restrict__ b, double* out) {
  __shared__ double sw[8];
  __shared__ int se[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * 8 + warp;
  double v = 0.0;
  int env = -1;
  if (s < n_slices) {
    env = slice_env[s];
    if (!env_mask || env_mask[env]) {
      const int64_t base = 3 * ((int64_t)s * kSlice + lane);
#pragma unroll
      for (int k = 0; k < 3; ++k) v += a[base + k] * b[base + k];
    } else {
      env = -1;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) {
    sw[warp] = v;
    se[warp] = env;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc = 0.0;
    int cur = -1;
    for (int w = 0; w < 8; ++w) {
      if (se[w] != cur) {
        if (cur >= 0) atomicAdd(out + cur, acc);
        cur = se[w];
        acc = 0.0;
      }
      acc += sw[w];
    }
    if (cur >= 0) atomicAdd(out + cur, acc);
  }
}

void launch_env_dot(int n_slices, const int* slice_env, const uint8_t* env_mask, const double* a,
                    const double* b, double* out, cudaStream_t st) {
  if (n_slices == 0) return;
  k_env_dot<<<(n_slices + 7) / 8, 256, 0, st>>>(n_slices, slice_env, env_mask, a, b, out);
}

__global__ void k_zero_rows(int n_slices, const int* __restrict__ slice_env, const uint8_t* __restrict__ env_mask,
                            double* v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // component index
  if (i >= (int64_t)n_slices * kSlice * 3) return;
  const int s = (int)(i / (kSlice * 3));
  if (env_mask && !env_mask[slice_env[s]]) return;
  v[i] = 0.0;
}

void launch_zero_rows(int n_slices, const int* slice_env, const uint8_t* env_mask, double* v,
                      cudaStream_t st) {
  const int64_t n = (int64_t)n_slices * kSlice * 3;
  if (n == 0) return;
  k_zero_rows<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_slices, slice_env, env_mask, v);
}

__global__ void k_pred(int64_t n3, const double* __restrict__ u, const double* __restrict__ v, double dt,
                       double* ut, double* u0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  const double ui = u[i];
  ut[i] = ui + dt * v[i];  // GatherPredTarget: x~ = x0 + dt v0 (batched_element_utils.h:90-123)
  u0[i] = ui;
}

void launch_pred(int64_t n3, const double* u, const double* v, double dt, double* ut, double* u0,
                 cudaStream_t st) {
  if (n3 == 0) return;
  k_pred<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(n3, u, v, dt, ut, u0);
}

__global__ void k_ls_candidate(int n_slices, const int* __restrict__ slice_env,
                               const uint8_t* __restrict__ env_mask, const double* __restrict__ ubase,
                               const double* __restrict__ dx, const double* __restrict__ scale, double* u) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n_slices * kSlice * 3) return;
  const int env = slice_env[i / (kSlice * 3)];
  if (env_mask && !env_mask[env]) return;
  u[i] = ubase[i] - scale[env] * dx[i];
}

void launch_ls_candidate(int n_slices, const int* slice_env, const uint8_t* env_mask,
                         const double* ubase, const double* dx, const double* scale, double* u,
                         cudaStream_t st) {
  const int64_t n = (int64_t)n_slices * kSlice * 3;
  if (n == 0) return;
  k_ls_candidate<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_slices, slice_env, env_mask, ubase, dx,
                                                               scale, u);
}

__global__ void k_copy_rows(int n_slices, const int* __restrict__ slice_env, const uint8_t* __restrict__ env_mask,
                            const double* __restrict__ src, double* dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n_slices * kSlice * 3) return;
  if (env_mask && !env_mask[slice_env[i / (kSlice * 3)]]) return;
  dst[i] = src[i];
}

void launch_copy_rows(int n_slices, const int* slice_env, const uint8_t* env_mask, const double* src,
                      double* dst, cudaStream_t st) {
  const int64_t n = (int64_t)n_slices * kSlice * 3;
  if (n == 0) return;
  k_copy_rows<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_slices, slice_env, env_mask, src, dst);
}

__global__ void k_velocity(int64_t n3, const double* __restrict__ u, const double* __restrict__ u0, double dt,
                           double* v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  v[i] = (u[i] - u0[i]) / dt;
}

void launch_velocity(int64_t n3, const double* u, const double* u0, double dt, double* v,
                     cudaStream_t st) {
  if (n3 == 0) return;
  k_velocity<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(n3, u, u0, dt, v);
}

__global__ void k_pack_z(int64_t n_rows, const double* __restrict__ x, float4* z) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rows) return;
  z[i] = make_float4((float)x[3 * i], (float)x[3 * i + 1], (float)x[3 * i + 2], 0.0f);
}

void launch_pack_z(int64_t n_rows, const double* x, float4* z, cudaStream_t st) {
  if (n_rows == 0) return;
  k_pack_z<<<(unsigned)((n_rows + 255) / 256), 256, 0, st>>>(n_rows, x, z);
}

// ------------------------------------------------------------------------------------------------
// SELL-32 3x3 SpMV building block: acc = A_row . src (one warp per slice, lane = row)

// loads of one (slice, k) group for lane `lane`: 9 values (4 + 4 + 1 split, see val_index)
__device__ __forceinline__ void load_block(const float* g, int lane, float v[9]) {
  const float4 a = __ldcs(reinterpret_cast<const float4*>(g) + lane);
  const float4 b = __ldcs(reinterpret_cast<const float4*>(g + 128) + lane);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
  v[4] = b.x;
  v[5] = b.y;
  v[6] = b.z;
  v[7] = b.w;
  v[8] = __ldcs(g + 256 + lane);
}

// Batched: the column, value and gather loads of 4 groups are issued before their FMAs (fits 64 registers).
template <class Load>
__device__ __forceinline__ void sell_row_product(const Matrix& A, int s, int lane, Load load, float& a0,
                                                 float& a1, float& a2) {
  const int base = A.slice_ptr[s], w = A.slice_w[s];
  a0 = a1 = a2 = 0.0f;
  int k = 0;
  // four groups per batch: all column, value and gather loads are issued before the FMAs
  for (; k + 4 <= w; k += 4) {
    int j[4];
    float v[4][9];
    float4 xj[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) j[u] = __ldcs(A.col + base + (k + u) * kSlice + lane) & 0x7fffffff;
#pragma unroll
    for (int u = 0; u < 4; ++u) load_block(A.val + (size_t)(base + (k + u) * kSlice) * 9, lane, v[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) xj[u] = load(j[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a0 = fmaf(v[u][0], xj[u].x, fmaf(v[u][1], xj[u].y, fmaf(v[u][2], xj[u].z, a0)));
      a1 = fmaf(v[u][3], xj[u].x, fmaf(v[u][4], xj[u].y, fmaf(v[u][5], xj[u].z, a1)));
      a2 = fmaf(v[u][6], xj[u].x, fmaf(v[u][7], xj[u].y, fmaf(v[u][8], xj[u].z, a2)));
    }
  }
  for (; k < w; ++k) {
    const int j = __ldcs(A.col + base + k * kSlice + lane) & 0x7fffffff;
    float v[9];
    load_block(A.val + (size_t)(base + k * kSlice) * 9, lane, v);
    const float4 xj = load(j);
    a0 = fmaf(v[0], xj.x, fmaf(v[1], xj.y, fmaf(v[2], xj.z, a0)));
    a1 = fmaf(v[3], xj.x, fmaf(v[4], xj.y, fmaf(v[5], xj.z, a1)));
    a2 = fmaf(v[6], xj.x, fmaf(v[7], xj.y, fmaf(v[8], xj.z, a2)));
  }
}

// loads of 4 consecutive (slice, k) groups starting at k (groups past the row width load group k with
// zero weight, so the batch needs no branch)
__device__ __forceinline__ void load_batch(const Matrix& A, int base, int k, int w, int lane, int row, int j[4],
                                           float v[4][9]) {
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const bool ok = k + u < w;
    const int kk = ok ? k + u : k;
    j[u] = ok ? (__ldcs(A.col + base + kk * kSlice + lane) & 0x7fffffff) : row;
    load_block(A.val + (size_t)(base + kk * kSlice) * 9, lane, v[u]);
    if (!ok) {
#pragma unroll
      for (int e = 0; e < 9; ++e) v[u][e] = 0.0f;
    }
  }
}

// Software-pipelined: the columns and values of the next batch of 4 groups are in flight while the
// current batch gathers its x entries, so the matrix stream does not stall on the gather latency.
template <class Load>
__device__ __forceinline__ void sell_row_product_pipe(const Matrix& A, int s, int lane, Load load, float& a0,
                                                      float& a1, float& a2) {
  const int base = A.slice_ptr[s], w = A.slice_w[s];
  const int row = s * kSlice + lane;
  a0 = a1 = a2 = 0.0f;
  if (w <= 0) return;
  int j0[4], j1[4];
  float v0[4][9], v1[4][9];
  load_batch(A, base, 0, w, lane, row, j0, v0);
  for (int k = 0; k < w; k += 4) {
    const bool more = k + 4 < w;
    if (more) load_batch(A, base, k + 4, w, lane, row, j1, v1);
    float4 xj[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) xj[u] = load(j0[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a0 = fmaf(v0[u][0], xj[u].x, fmaf(v0[u][1], xj[u].y, fmaf(v0[u][2], xj[u].z, a0)));
      a1 = fmaf(v0[u][3], xj[u].x, fmaf(v0[u][4], xj[u].y, fmaf(v0[u][5], xj[u].z, a1)));
      a2 = fmaf(v0[u][6], xj[u].x, fmaf(v0[u][7], xj[u].y, fmaf(v0[u][8], xj[u].z, a2)));
    }
    if (more) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        j0[u] = j1[u];
#pragma unroll
        for (int e = 0; e < 9; ++e) v0[u][e] = v1[u][e];
      }
    }
  }
}

__global__ void k_spmv(Matrix A, const float4* __restrict__ x, float* __restrict__ y) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= A.n_slices) return;
  float a0, a1, a2;
  sell_row_product_pipe(A, s, lane, [&](int j) { return __ldg(x + j); }, a0, a1, a2);
  const int64_t row = (int64_t)s * kSlice + lane;
  y[3 * row] = a0;
  y[3 * row + 1] = a1;
  y[3 * row + 2] = a2;
}

void launch_spmv(const Matrix& A, const float4* x, float* y, int threads, cudaStream_t st) {
  if (A.n_slices == 0) return;
  const int64_t t = (int64_t)A.n_slices * 32;
  k_spmv<<<(unsigned)((t + threads - 1) / threads), threads, 0, st>>>(A, x, y);
}

// ------------------------------------------------------------------------------------------------
// BSR (FP32) -> SELL-32. One thread per block row. Values either as contiguous row-major 3x3 blocks, or
// as the reference's row strips (strips = true): block row br with len blocks is one row-major 3 x 3len
// strip at 9 row_ptr[br], entry (lr, lc) of its k-th block at 3 (lr len + k) + lc (block_sparse_matrix.h:
// 459-475).

__global__ void k_bsr_to_sell(int n_rows, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ bcol,
                              const float* __restrict__ bval, int strips, const int* __restrict__ slice_ptr,
                              int* col, float* val, int* diag_pos) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n_rows) return;
  const int s = row >> 5, lane = row & 31;
  const int base = slice_ptr[s];
  const int w = (slice_ptr[s + 1] - base) / kSlice;
  const int64_t b0 = row_ptr[row], len = row_ptr[row + 1] - b0;
  diag_pos[row] = -1;
  for (int k = 0; k < w; ++k) {
    const int p = base + k * kSlice + lane;
    if (k < len) {
      const int j = bcol[b0 + k];
      col[p] = j;
      if (j == row) diag_pos[row] = p;
#pragma unroll
      for (int e = 0; e < 9; ++e)
        val[val_index(p, e)] = strips ? bval[9 * b0 + 3 * ((e / 3) * len + k) + e % 3] : bval[9 * (b0 + k) + e];
    } else {
      col[p] = row | kPadBit;
#pragma unroll
      for (int e = 0; e < 9; ++e) val[val_index(p, e)] = 0.0f;
    }
  }
}

void launch_bsr_to_sell(int n_rows, const int64_t* row_ptr, const int32_t* bcol, const float* bval, bool strips,
                        const int* slice_ptr, int* col, float* val, int* diag_pos, cudaStream_t st) {
  if (n_rows == 0) return;
  k_bsr_to_sell<<<(n_rows + 127) / 128, 128, 0, st>>>(n_rows, row_ptr, bcol, bval, strips ? 1 : 0, slice_ptr, col,
                                                       val, diag_pos);
}

// ------------------------------------------------------------------------------------------------
// Persistent Jacobi-PCG (one cooperative launch per solve, every env of the batch at once).
//
// Per iteration two grid barriers:
//   phase 1: p <- z + beta p, q <- A z + beta q (= A p by linearity), partial p.q
//   phase 2: x += alpha p, r -= alpha q (FP64), z <- M^-1 r, partials r.r, r.z_old, r.z
// Every `replace_every` iterations, and one iteration after an env's recurrence residual first meets
// the tolerance, r is recomputed as b - A x with FP64 accumulation (extra barrier) and the stop test
// uses that true residual. Per-env scalars are reduced deterministically: each CTA writes one partial
// per (CTA, env) it covers and every CTA that needs an env's total sums that env's partials in a fixed
// order, so all CTAs hold bit-identical alpha / beta / status for their envs.


struct EnvState {
  double rz, alpha, beta, conv_thr, div_thr, bb;
  double rr;   // the latest checked r.r (reported on a non-SPD abort, as pcg.h:152-169 reports it)
  int status;  // 0 active, 1 converged, 2 stopped, 3 diverged, 4 not requested, 5 diverging
  int first;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier on a monotonically increasing arrival counter (sync[0], zero at launch): the k-th barrier
// of a launch completes when the counter reaches k * nblocks. One atomic per CTA and no reset, so the
// last arrival releases every waiting CTA within one L2 round trip. The spin is bounded: on timeout
// sync[2] is set and every CTA unwinds.
__device__ __forceinline__ bool grid_barrier(unsigned* sync, unsigned nblocks, long long spin_limit) {
  __shared__ unsigned s_bar_err;
  __syncthreads();
  if (threadIdx.x == 0) {
    // release: this CTA's writes (ordered before thread 0 by the CTA barrier) become visible with the
    // arrival; acquire: the poll that sees the last arrival orders every later load of the CTA after all
    // CTAs' pre-barrier writes (the CTA barrier below extends it to the other threads)
    unsigned prev;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], 1;" : "=r"(prev) : "l"(sync) : "memory");
    const unsigned target = (prev / nblocks + 1u) * nblocks;
    long long spins = 0;
    unsigned err;
    for (;;) {
      // the error word is read beside each poll (a relaxed load issued first, so both are in flight at
      // once): a CTA that timed out stops arriving, so the others time out at a later barrier at worst
      err = ld_relaxed_gpu(sync + 2);
      if ((int)(ld_acquire_gpu(sync) - target) >= 0) break;
      if (++spins > spin_limit) {
        atomicExch(sync + 2, 1u);  // device timeout: recorded, the kernel unwinds
        err = 1u;
        break;
      }
      __nanosleep(32);
    }
    s_bar_err = err;
  }
  __syncthreads();
  return s_bar_err == 0u;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void prec_apply(const PcgArgs& a, int64_t row, const double r[3], float z[3]) {
  if (a.precond == 1) {
    const float* d = a.dinv + 3 * row;
    z[0] = (float)(d[0] * r[0]);
    z[1] = (float)(d[1] * r[1]);
    z[2] = (float)(d[2] * r[2]);
  } else if (a.precond == 2) {
    const float* B = a.dinv + 9 * row;
#pragma unroll
    for (int k = 0; k < 3; ++k) z[k] = (float)(B[3 * k] * r[0] + B[3 * k + 1] * r[1] + B[3 * k + 2] * r[2]);
  } else {
    z[0] = (float)r[0];
    z[1] = (float)r[1];
    z[2] = (float)r[2];
  }
}

// y = A v for the 32 rows of slice s, FP64 accumulation (FP32 matrix values, FP64 v gathered from L2)
// y = A v (and y2 = A v2 with kVec = 2) for one slice row: FP32 blocks times FP64 gathers, accumulated in
// FP64 in ascending block order. The column, value and gather loads of kBatch consecutive groups are issued
// before their FMAs (the loop was latency bound one group at a time).
template <int kBatch, int kVec>
__device__ __forceinline__ void spmv_f64_rows(const Matrix& A, int s, int lane, const double* __restrict__ v1,
                                              const double* __restrict__ v2, double y1[3], double y2[3]) {
  const int base = A.slice_ptr[s], w = A.slice_w[s];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
  auto acc = [&](const float v[9], const double x[3], const double z[3]) {
    a0 += (double)v[0] * x[0] + (double)v[1] * x[1] + (double)v[2] * x[2];
    a1 += (double)v[3] * x[0] + (double)v[4] * x[1] + (double)v[5] * x[2];
    a2 += (double)v[6] * x[0] + (double)v[7] * x[1] + (double)v[8] * x[2];
    if constexpr (kVec == 2) {
      b0 += (double)v[0] * z[0] + (double)v[1] * z[1] + (double)v[2] * z[2];
      b1 += (double)v[3] * z[0] + (double)v[4] * z[1] + (double)v[5] * z[2];
      b2 += (double)v[6] * z[0] + (double)v[7] * z[1] + (double)v[8] * z[2];
    }
  };
  int k = 0;
  for (; k + kBatch <= w; k += kBatch) {
    int j[kBatch];
    float v[kBatch][9];
    double x[kBatch][3], z[kBatch][3];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) j[u] = __ldcs(A.col + base + (k + u) * kSlice + lane) & 0x7fffffff;
#pragma unroll
    for (int u = 0; u < kBatch; ++u) load_block(A.val + (size_t)(base + (k + u) * kSlice) * 9, lane, v[u]);
#pragma unroll
    for (int u = 0; u < kBatch; ++u)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        x[u][c] = __ldcg(v1 + 3 * (int64_t)j[u] + c);
        if constexpr (kVec == 2) z[u][c] = __ldcg(v2 + 3 * (int64_t)j[u] + c);
      }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) acc(v[u], x[u], z[u]);
  }
  for (; k < w; ++k) {
    const int j = __ldcs(A.col + base + k * kSlice + lane) & 0x7fffffff;
    float v[9];
    load_block(A.val + (size_t)(base + k * kSlice) * 9, lane, v);
    double x[3], z[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      x[c] = __ldcg(v1 + 3 * (int64_t)j + c);
      if constexpr (kVec == 2) z[c] = __ldcg(v2 + 3 * (int64_t)j + c);
    }
    acc(v, x, z);
  }
  y1[0] = a0;
  y1[1] = a1;
  y1[2] = a2;
  if constexpr (kVec == 2) {
    y2[0] = b0;
    y2[1] = b1;
    y2[2] = b2;
  }
}

// r = b - A x with FP64 accumulation (FP32 matrix values, FP64 x gathered from L2)
template <int kBatch>
__device__ __forceinline__ void true_residual(const PcgArgs& a, int s, int lane, double r[3]) {
  double ax[3];
  spmv_f64_rows<kBatch, 1>(a.A, s, lane, a.x, nullptr, ax, nullptr);
  const int64_t row = (int64_t)s * kSlice + lane;
  r[0] = a.b[3 * row] - ax[0];
  r[1] = a.b[3 * row + 1] - ax[1];
  r[2] = a.b[3 * row + 2] - ax[2];
}

// Iterative refinement: r = b - A x in FP64 (FP32 matrix values) for the slices of the envs in env_mask, one
// warp per slice, one row per lane.
__global__ void k_residual64(Matrix A, const uint8_t* __restrict__ env_mask, const double* __restrict__ x,
                             const double* __restrict__ b, double* __restrict__ r) {
  const int s = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= A.n_slices) return;
  if (env_mask && !env_mask[A.slice_env[s]]) return;
  double ax[3];
  spmv_f64_rows<4, 1>(A, s, lane, x, nullptr, ax, nullptr);
  const int64_t row = (int64_t)s * kSlice + lane;
#pragma unroll
  for (int c = 0; c < 3; ++c) r[3 * row + c] = b[3 * row + c] - ax[c];
}

void launch_residual64(const Matrix& A, const uint8_t* env_mask, const double* x, const double* b, double* r,
                       cudaStream_t st) {
  if (A.n_slices == 0) return;
  const int64_t threads = (int64_t)A.n_slices * kSlice;
  k_residual64<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(A, env_mask, x, b, r);
}

// x += d on the rows of the envs in env_mask
__global__ void k_add_rows(int n_slices, const int* __restrict__ slice_env, const uint8_t* __restrict__ env_mask,
                           const double* __restrict__ d, double* x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n_slices * kSlice * 3) return;
  if (env_mask && !env_mask[slice_env[i / (kSlice * 3)]]) return;
  x[i] += d[i];
}

void launch_add_rows(int n_slices, const int* slice_env, const uint8_t* env_mask, const double* d, double* x,
                     cudaStream_t st) {
  const int64_t n = (int64_t)n_slices * kSlice * 3;
  if (n == 0) return;
  k_add_rows<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_slices, slice_env, env_mask, d, x);
}

// Bulk L2 prefetch of [ptr, ptr + bytes) (one instruction, no registers held; address and size multiples of
// 16 bytes). A warp issues these for the slice it will process next, so that slice's loads hit L2.
__device__ __forceinline__ void prefetch_l2(const void* ptr, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ptr), "r"(bytes) : "memory");
}

// Phase-2 operands of slice s (DoF-linear: p, q, Jacobi diagonal FP32, z float4 rows; x and r FP64, or the
// FP32 increment of x when z carries r), one array per lane 0..5.
__device__ __forceinline__ void prefetch_update_operands(const PcgArgs& a, int s, int lane) {
  const int64_t d0 = (int64_t)s * (3 * kSlice);
  if (lane == 0) {
    if (a.r_in_z)
      prefetch_l2(a.xi + d0, 3 * kSlice * 4);
    else
      prefetch_l2(a.x + d0, 3 * kSlice * 8);
  }
  if (lane == 1 && !a.r_in_z) prefetch_l2(a.r + d0, 3 * kSlice * 8);
  if (lane == 2) prefetch_l2(a.p + d0, 3 * kSlice * 4);
  if (lane == 3) prefetch_l2(a.q + d0, 3 * kSlice * 4);
  if (lane == 4 && a.precond == 1) prefetch_l2(a.dinv + d0, 3 * kSlice * 4);
  if (lane == 5) prefetch_l2(a.z + (int64_t)s * kSlice, kSlice * 16);
}

// x += xi, xi = 0 on slice s (DoF-linear): folds the FP32 increment of x accumulated since the last
// true-residual replacement into the FP64 x.
__device__ __forceinline__ void fold_x_increment(const PcgArgs& a, int s, int lane) {
  const int64_t d0 = (int64_t)s * (3 * kSlice);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int64_t d = d0 + lane + 32 * j;
    a.x[d] += (double)a.xi[d];
    a.xi[d] = 0.0f;
  }
}

// Matrix range of slice s (column indices and the 9 values of every block position), lanes 6 and 7.
__device__ __forceinline__ void prefetch_slice_matrix(const Matrix& A, int s, int lane) {
  if (lane != 6 && lane != 7) return;
  const int base = A.slice_ptr[s], w = A.slice_w[s];
  if (w <= 0) return;
  if (lane == 6)
    prefetch_l2(A.col + base, (uint32_t)(w * kSlice * 4));
  else
    prefetch_l2(A.val + (size_t)base * 9, (uint32_t)(w * kSlice * 36));
}

// kPipe: SpMV phase with the software-pipelined row product (128 registers, so at most 512 threads per
// SM); otherwise the batched product that fits 64 registers at 1024 threads.
// kTimed: the variant with the per-CTA phase timers (launched only when they are asked for, so that the
// default variant's code is exactly the untimed one)
template <bool kPipe, bool kTimed>
__global__ void __launch_bounds__(kPipe ? 512 : 1024, 1) k_pcg(PcgArgs a) {
  extern __shared__ double wacc[];  // [nwarps][a.wstride][kPcgNq]
  __shared__ EnvState st[kPcgMaxEnvsPerCta];
  constexpr int kB64 = kPipe ? 4 : 2;  // groups per batch of the FP64 SpMVs (register budget of the variant)
  __shared__ double tot[kPcgMaxEnvsPerCta][kPcgNq];
  __shared__ int s_exit, s_replace;
  __shared__ float s_tr[(kPipe ? 16 : 32) * 3 * kSlice];  // per warp: a slice's row products, DoF order
  const int c = blockIdx.x;
  const unsigned ncta = gridDim.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // this CTA's entries [s0, s1) of the slice list and its envs (ascending) s_env[0 .. ne)
  const int s0 = a.cta_slice[c], s1 = a.cta_slice[c + 1];
  const int eo = a.cta_eoff[c];
  const int ne = (s1 > s0) ? (a.cta_eoff[c + 1] - eo) : 0;
  __shared__ int s_env[kPcgMaxEnvsPerCta];
  __shared__ int s_repart;
  for (int le = threadIdx.x; le < ne; le += blockDim.x) s_env[le] = a.cta_envs[eo + le];
  auto slice_of = [&](int i) { return a.slice_list ? a.slice_list[i] : i; };
  auto local_env = [&](int ev) {  // index of env ev in s_env
    int lo = 0, hi = ne - 1;
    while (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (s_env[m] < ev)
        lo = m + 1;
      else
        hi = m;
    }
    return lo;
  };

  const int ws = a.wstride;
  auto clear_acc = [&]() {  // the slots of this CTA's envs only
    const int per_warp = ne * kPcgNq;
    for (int i = threadIdx.x; i < nwarps * per_warp; i += blockDim.x) {
      const int w = i / per_warp, j = i - w * per_warp;
      wacc[w * ws * kPcgNq + j] = 0.0;
    }
    __syncthreads();
  };
  auto add_acc = [&](int le, int k, double v) {
    v = warp_sum(v);
    if (lane == 0) wacc[(warp * ws + le) * kPcgNq + k] += v;
  };
  // Partials of phase 1 live in buffer 1, those of phases 0 and 2 in buffer 0, so a CTA writing the
  // next phase's partials never overwrites values another CTA is still reducing. The partials of one
  // env are contiguous (one per covering CTA, in CTA order), so a reduction is a coalesced read.
  const size_t pstride = (size_t)a.env_poff[a.n_envs] * kPcgNq;
  auto flush_acc = [&](int nq, int buf) {
    __syncthreads();
    for (int i = threadIdx.x; i < ne * nq; i += blockDim.x) {
      const int le = i / nq, k = i % nq;
      double v = 0.0;
      for (int w = 0; w < nwarps; ++w) v += wacc[(w * ws + le) * kPcgNq + k];
      const int e = s_env[le];
      a.part[buf * pstride + (size_t)(a.env_poff[e] + (c - a.env_cta0[e])) * kPcgNq + k] = v;
    }
  };
  auto reduce_tot = [&](int nq, int buf) {
    // fixed summation order, identical in every CTA. Envs spread over at most 8 CTAs: one thread per
    // (env, quantity) sums the partials in CTA order (one load round for all of this CTA's envs) ...
    for (int i = threadIdx.x; i < ne * nq; i += blockDim.x) {
      const int le = i / nq, k = i % nq;
      const int e = s_env[le];
      const int n = a.env_cta1[e] - a.env_cta0[e] + 1;
      if (n > 8) continue;
      const double* src = a.part + buf * pstride + (size_t)a.env_poff[e] * kPcgNq + k;
      double v = 0.0;
      for (int j = 0; j < n; ++j) v += __ldcg(src + (size_t)j * kPcgNq);
      tot[le][k] = v;
    }
    // ... wider envs: one warp per (env, quantity)
    for (int i = warp; i < ne * nq; i += nwarps) {
      const int le = i / nq, k = i % nq;
      const int e = s_env[le];
      const int n = a.env_cta1[e] - a.env_cta0[e] + 1;
      if (n <= 8) continue;
      const double* src = a.part + buf * pstride + (size_t)a.env_poff[e] * kPcgNq + k;
      double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
      int j = lane;
      for (; j + 96 < n; j += 128) {
        v0 += __ldcg(src + (size_t)j * kPcgNq);
        v1 += __ldcg(src + (size_t)(j + 32) * kPcgNq);
        v2 += __ldcg(src + (size_t)(j + 64) * kPcgNq);
        v3 += __ldcg(src + (size_t)(j + 96) * kPcgNq);
      }
      for (; j < n; j += 32) v0 += __ldcg(src + (size_t)j * kPcgNq);
      const double v = warp_sum((v0 + v1) + (v2 + v3));
      if (lane == 0) tot[le][k] = v;
    }
    __syncthreads();
  };
  auto finish_env = [&](int le, int it, double rr) {
    const int e = s_env[le];
    if (a.env_cta0[e] == c) {
      a.out_iters[e] = it;
      a.out_res[e] = sqrt(fmax(rr, 0.0));
      a.out_relres[e] = st[le].bb == 0.0 ? 0.0 : sqrt(fmax(rr, 0.0) / st[le].bb);
      a.out_conv[e] = st[le].status;
      atomicSub((int*)(a.sync + 3), 1);
      if (a.env_nrows) atomicSub((int*)(a.sync + 5), a.env_nrows[e]);
    }
  };

  // Dot-product partials stay in registers while a warp's consecutive slices belong to one env (its
  // slices ascend, so the env changes rarely); the warp sums them into the shared per-(warp, env) slots
  // only when the env changes and at the end of the phase (acc_end). acc_le is uniform in the warp.
  double acc[3] = {0.0, 0.0, 0.0};
  int acc_le = -1;
  auto acc_flush = [&]() {
    if (acc_le < 0) return;
    add_acc(acc_le, 0, acc[0]);
    add_acc(acc_le, 1, acc[1]);
    add_acc(acc_le, 2, acc[2]);
    acc[0] = acc[1] = acc[2] = 0.0;
  };
  auto acc_add = [&](int le, int k, double v) {
    if (le != acc_le) {
      acc_flush();
      acc_le = le;
    }
    acc[k] += v;
  };
  auto acc_end = [&](int nq) {  // nq is 1 or 3; constant indices keep acc[] in registers
    if (nq == 1) {
      if (acc_le >= 0) add_acc(acc_le, 0, acc[0]);
      acc[0] = 0.0;
    } else {
      acc_flush();
    }
    acc_le = -1;
  };

  for (int le = threadIdx.x; le < ne; le += blockDim.x) {
    if (a.resume) {  // continue a re-partitioned solve: the CG scalars saved at the previous exit
      const EnvSave& sv = a.es[s_env[le]];
      st[le].rz = sv.rz;
      st[le].rr = sv.rr;
      st[le].beta = sv.beta;
      st[le].bb = sv.bb;
      st[le].conv_thr = sv.conv_thr;
      st[le].div_thr = sv.div_thr;
      st[le].first = sv.first;
      st[le].status = sv.status;
    } else {
      st[le].status = (a.env_mask && !a.env_mask[s_env[le]]) ? 4 : 0;
      st[le].first = 1;
      st[le].beta = 0.0;
    }
  }
  if (threadIdx.x == 0) s_repart = 0;
  __syncthreads();

  if (!a.resume) {
    // ---- phase 0: r = b - A x0, z = M^-1 r, partials b.b, r.r, r.z ----
    const bool zero_guess = a.zero_guess_dev ? (*a.zero_guess_dev != 0) : (a.zero_guess != 0);
    const bool scaled = !zero_guess && a.scale_guess;
    const bool two = scaled && a.x2 != nullptr;
    if (two) {
      // Galerkin start on span{x, x2} (the temporal guess and the learned correction): with Ah = A x,
      // Ay = A x2, the coefficients (ca, cb) minimise the A-norm error, i.e. solve
      // [x.Ah x.Ay; x.Ay x2.Ay] (ca, cb) = (x.b, x2.b). Among that pair and the one-vector optima, the
      // env keeps the one with the smallest A-norm error whose residual ||b - ca Ah - cb Ay|| is below
      // ||b|| (the measure of the stop test); failing all, the zero start.
      clear_acc();
      for (int i = s0 + warp; i < s1; i += nwarps) {
        const int s = slice_of(i);
        const int le = local_env(a.A.slice_env[s]);
        if (st[le].status != 0) continue;
        const int64_t row = (int64_t)s * kSlice + lane;
        double ah[3], ay[3];
        spmv_f64_rows<kB64, 2>(a.A, s, lane, a.x, a.x2, ah, ay);  // one pass over the matrix for both
        // kept for the residual of the combination (r is not gathered in this pass)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.r[3 * row + k] = ah[k];
          a.gal[3 * row + k] = ay[k];
        }
        double q[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double h = a.x[3 * row + k], y = a.x2[3 * row + k], bk = a.b[3 * row + k];
          q[0] += bk * bk;
          q[1] += h * bk;
          q[2] += y * bk;
          q[3] += h * ah[k];
          q[4] += h * ay[k];
          q[5] += y * ay[k];
          q[6] += bk * ah[k];
          q[7] += bk * ay[k];
          q[8] += ah[k] * ah[k];
          q[9] += ah[k] * ay[k];
          q[10] += ay[k] * ay[k];
        }
#pragma unroll
        for (int k = 0; k < 11; ++k) add_acc(le, k, q[k]);
      }
      flush_acc(11, 1);
      if (!grid_barrier(a.sync, ncta, a.spin_limit)) return;
      reduce_tot(11, 1);
      for (int le = threadIdx.x; le < ne; le += blockDim.x) {
        const double* t = tot[le];
        const double bb = t[0];
        auto res2 = [&](double ca, double cb) {
          return bb - 2.0 * (ca * t[6] + cb * t[7]) + ca * ca * t[8] + 2.0 * ca * cb * t[9] + cb * cb * t[10];
        };
        double best_gain = 0.0, ba = 0.0, bc = 0.0;
        auto consider = [&](double ca, double cb) {
          const double gain = ca * t[1] + cb * t[2];  // A-norm error reduction at a Galerkin optimum
          if (isfinite(gain) && gain > best_gain && res2(ca, cb) < bb) {
            best_gain = gain;
            ba = ca;
            bc = cb;
          }
        };
        const double det = t[3] * t[5] - t[4] * t[4];
        if (t[3] > 0.0 && t[5] > 0.0 && det > 1e-12 * t[3] * t[5])
          consider((t[1] * t[5] - t[2] * t[4]) / det, (t[3] * t[2] - t[4] * t[1]) / det);
        if (t[3] > 0.0) consider(t[1] / t[3], 0.0);
        if (t[5] > 0.0) consider(0.0, t[2] / t[5]);
        st[le].alpha = ba;
        st[le].beta = bc;
      }
      __syncthreads();
      for (int i = s0 + warp; i < s1; i += nwarps) {
        const int s = slice_of(i);
        const int le = local_env(a.A.slice_env[s]);
        if (st[le].status != 0) continue;
        const int64_t row = (int64_t)s * kSlice + lane;
        const double ca = st[le].alpha, cb = st[le].beta;
        // x = ca h + cb y and its residual b - ca A h - cb A y from the kept products: row-local, so the
        // pass below needs neither a barrier nor another SpMV
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.x[3 * row + k] = ca * a.x[3 * row + k] + cb * a.x2[3 * row + k];
          a.r[3 * row + k] = a.b[3 * row + k] - ca * a.r[3 * row + k] - cb * a.gal[3 * row + k];
        }
      }
      __syncthreads();
      for (int le = threadIdx.x; le < ne; le += blockDim.x) st[le].beta = 0.0;
      __syncthreads();
    } else if (scaled) {
      // energy-optimal scaling of the guess: alpha = (x0.b) / (x0.A x0), A x0 = b - r0; the scaled start
      // alpha x0 never has a larger A-norm error than the zero start. The guess is kept only if it also
      // lowers the residual the stop test measures: ||b - alpha A x0||^2 = (1-alpha)^2 b.b
      // + 2 alpha (1-alpha) b.r0 + alpha^2 r0.r0 < b.b; otherwise the env falls back to the zero start.
      clear_acc();
      for (int i = s0 + warp; i < s1; i += nwarps) {
        const int s = slice_of(i);
        const int le = local_env(a.A.slice_env[s]);
        if (st[le].status != 0) continue;
        const int64_t row = (int64_t)s * kSlice + lane;
        double r[3];
        true_residual<kB64>(a, s, lane, r);
        double xb = 0.0, xr = 0.0, bb = 0.0, br = 0.0, rr = 0.0;
  #pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.r[3 * row + k] = r[k];
          const double xk = a.x[3 * row + k], bk = a.b[3 * row + k];
          xb += xk * bk;
          xr += xk * r[k];
          bb += bk * bk;
          br += bk * r[k];
          rr += r[k] * r[k];
        }
        add_acc(le, 0, bb);
        add_acc(le, 1, xb);
        add_acc(le, 2, xr);
        add_acc(le, 3, br);
        add_acc(le, 4, rr);
      }
      flush_acc(5, 1);
      if (!grid_barrier(a.sync, ncta, a.spin_limit)) return;
      reduce_tot(5, 1);
      for (int le = threadIdx.x; le < ne; le += blockDim.x) {
        const double bb = tot[le][0], xb = tot[le][1], xax = tot[le][1] - tot[le][2];
        double al = (xax > 0.0 && xb > 0.0 && isfinite(xb / xax)) ? xb / xax : 0.0;
        const double ra = (1.0 - al) * (1.0 - al) * bb + 2.0 * al * (1.0 - al) * tot[le][3] + al * al * tot[le][4];
        if (!(ra < bb)) al = 0.0;
        st[le].alpha = al;
      }
      __syncthreads();
    }
    clear_acc();
    for (int i = s0 + warp; i < s1; i += nwarps) {
      const int s = slice_of(i);
      const int le = local_env(a.A.slice_env[s]);
      if (st[le].status != 0) continue;
      const int64_t row = (int64_t)s * kSlice + lane;
      // preconditioner from the diagonal block (BlockJacobiPrec<1> / <3>, block_jacobi_prec.h:35-151)
      const int dp = a.diag_pos[row];
      if (a.precond == 1) {
  #pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float d = dp >= 0 ? a.A.val[val_index(dp, 4 * k)] : 0.0f;
          a.dinv[3 * row + k] = d != 0.0f ? 1.0f / d : 1.0f;
        }
      } else if (a.precond == 2) {
        float B[9];
  #pragma unroll
        for (int e = 0; e < 9; ++e) B[e] = dp >= 0 ? a.A.val[val_index(dp, e)] : 0.0f;
        float cof[9];
        cof3(B, cof);
        const float det = det3(B);
        const float inv = det != 0.0f ? 1.0f / det : 0.0f;
  #pragma unroll
        for (int i = 0; i < 3; ++i)
  #pragma unroll
          for (int j = 0; j < 3; ++j) a.dinv[9 * row + 3 * i + j] = cof[3 * j + i] * inv;
      }
      double r[3];
      if (zero_guess) {
  #pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.x[3 * row + k] = 0.0;
          r[k] = a.b[3 * row + k];
        }
      }
      if (!zero_guess && !scaled) true_residual<kB64>(a, s, lane, r);
      if (two) {
  #pragma unroll
        for (int k = 0; k < 3; ++k) r[k] = a.r[3 * row + k];
      }
      if (scaled && !two) {
        const double al = st[le].alpha;
  #pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.x[3 * row + k] *= al;
          r[k] = (1.0 - al) * a.b[3 * row + k] + al * a.r[3 * row + k];
        }
      }
      float z[3];
      prec_apply(a, row, r, z);
  #pragma unroll
      for (int k = 0; k < 3; ++k) {
        a.r[3 * row + k] = r[k];
        if (a.r_in_z) a.xi[3 * row + k] = 0.0f;
      }
      a.z[row] = make_float4(z[0], z[1], z[2], 0.0f);
      const double b0 = a.b[3 * row], b1 = a.b[3 * row + 1], b2 = a.b[3 * row + 2];
      add_acc(le, 0, b0 * b0 + b1 * b1 + b2 * b2);
      add_acc(le, 1, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      add_acc(le, 2, r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
    }
    flush_acc(3, 0);
    if (!grid_barrier(a.sync, ncta, a.spin_limit)) return;
    reduce_tot(3, 0);
    for (int le = threadIdx.x; le < ne; le += blockDim.x) {
      if (st[le].status != 0) continue;
      const double bb = tot[le][0], rr = tot[le][1];
      st[le].bb = bb;
      const double rt = a.env_rel_tol ? a.env_rel_tol[s_env[le]] : a.rel_tol;
      st[le].conv_thr = fmax(a.abs_tol * a.abs_tol, (bb * rt) * rt);
      st[le].div_thr = (bb * a.rel_div_tol) * a.rel_div_tol;
      st[le].rz = tot[le][2];
      st[le].rr = rr;
      if (!isfinite(rr) || rr > st[le].div_thr) {
        st[le].status = 3;
        finish_env(le, 0, rr);
      } else if (rr <= st[le].conv_thr) {
        st[le].status = 1;
        finish_env(le, 0, rr);
      }
    }
    __syncthreads();
  }

  // per-CTA phase timing (thread 0, when asked for): a phase's mark follows flush_acc, whose CTA barrier
  // has seen every warp finish the phase. The SM cycle counter: a %globaltimer read just before each
  // barrier arrival delayed the arrival measurably (about 3 us per iteration)
  __shared__ unsigned long long t_ph[kTimed ? 5 : 1];  // 4 phase sums and the last mark
  if constexpr (kTimed) {
    if (threadIdx.x == 0)
      for (int k = 0; k < 5; ++k) t_ph[k] = 0ull;
  }
  auto mark = [&](int k) {
    if constexpr (kTimed) {
      if (threadIdx.x == 0) {
        const unsigned long long t = (unsigned long long)clock64();
        if (k >= 0) t_ph[k] += t - t_ph[4];
        t_ph[4] = t;
      }
    }
  };
  auto mark_out = [&]() {
    if constexpr (kTimed) {
      if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) atomicAdd(a.cta_ns + 4 * c + k, t_ph[k]);
    }
  };
  // At a launch's exit every env of this CTA's slices that took part gets its x increment folded in (an
  // env that stopped between replacements, or every env before a re-partition relaunch).
  auto fold_all = [&]() {
    if (!a.r_in_z || a.precond == 2) return;
    for (int i = s0 + warp; i < s1; i += nwarps) {
      const int s = slice_of(i);
      if (st[local_env(a.A.slice_env[s])].status == 4) continue;
      fold_x_increment(a, s, lane);
    }
  };
  mark(-1);
  for (int it = a.resume ? a.it0 : 1;; ++it) {
    // ---- phase 1 ----
    // The row product runs one row per lane; the vector updates run DoF-linear: DoF dl = lane + 32 j
    // (j = 0, 1, 2) of the slice, i.e. row 32 s + dl / 3, component dl % 3, so every load and store of p
    // and q is one contiguous 128-byte line per warp. The row products reach the DoF layout through the
    // warp's 96-float staging row in shared memory; z (just gathered by the product) comes from L1.
    clear_acc();
    float* tr = s_tr + warp * (3 * kSlice);
    const float* zf = reinterpret_cast<const float*>(a.z);
    for (int i = s0 + warp; i < s1; i += nwarps) {
      const int s = slice_of(i);
      const int le = local_env(a.A.slice_env[s]);
      if (st[le].status != 0) continue;
      if (a.prefetch && i + nwarps < s1) prefetch_slice_matrix(a.A, slice_of(i + nwarps), lane);
      const int64_t d0 = (int64_t)s * (3 * kSlice);
      // own DoF operands are loaded before the row product so that their latency overlaps it
      const bool first = st[le].first != 0;
      float po[3] = {0.0f, 0.0f, 0.0f}, qo[3] = {0.0f, 0.0f, 0.0f};
      if (!first) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          po[j] = a.p[d0 + lane + 32 * j];
          qo[j] = a.q[d0 + lane + 32 * j];
        }
      }
      float a0, a1, a2;
      // z gathers are weak L1-cacheable loads: z was last written before the grid barrier, whose acquire
      // fence (thread 0, then __syncthreads) orders every thread of the CTA after those writes, as with
      // cooperative-groups grid.sync(); neighbour rows of the same slice then hit in L1
      if constexpr (kPipe)
        sell_row_product_pipe(a.A, s, lane, [&](int j) { return a.z[j]; }, a0, a1, a2);
      else
        sell_row_product(a.A, s, lane, [&](int j) { return a.z[j]; }, a0, a1, a2);
      tr[3 * lane] = a0;
      tr[3 * lane + 1] = a1;
      tr[3 * lane + 2] = a2;
      __syncwarp();
      const float beta = first ? 0.0f : (float)st[le].beta;
      double pq = 0.0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int dl = lane + 32 * j;
        const float zv = zf[4 * ((int64_t)s * kSlice + dl / 3) + dl % 3];
        const float pn = fmaf(beta, po[j], zv);
        const float qn = fmaf(beta, qo[j], tr[dl]);
        a.p[d0 + dl] = pn;
        a.q[d0 + dl] = qn;
        pq += (double)pn * qn;
      }
      __syncwarp();
      acc_add(le, 0, pq);
    }
    acc_end(1);
    flush_acc(1, 1);
    mark(0);
    if (!grid_barrier(a.sync, ncta, a.spin_limit)) return;
    mark(1);
    // the last thread reads the run flags while the others load the partials: both round trips overlap
    if (threadIdx.x == blockDim.x - 1) {
      s_exit = *((volatile int*)(a.sync + 3)) <= 0;
      // re-partition after this iteration once few rows are left to iterate
      s_repart = a.repart_rows > 0 && (long long)*((volatile int*)(a.sync + 5)) <= a.repart_rows;
      const int vi = *((volatile int*)(a.sync + 4));
      s_replace = (vi > 0 && vi == it - 1) || (a.replace_every > 0 && it % a.replace_every == 0);
    }
    reduce_tot(1, 1);
    if (s_exit) {
      fold_all();
      mark_out();
      break;
    }
    const bool replace = s_replace != 0;
    for (int le = threadIdx.x; le < ne; le += blockDim.x) {
      if (st[le].status != 0) continue;
      const double pq = tot[le][0];
      st[le].alpha = st[le].rz / pq;
      // non-SPD abort (pcg.h:152-169): the env stops now, its exit is published in the post-barrier
      // stage below so that every CTA reads the same active count after the next barrier
      if (pq <= 0.0 && a.abort_spd) st[le].status = 5;
    }
    __syncthreads();

    // ---- phase 2 ----
    clear_acc();
    if (a.precond != 2) {
      // none / Jacobi: element-wise, DoF-linear (contiguous 256-byte lines of x and r per warp instruction);
      // prefetch distance a.prefetch slices of this warp (one slice's update is shorter than an HBM round
      // trip)
      const int ahead = a.prefetch;
      for (int k = 0; k < ahead && s0 + warp + k * nwarps < s1; ++k)
        prefetch_update_operands(a, slice_of(s0 + warp + k * nwarps), lane);
      for (int i = s0 + warp; i < s1; i += nwarps) {
        const int s = slice_of(i);
        if (ahead > 0 && i + ahead * nwarps < s1) prefetch_update_operands(a, slice_of(i + ahead * nwarps), lane);
        const int le = local_env(a.A.slice_env[s]);
        if (st[le].status != 0) continue;
        const int64_t d0 = (int64_t)s * (3 * kSlice);
        const double al = st[le].alpha;
        if (replace) {  // only x (and its folded increment): the true residual that follows recomputes r, z
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int64_t d = d0 + lane + 32 * j;
            const double inc = a.r_in_z ? (double)a.xi[d] : 0.0;
            a.x[d] += inc + al * (double)a.p[d];
            if (a.r_in_z) a.xi[d] = 0.0f;
          }
          continue;
        }
        // With r_in_z, r is carried by z between true-residual replacements: r = z / d (FP32 precision;
        // d = 1 without a preconditioner), and x by its FP64 value at the last replacement plus the FP32
        // increment xi, so the update reads and writes no FP64 vector. Every operand load is issued before
        // the first store (the update is latency bound).
        double xo[3] = {0.0, 0.0, 0.0}, ro[3] = {0.0, 0.0, 0.0};
        float xio[3] = {0.0f, 0.0f, 0.0f};
        float pp[3], qq[3], dd[3], zo[3];
        // the old z arrives as whole float4 rows (one per lane) and reaches the DoF layout through the
        // warp's staging row
        const float4 zrow = a.z[(int64_t)s * kSlice + lane];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const int dl = lane + 32 * j;
          if (a.r_in_z) {
            xio[j] = a.xi[d0 + dl];
          } else {
            xo[j] = a.x[d0 + dl];
            ro[j] = a.r[d0 + dl];
          }
          pp[j] = a.p[d0 + dl];
          qq[j] = a.q[d0 + dl];
          dd[j] = a.precond == 1 ? a.dinv[d0 + dl] : 1.0f;
        }
        tr[3 * lane] = zrow.x;
        tr[3 * lane + 1] = zrow.y;
        tr[3 * lane + 2] = zrow.z;
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 3; ++j) zo[j] = tr[lane + 32 * j];
        __syncwarp();
        double rr = 0.0, rzo = 0.0, rz = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const int dl = lane + 32 * j;
          if (a.r_in_z)
            a.xi[d0 + dl] = (float)((double)xio[j] + al * (double)pp[j]);
          else
            a.x[d0 + dl] = xo[j] + al * (double)pp[j];
          const double rp =
              !a.r_in_z ? ro[j] : (a.precond == 1 ? (double)(zo[j] / dd[j]) : (double)zo[j]);
          const double r = rp - al * (double)qq[j];
          if (!a.r_in_z) a.r[d0 + dl] = r;
          const float z = (float)(dd[j] * r);
          tr[dl] = z;
          rr += r * r;
          rzo += r * zo[j];
          rz += r * z;
        }
        __syncwarp();
        // new z: whole float4 rows (full sectors, no partial writes)
        a.z[(int64_t)s * kSlice + lane] = make_float4(tr[3 * lane], tr[3 * lane + 1], tr[3 * lane + 2], 0.0f);
        __syncwarp();
        acc_add(le, 0, rr);
        acc_add(le, 1, rzo);
        acc_add(le, 2, rz);
      }
    } else {
    for (int i = s0 + warp; i < s1; i += nwarps) {
      const int s = slice_of(i);
      const int le = local_env(a.A.slice_env[s]);
      if (st[le].status != 0) continue;
      const int64_t row = (int64_t)s * kSlice + lane;
      // block Jacobi: the row's 3x3 inverse diagonal block, one row per lane
      double xo[3], ro[3];
      float pp[3], qq[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        xo[k] = a.x[3 * row + k];
        pp[k] = a.p[3 * row + k];
        ro[k] = a.r[3 * row + k];
        qq[k] = a.q[3 * row + k];
      }
      const float4 zo = replace ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : a.z[row];
      const double al = st[le].alpha;
      double r[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        a.x[3 * row + k] = xo[k] + al * (double)pp[k];
        r[k] = ro[k] - al * (double)qq[k];
      }
      if (replace) continue;
      float z[3];
      prec_apply(a, row, r, z);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.r[3 * row + k] = r[k];
      a.z[row] = make_float4(z[0], z[1], z[2], 0.0f);
      acc_add(le, 0, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      acc_add(le, 1, r[0] * zo.x + r[1] * zo.y + r[2] * zo.z);
      acc_add(le, 2, r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
    }
    }
    acc_end(3);
    if (replace) {
      if (!grid_barrier(a.sync, ncta, a.spin_limit)) return;
      for (int i = s0 + warp; i < s1; i += nwarps) {
        const int s = slice_of(i);
        const int le = local_env(a.A.slice_env[s]);
        if (st[le].status != 0) continue;
        const int64_t row = (int64_t)s * kSlice + lane;
        double r[3];
        true_residual<kB64>(a, s, lane, r);
        const float4 zo = a.z[row];
        float z[3];
        prec_apply(a, row, r, z);
#pragma unroll
        for (int k = 0; k < 3; ++k) a.r[3 * row + k] = r[k];
        a.z[row] = make_float4(z[0], z[1], z[2], 0.0f);
        acc_add(le, 0, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        acc_add(le, 1, r[0] * zo.x + r[1] * zo.y + r[2] * zo.z);
        acc_add(le, 2, r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
      }
      acc_end(3);
    }
    flush_acc(3, 0);
    mark(2);
    if (!grid_barrier(a.sync, ncta, a.spin_limit)) return;
    mark(3);
    reduce_tot(3, 0);
    for (int le = threadIdx.x; le < ne; le += blockDim.x) {
      if (st[le].status == 5) {  // non-SPD abort: the residual of the last completed iteration
        st[le].status = 3;
        finish_env(le, it, st[le].rr);
        continue;
      }
      if (st[le].status != 0) continue;
      const double rr = tot[le][0], rzo = tot[le][1], rzn = tot[le][2];
      if (!isfinite(rr) || rr > st[le].div_thr) {
        st[le].status = 3;
        finish_env(le, it, rr);
        continue;
      }
      if (rr <= st[le].conv_thr) {
        if (replace) {
          st[le].status = 1;
          finish_env(le, it, rr);
          continue;
        }
        if (a.env_cta0[s_env[le]] == c) atomicMax((int*)(a.sync + 4), it);
      }
      if (it >= a.max_iter) {
        st[le].status = 2;
        finish_env(le, it, rr);
        continue;
      }
      if (rzn == 0.0) {
        st[le].status = 3;
        finish_env(le, it, rr);
        continue;
      }
      const double bpr = (a.polak_ribiere && !st[le].first) ? rzo : 0.0;
      st[le].beta = (rzn - bpr) / st[le].rz;
      st[le].rz = rzn;
      st[le].rr = rr;
      st[le].first = 0;
    }
    __syncthreads();
    if (s_repart) {
      // save the CG scalars (the env's first CTA writes them) and exit; the host re-partitions the envs
      // still iterating and relaunches from iteration it + 1
      for (int le = threadIdx.x; le < ne; le += blockDim.x) {
        const int e = s_env[le];
        if (a.env_cta0[e] != c) continue;
        EnvSave sv;
        sv.rz = st[le].rz;
        sv.rr = st[le].rr;
        sv.beta = st[le].beta;
        sv.bb = st[le].bb;
        sv.conv_thr = st[le].conv_thr;
        sv.div_thr = st[le].div_thr;
        sv.first = st[le].first;
        sv.status = st[le].status;
        a.es[e] = sv;
      }
      if (c == 0 && threadIdx.x == 0) {
        a.sync[6] = (unsigned)(it + 1);
        a.sync[7] = 1u;
      }
      fold_all();
      mark_out();
      return;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Cluster PCG for batches of small envs. The grid kernel above iterates every env of a batch in lockstep
// with grid-wide barriers, so once most envs have converged each iteration costs the grid barrier's
// latency (~11 us) for a few thousand rows. Here a thread-block cluster solves one env at a time and
// takes the next env from a queue (largest first) when it finishes: the clusters never wait on each other,
// and the reductions and barriers inside a cluster go through distributed shared memory (a counter in
// CTA 0's shared memory, polled with cluster-scope acquire loads; partial sums read from every CTA's
// shared memory in rank order, so every CTA holds bit-identical scalars and takes the same branches).
// Same recurrence, stop tests, FP64 residual replacement and verification iteration as k_pcg, per env.
// Every wait is bounded: a timeout records the error word and the kernel unwinds to its final cluster
// barrier, which every CTA reaches exactly once.

constexpr int kClNq = 11;

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_size() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// address of this CTA's shared variable p in the shared memory of cluster CTA `rank`
__device__ __forceinline__ uint32_t cluster_map(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(r)
               : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ double cluster_ld_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ int cluster_ld_s32(uint32_t addr) {
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ void cluster_hw_sync() {
  asm volatile("barrier.cluster.arrive.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}

// Software cluster barrier (every thread of every CTA calls it): arrivals counted on CTA 0's shared
// counter with a cluster-scope release, the poll acquires. false when the wait gave up (error recorded).
// Staged update phase of the cluster PCG: per warp 2 to 4 buffers of one slice's operands (x increment,
// p, q, Jacobi diagonal: 96 floats each; z: 32 float4 rows), filled by bulk asynchronous copies whose bytes
// an mbarrier per buffer counts.
constexpr int kClMaxStages = 4;  // buffers per warp: PcgArgs::stage_update (2..4) of them are used
constexpr int kClStageBytes = 4 * (3 * kSlice * 4) + kSlice * 16;  // 2,048
constexpr int kClWarps = 16;
__host__ __device__ constexpr int cl_dyn_smem(int stages) { return kClWarps * stages * (kClStageBytes + 8); }

__device__ __forceinline__ uint32_t shared_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

// bounded wait for the completion of phase `parity` of the mbarrier at `bar`; false on timeout
__device__ __forceinline__ bool stage_wait(uint32_t bar, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// lane 0: the copies of slice s's update operands into stage buffer `buf` (all addresses 16-byte aligned, all
// sizes multiples of 16 bytes: the vectors start on 256-byte boundaries and a slice is 384 / 512 bytes)
__device__ __forceinline__ void stage_issue(const PcgArgs& a, int s, uint32_t buf, uint32_t bar) {
  const int64_t d0 = (int64_t)s * (3 * kSlice);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier generic reads of the buffer first
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"((uint32_t)kClStageBytes)
               : "memory");
  bulk_g2s(buf, a.xi + d0, 3 * kSlice * 4, bar);
  bulk_g2s(buf + 384, a.p + d0, 3 * kSlice * 4, bar);
  bulk_g2s(buf + 768, a.q + d0, 3 * kSlice * 4, bar);
  bulk_g2s(buf + 1152, a.dinv + d0, 3 * kSlice * 4, bar);
  bulk_g2s(buf + 1536, a.z + (int64_t)s * kSlice, kSlice * 16, bar);
}

__device__ __forceinline__ bool cluster_sync(uint32_t cnt, unsigned n, long long limit, unsigned* err, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev;
    asm volatile("atom.release.cluster.shared::cluster.add.u32 %0, [%1], 1;" : "=r"(prev) : "r"(cnt) : "memory");
    const unsigned target = (prev / n + 1u) * n;
    long long spins = 0;
    int ok = 1;
    for (;;) {
      unsigned v;
      asm volatile("ld.acquire.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(cnt) : "memory");
      if ((int)(v - target) >= 0) break;
      if (++spins > limit) {
        atomicExch(err, 1u);
        ok = 0;
        break;
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

__global__ void __launch_bounds__(512, 1) k_pcg_cluster(PcgArgs a) {
  __shared__ double wq[16][kClNq];     // per-warp partial sums
  __shared__ double s_part[2][kClNq];  // this CTA's partials, two buffers (consecutive reductions)
  __shared__ double s_tot[kClNq];
  __shared__ double s_gather[16][kClNq];  // every CTA's partials, gathered by one pass of remote loads
  __shared__ unsigned s_cnt;           // the cluster barrier counter (used in CTA 0)
  __shared__ int s_env, s_env_here, s_ok;
  __shared__ float s_tr[16 * 3 * kSlice];  // per warp: a slice's row products, DoF order
  __shared__ int s_stage_fail;              // a warp's staged copy did not arrive in time
  extern __shared__ __align__(128) unsigned char cl_dyn[];  // staged update phase (cl_dyn_smem bytes)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  float* const tr = s_tr + warp * (3 * kSlice);
  const float* const zf = reinterpret_cast<const float*>(a.z);
  const uint32_t rank = cluster_rank(), csize = cluster_size();
  // this warp's stage buffers and their mbarriers; ph holds the parity each buffer waits for next
  const int nst = a.stage_update;  // stage buffers per warp (0: the update phase reads global memory)
  const uint32_t stage_buf = shared_u32(cl_dyn) + (uint32_t)(warp * nst * kClStageBytes);
  const uint32_t stage_bar = shared_u32(cl_dyn) + (uint32_t)(kClWarps * nst * kClStageBytes + warp * nst * 8);
  const unsigned char* const stage_ptr = cl_dyn + warp * nst * kClStageBytes;
  uint32_t ph = 0u;
  if (nst > 0 && lane == 0) {
    for (int b = 0; b < nst; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(stage_bar + 8u * b), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (threadIdx.x == 0) {
    s_cnt = 0u;
    s_stage_fail = 0;
  }
  cluster_hw_sync();  // every CTA's shared memory is live before any remote access
  const uint32_t cnt = cluster_map(&s_cnt, 0);
  const uint32_t env0 = cluster_map(&s_env, 0);
  unsigned* const err = a.sync + 2;
  int rb = 0;  // partial buffer of the next reduction (the same sequence in every CTA)
  bool fail = false;

  auto acc_reset = [&]() {
    for (int i = threadIdx.x; i < nwarps * kClNq; i += blockDim.x) (&wq[0][0])[i] = 0.0;
    __syncthreads();
  };
  auto acc_add = [&](int k, double v) {
    v = warp_sum(v);
    if (lane == 0) wq[warp][k] += v;
  };
  // publish this CTA's partials, synchronise the cluster, gather all CTAs' partials (one remote load per
  // thread, all in flight at once) and sum them in rank order
  auto reduce = [&](int nq) {
    __syncthreads();
    if (threadIdx.x < nq) {
      double v = 0.0;
      for (int w = 0; w < nwarps; ++w) v += wq[w][threadIdx.x];
      s_part[rb][threadIdx.x] = v;
    }
    if (!cluster_sync(cnt, csize, a.spin_limit, err, &s_ok)) return false;
    if (threadIdx.x < (int)csize * nq) {
      const int r = threadIdx.x / nq, k = threadIdx.x - r * nq;
      s_gather[r][k] = cluster_ld_f64(cluster_map(&s_part[rb][k], (uint32_t)r));
    }
    __syncthreads();
    if (threadIdx.x < nq) {
      double v = 0.0;
      for (uint32_t r = 0; r < csize; ++r) v += s_gather[r][threadIdx.x];
      s_tot[threadIdx.x] = v;
    }
    rb ^= 1;
    __syncthreads();
    return true;
  };

  for (;;) {
    // ---- next env from the queue (CTA 0 takes it, every CTA reads it from CTA 0) ----
    if (rank == 0 && threadIdx.x == 0) {
      int h = (int)atomicAdd(a.sync + 1, 1u);
      // a queue of every env of the batch (built once for a graph-captured step) passes over the envs
      // outside this solve; at most cl_n takes in all
      if (a.cl_skip_masked && a.env_mask)
        while (h < a.cl_n && !a.env_mask[a.cl_envs[h]]) h = (int)atomicAdd(a.sync + 1, 1u);
      s_env = h < a.cl_n ? a.cl_envs[h] : -1;
    }
    if (!cluster_sync(cnt, csize, a.spin_limit, err, &s_ok)) break;
    if (threadIdx.x == 0) s_env_here = cluster_ld_s32(env0);
    __syncthreads();
    const int e = s_env_here;
    if (e < 0) break;
    const int sa = a.env_soff[e], ns = a.env_soff[e + 1] - sa;
    const int c0 = sa + (int)((int64_t)ns * rank / csize), c1 = sa + (int)((int64_t)ns * (rank + 1) / csize);

    // ---- phase 0: diagonal, start vector, r0, z0 ----
    const bool zero_guess = a.zero_guess_dev ? (*a.zero_guess_dev != 0) : (a.zero_guess != 0);
    const bool scaled = !zero_guess && a.scale_guess;
    const bool two = scaled && a.x2 != nullptr;
    double al0 = 0.0;
    if (two) {
      // Galerkin start on span{x, x2}, as in k_pcg: A h and A y in one FP64 pass, 11 reduced quantities,
      // the best of the pair and the one-vector optima whose residual is below ||b||, else the zero start
      acc_reset();
      for (int s = c0 + warp; s < c1; s += nwarps) {
        const int64_t row = (int64_t)s * kSlice + lane;
        double ah[3], ay[3];
        spmv_f64_rows<4, 2>(a.A, s, lane, a.x, a.x2, ah, ay);
        double q[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.r[3 * row + k] = ah[k];
          a.gal[3 * row + k] = ay[k];
          const double h = a.x[3 * row + k], y = a.x2[3 * row + k], bk = a.b[3 * row + k];
          q[0] += bk * bk;
          q[1] += h * bk;
          q[2] += y * bk;
          q[3] += h * ah[k];
          q[4] += h * ay[k];
          q[5] += y * ay[k];
          q[6] += bk * ah[k];
          q[7] += bk * ay[k];
          q[8] += ah[k] * ah[k];
          q[9] += ah[k] * ay[k];
          q[10] += ay[k] * ay[k];
        }
#pragma unroll
        for (int k = 0; k < 11; ++k) acc_add(k, q[k]);
      }
      if (!reduce(11)) {
        fail = true;
        break;
      }
      const double* t = s_tot;
      const double bb0 = t[0];
      auto res2 = [&](double ca, double cb) {
        return bb0 - 2.0 * (ca * t[6] + cb * t[7]) + ca * ca * t[8] + 2.0 * ca * cb * t[9] + cb * cb * t[10];
      };
      double best_gain = 0.0, ca = 0.0, cb = 0.0;
      auto consider = [&](double xa, double xb) {
        const double gain = xa * t[1] + xb * t[2];
        if (isfinite(gain) && gain > best_gain && res2(xa, xb) < bb0) {
          best_gain = gain;
          ca = xa;
          cb = xb;
        }
      };
      const double det = t[3] * t[5] - t[4] * t[4];
      if (t[3] > 0.0 && t[5] > 0.0 && det > 1e-12 * t[3] * t[5])
        consider((t[1] * t[5] - t[2] * t[4]) / det, (t[3] * t[2] - t[4] * t[1]) / det);
      if (t[3] > 0.0) consider(t[1] / t[3], 0.0);
      if (t[5] > 0.0) consider(0.0, t[2] / t[5]);
      for (int s = c0 + warp; s < c1; s += nwarps) {
        const int64_t row = (int64_t)s * kSlice + lane;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.x[3 * row + k] = ca * a.x[3 * row + k] + cb * a.x2[3 * row + k];
          a.r[3 * row + k] = a.b[3 * row + k] - ca * a.r[3 * row + k] - cb * a.gal[3 * row + k];
        }
      }
    } else if (scaled) {
      acc_reset();
      for (int s = c0 + warp; s < c1; s += nwarps) {
        const int64_t row = (int64_t)s * kSlice + lane;
        double r[3];
        true_residual<4>(a, s, lane, r);
        double xb = 0.0, xr = 0.0, bb = 0.0, br = 0.0, rr = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.r[3 * row + k] = r[k];
          const double xk = a.x[3 * row + k], bk = a.b[3 * row + k];
          xb += xk * bk;
          xr += xk * r[k];
          bb += bk * bk;
          br += bk * r[k];
          rr += r[k] * r[k];
        }
        acc_add(0, bb);
        acc_add(1, xb);
        acc_add(2, xr);
        acc_add(3, br);
        acc_add(4, rr);
      }
      if (!reduce(5)) {
        fail = true;
        break;
      }
      const double bb = s_tot[0], xb = s_tot[1], xax = s_tot[1] - s_tot[2];
      al0 = (xax > 0.0 && xb > 0.0 && isfinite(xb / xax)) ? xb / xax : 0.0;
      const double ra = (1.0 - al0) * (1.0 - al0) * bb + 2.0 * al0 * (1.0 - al0) * s_tot[3] + al0 * al0 * s_tot[4];
      if (!(ra < bb)) al0 = 0.0;
    }
    acc_reset();
    for (int s = c0 + warp; s < c1; s += nwarps) {
      const int64_t row = (int64_t)s * kSlice + lane;
      const int dp = a.diag_pos[row];
      if (a.precond == 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float d = dp >= 0 ? a.A.val[val_index(dp, 4 * k)] : 0.0f;
          a.dinv[3 * row + k] = d != 0.0f ? 1.0f / d : 1.0f;
        }
      } else if (a.precond == 2) {
        float B[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) B[q] = dp >= 0 ? a.A.val[val_index(dp, q)] : 0.0f;
        float cof[9];
        cof3(B, cof);
        const float det = det3(B);
        const float inv = det != 0.0f ? 1.0f / det : 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) a.dinv[9 * row + 3 * i + j] = cof[3 * j + i] * inv;
      }
      double r[3];
      if (zero_guess) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.x[3 * row + k] = 0.0;
          r[k] = a.b[3 * row + k];
        }
      } else if (two) {
#pragma unroll
        for (int k = 0; k < 3; ++k) r[k] = a.r[3 * row + k];  // this row's, written by this warp above
      } else if (scaled) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.x[3 * row + k] *= al0;
          r[k] = (1.0 - al0) * a.b[3 * row + k] + al0 * a.r[3 * row + k];
        }
      } else {
        true_residual<4>(a, s, lane, r);
      }
      float z[3];
      prec_apply(a, row, r, z);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        a.r[3 * row + k] = r[k];
        if (a.r_in_z) a.xi[3 * row + k] = 0.0f;
      }
      a.z[row] = make_float4(z[0], z[1], z[2], 0.0f);
      const double b0 = a.b[3 * row], b1 = a.b[3 * row + 1], b2 = a.b[3 * row + 2];
      acc_add(0, b0 * b0 + b1 * b1 + b2 * b2);
      acc_add(1, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      acc_add(2, r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
    }
    if (!reduce(3)) {
      fail = true;
      break;
    }
    const double bb = s_tot[0];
    const double rt = a.env_rel_tol ? a.env_rel_tol[e] : a.rel_tol;
    const double conv_thr = fmax(a.abs_tol * a.abs_tol, (bb * rt) * rt);
    const double div_thr = (bb * a.rel_div_tol) * a.rel_div_tol;
    double rz = s_tot[2], rr = s_tot[1], beta = 0.0;
    int status = 0, it_done = 0, verify_it = 0;
    bool first = true;
    if (!isfinite(rr) || rr > div_thr)
      status = 3;
    else if (rr <= conv_thr)
      status = 1;

    // ---- iterations ----
    for (int it = 1; status == 0; ++it) {
      // phase 1: p = z + beta p, q = A z + beta q, p.q (vector updates DoF-linear, as in k_pcg); every slice of
      // the CTA belongs to its one env, so each lane sums its slices and the warp reduces once per phase
      acc_reset();
      double pq_sum = 0.0;
      for (int s = c0 + warp; s < c1; s += nwarps) {
        if (a.prefetch && s + nwarps < c1) prefetch_slice_matrix(a.A, s + nwarps, lane);
        const int64_t d0 = (int64_t)s * (3 * kSlice);
        float po[3] = {0.0f, 0.0f, 0.0f}, qo[3] = {0.0f, 0.0f, 0.0f};
        if (!first) {
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            po[j] = a.p[d0 + lane + 32 * j];
            qo[j] = a.q[d0 + lane + 32 * j];
          }
        }
        float a0, a1, a2;
        sell_row_product_pipe(a.A, s, lane, [&](int j) { return a.z[j]; }, a0, a1, a2);
        tr[3 * lane] = a0;
        tr[3 * lane + 1] = a1;
        tr[3 * lane + 2] = a2;
        __syncwarp();
        const float fb = first ? 0.0f : (float)beta;
        double pq = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const int dl = lane + 32 * j;
          const float zv = zf[4 * ((int64_t)s * kSlice + dl / 3) + dl % 3];
          const float pn = fmaf(fb, po[j], zv);
          const float qn = fmaf(fb, qo[j], tr[dl]);
          a.p[d0 + dl] = pn;
          a.q[d0 + dl] = qn;
          pq += (double)pn * qn;
        }
        __syncwarp();
        pq_sum += pq;
      }
      acc_add(0, pq_sum);
      if (!reduce(1)) {
        fail = true;
        break;
      }
      const double pq = s_tot[0];
      const double al = rz / pq;
      if (pq <= 0.0 && a.abort_spd) {  // non-SPD abort (pcg.h:152-169): x keeps the previous iterate and
        it_done = it;                  // the reported residual is the last completed iteration's
        status = 3;
        break;
      }
      const bool replace = (verify_it > 0 && verify_it == it - 1) || (a.replace_every > 0 && it % a.replace_every == 0);
      // phase 2: x += alpha p, r -= alpha q, z = M^-1 r, r.r, r.z_old, r.z (DoF-linear unless block Jacobi)
      acc_reset();
      if (nst > 0 && !replace && a.precond == 1 && a.r_in_z) {
        // the operands of the warp's next nst slices are in flight into shared memory while it updates one
        double rr_sum = 0.0, rzo_sum = 0.0, rz_sum = 0.0;
        uint32_t pending = 0u;  // buffers with copies issued and not yet waited for
        bool ok = true;
        if (lane == 0)
          for (int b = 0; b < nst; ++b) {
            const int sb = c0 + warp + b * nwarps;
            if (sb < c1) stage_issue(a, sb, stage_buf + (uint32_t)(b * kClStageBytes), stage_bar + 8u * b);
          }
        for (int b = 0; b < nst; ++b)
          if (c0 + warp + b * nwarps < c1) pending |= 1u << b;
        int k = 0;
        for (int s = c0 + warp; s < c1; s += nwarps, ++k) {
          const int b = k % nst;
          const bool got = stage_wait(stage_bar + 8u * b, (ph >> b) & 1u, a.spin_limit);
          if (!__all_sync(0xffffffffu, got)) {
            ok = false;
            break;
          }
          ph ^= 1u << b;
          pending &= ~(1u << b);
          const float* const sx = reinterpret_cast<const float*>(stage_ptr + b * kClStageBytes);
          const float* const sp = sx + 3 * kSlice;
          const float* const sq = sp + 3 * kSlice;
          const float* const sd = sq + 3 * kSlice;
          const float* const sz = sd + 3 * kSlice;  // 32 float4 rows
          const int64_t d0 = (int64_t)s * (3 * kSlice);
          double rr2 = 0.0, rzo2 = 0.0, rz2 = 0.0;
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int dl = lane + 32 * j;
            const float zo = sz[4 * (dl / 3) + dl % 3], dd = sd[dl], pp = sp[dl], qq = sq[dl];
            a.xi[d0 + dl] = (float)((double)sx[dl] + al * (double)pp);
            const double r = (double)(zo / dd) - al * (double)qq;
            const float z = (float)(dd * r);
            tr[dl] = z;
            rr2 += r * r;
            rzo2 += r * zo;
            rz2 += r * z;
          }
          __syncwarp();
          a.z[(int64_t)s * kSlice + lane] = make_float4(tr[3 * lane], tr[3 * lane + 1], tr[3 * lane + 2], 0.0f);
          __syncwarp();  // every lane is done with buffer b and with tr
          rr_sum += rr2;
          rzo_sum += rzo2;
          rz_sum += rz2;
          const int sn = s + nst * nwarps;
          if (sn < c1) {
            if (lane == 0) stage_issue(a, sn, stage_buf + (uint32_t)(b * kClStageBytes), stage_bar + 8u * b);
            pending |= 1u << b;
          }
        }
        if (!ok) {
          // the copies still in flight land before the warp leaves (bounded again); the CTA stops after the
          // reduction below and the error word makes the host return SDX_ERR_DEVICE_TIMEOUT
          for (int b = 0; b < nst; ++b)
            if (pending & (1u << b)) stage_wait(stage_bar + 8u * b, (ph >> b) & 1u, a.spin_limit);
          if (lane == 0) {
            atomicExch(err, 1u);
            s_stage_fail = 1;
          }
        }
        acc_add(0, rr_sum);
        acc_add(1, rzo_sum);
        acc_add(2, rz_sum);
      } else if (a.precond != 2) {
        double rr_sum = 0.0, rzo_sum = 0.0, rz_sum = 0.0;  // this lane's sums over the warp's slices
        const int ahead = a.prefetch;  // prefetch distance in this warp's slices (as in k_pcg)
        for (int k = 0; k < ahead && c0 + warp + k * nwarps < c1; ++k)
          prefetch_update_operands(a, c0 + warp + k * nwarps, lane);
        for (int s = c0 + warp; s < c1; s += nwarps) {
          if (ahead > 0 && s + ahead * nwarps < c1) prefetch_update_operands(a, s + ahead * nwarps, lane);
          const int64_t d0 = (int64_t)s * (3 * kSlice);
          if (replace) {  // only x (and its folded increment): the true residual that follows recomputes r, z
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const int64_t d = d0 + lane + 32 * j;
              const double inc = a.r_in_z ? (double)a.xi[d] : 0.0;
              a.x[d] += inc + al * (double)a.p[d];
              if (a.r_in_z) a.xi[d] = 0.0f;
            }
            continue;
          }
          // r carried by z (r = z / d) and x by its FP32 increment between true-residual replacements with
          // r_in_z; old z as whole float4 rows through the warp's staging row (as in k_pcg)
          double xo[3] = {0.0, 0.0, 0.0}, ro[3] = {0.0, 0.0, 0.0};
          float xio[3] = {0.0f, 0.0f, 0.0f};
          float pp[3], qq[3], dd[3], zo[3];
          const float4 zrow = a.z[(int64_t)s * kSlice + lane];
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int dl = lane + 32 * j;
            if (a.r_in_z) {
              xio[j] = a.xi[d0 + dl];
            } else {
              xo[j] = a.x[d0 + dl];
              ro[j] = a.r[d0 + dl];
            }
            pp[j] = a.p[d0 + dl];
            qq[j] = a.q[d0 + dl];
            dd[j] = a.precond == 1 ? a.dinv[d0 + dl] : 1.0f;
          }
          tr[3 * lane] = zrow.x;
          tr[3 * lane + 1] = zrow.y;
          tr[3 * lane + 2] = zrow.z;
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 3; ++j) zo[j] = tr[lane + 32 * j];
          __syncwarp();
          double rr2 = 0.0, rzo2 = 0.0, rz2 = 0.0;
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int dl = lane + 32 * j;
            if (a.r_in_z)
              a.xi[d0 + dl] = (float)((double)xio[j] + al * (double)pp[j]);
            else
              a.x[d0 + dl] = xo[j] + al * (double)pp[j];
            const double rp =
                !a.r_in_z ? ro[j] : (a.precond == 1 ? (double)(zo[j] / dd[j]) : (double)zo[j]);
            const double r = rp - al * (double)qq[j];
            if (!a.r_in_z) a.r[d0 + dl] = r;
            const float z = (float)(dd[j] * r);
            tr[dl] = z;
            rr2 += r * r;
            rzo2 += r * zo[j];
            rz2 += r * z;
          }
          __syncwarp();
          a.z[(int64_t)s * kSlice + lane] = make_float4(tr[3 * lane], tr[3 * lane + 1], tr[3 * lane + 2], 0.0f);
          __syncwarp();
          rr_sum += rr2;
          rzo_sum += rzo2;
          rz_sum += rz2;
        }
        acc_add(0, rr_sum);
        acc_add(1, rzo_sum);
        acc_add(2, rz_sum);
      } else {
        for (int s = c0 + warp; s < c1; s += nwarps) {
          const int64_t row = (int64_t)s * kSlice + lane;
          double xo[3], ro[3];
          float pp[3], qq[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            xo[k] = a.x[3 * row + k];
            pp[k] = a.p[3 * row + k];
            ro[k] = a.r[3 * row + k];
            qq[k] = a.q[3 * row + k];
          }
          const float4 zo = replace ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : a.z[row];
          double r[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            a.x[3 * row + k] = xo[k] + al * (double)pp[k];
            r[k] = ro[k] - al * (double)qq[k];
          }
          if (replace) continue;
          float z[3];
          prec_apply(a, row, r, z);
#pragma unroll
          for (int k = 0; k < 3; ++k) a.r[3 * row + k] = r[k];
          a.z[row] = make_float4(z[0], z[1], z[2], 0.0f);
          acc_add(0, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
          acc_add(1, r[0] * zo.x + r[1] * zo.y + r[2] * zo.z);
          acc_add(2, r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
        }
      }
      if (replace) {
        // true residual in FP64 (needs the neighbours' x updates)
        if (!cluster_sync(cnt, csize, a.spin_limit, err, &s_ok)) {
          fail = true;
          break;
        }
        for (int s = c0 + warp; s < c1; s += nwarps) {
          const int64_t row = (int64_t)s * kSlice + lane;
          double r[3];
          true_residual<4>(a, s, lane, r);
          const float4 zo = a.z[row];
          float z[3];
          prec_apply(a, row, r, z);
#pragma unroll
          for (int k = 0; k < 3; ++k) a.r[3 * row + k] = r[k];
          a.z[row] = make_float4(z[0], z[1], z[2], 0.0f);
          acc_add(0, r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
          acc_add(1, r[0] * zo.x + r[1] * zo.y + r[2] * zo.z);
          acc_add(2, r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
        }
      }
      if (!reduce(3)) {
        fail = true;
        break;
      }
      if (s_stage_fail) {  // read after the reduction's barriers: the same verdict in every thread of the CTA
        fail = true;
        break;
      }
      it_done = it;
      rr = s_tot[0];
      const double rzo = s_tot[1], rzn = s_tot[2];
      if (!isfinite(rr) || rr > div_thr) {
        status = 3;
        break;
      }
      if (rr <= conv_thr) {
        if (replace) {
          status = 1;
          break;
        }
        verify_it = it;
      }
      if (it >= a.max_iter) {
        status = 2;
        break;
      }
      if (rzn == 0.0) {
        status = 3;
        break;
      }
      const double bpr = (a.polak_ribiere && !first) ? rzo : 0.0;
      beta = (rzn - bpr) / rz;
      rz = rzn;
      first = false;
    }
    if (fail) break;
    // this CTA's rows of the env: the x increment since the last replacement into x
    if (a.r_in_z && a.precond != 2)
      for (int s = c0 + warp; s < c1; s += nwarps) fold_x_increment(a, s, lane);
    if (rank == 0 && threadIdx.x == 0) {
      a.out_iters[e] = it_done;
      a.out_res[e] = sqrt(fmax(rr, 0.0));
      a.out_relres[e] = bb == 0.0 ? 0.0 : sqrt(fmax(rr, 0.0) / bb);
      a.out_conv[e] = status;
    }
  }
  cluster_hw_sync();  // no CTA leaves while another may still read its shared memory
}

// The pipelined variant runs at 512 threads per CTA or fewer (SDX_PCG_PIPE=0 selects the batched one).
static bool pcg_pipelined(int threads) {
  static const int pipe = [] {
    const char* e = getenv("SDX_PCG_PIPE");
    return e ? atoi(e) : 1;
  }();
  return pipe != 0 && threads <= 512;
}

int pcg_max_ctas_per_sm(int threads) {
  int n = 0;
  for (const void* fn : {(const void*)k_pcg<true, false>, (const void*)k_pcg<false, false>,
                         (const void*)k_pcg<true, true>, (const void*)k_pcg<false, true>})
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, pcg_shared_bytes(1024));
  const cudaError_t e =
      pcg_pipelined(threads)
          ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pcg<true, false>, threads, pcg_shared_bytes(threads))
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pcg<false, false>, threads, pcg_shared_bytes(threads));
  return e == cudaSuccess ? n : 0;
}

int pcg_shared_bytes(int threads, int wstride) { return (threads / 32) * wstride * kPcgNq * (int)sizeof(double); }

// Cluster shapes for k_pcg_cluster (one 512-thread CTA per SM): how many clusters of 16, 8, 4 and 2 CTAs
// are co-resident on this device (occupancy queries, once).
static const int kClSizes[4] = {16, 8, 4, 2};
static const int* pcg_cluster_counts(int* last_error) {
  static int err = 0;
  static const std::array<int, 4> counts = [] {
    std::array<int, 4> n{0, 0, 0, 0};
    cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, cl_dyn_smem(kClMaxStages));
    for (int i = 0; i < 4; ++i) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = kClSizes[i];
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(kClSizes[i]);
      cfg.blockDim = dim3(512);
      cfg.dynamicSmemBytes = cl_dyn_smem(kClMaxStages);  // the largest staging the launches use
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      const cudaError_t e = cudaOccupancyMaxActiveClusters(&n[i], k_pcg_cluster, &cfg);
      if (e != cudaSuccess) {
        cudaGetLastError();
        n[i] = 0;
        err = (int)e;
      }
    }
    return n;
  }();
  if (last_error) *last_error = err;
  return counts.data();
}

// The shape for a queue of n_envs envs: the cluster size that keeps the most SMs busy with min(n_envs,
// co-resident clusters) clusters, ties to the larger clusters (an env's iterations are latency bound
// well before its rows fill a cluster; on the 1,024-body batch 37 x 4 beats 74 x 2 by 3 %).
// SDX_PCG_CLUSTER_SIZE=16/8/4/2 forces a size.
ClusterShape pcg_cluster_shape(int n_envs, int want_size) {
  int err = 0;
  const int* counts = pcg_cluster_counts(&err);
  const char* force = getenv("SDX_PCG_CLUSTER_SIZE");
  const int want = force ? atoi(force) : want_size;
  ClusterShape best{0, 0, err};
  int best_busy = 0;
  for (int i = 0; i < 4; ++i) {
    const int cs = kClSizes[i], n = std::min(counts[i], std::max(1, n_envs));
    if (counts[i] <= 0 || (want > 0 && cs != want)) continue;
    const int busy = n * cs;
    if (busy > best_busy) {  // sizes are tried largest first, so a tie keeps the larger
      best_busy = busy;
      best = ClusterShape{n, cs, err};
    }
  }
  return best;
}

cudaError_t launch_pcg_cluster(const PcgArgs& a, ClusterShape shape, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = shape.size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(shape.n_clusters * shape.size);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = (size_t)cl_dyn_smem(std::max(0, std::min(kClMaxStages, a.stage_update)));
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_pcg_cluster, a);
}

cudaError_t launch_pcg(const PcgArgs& a, int n_cta, int threads, cudaStream_t st) {
  PcgArgs args = a;
  args.wstride = (a.wstride > 0 && a.wstride < kPcgMaxEnvsPerCta) ? a.wstride : kPcgMaxEnvsPerCta;
  void* params[] = {&args};
  const bool timed = a.cta_ns != nullptr;
  const void* fn = pcg_pipelined(threads)
                       ? (timed ? (const void*)k_pcg<true, true> : (const void*)k_pcg<true, false>)
                       : (timed ? (const void*)k_pcg<false, true> : (const void*)k_pcg<false, false>);
  return cudaLaunchCooperativeKernel(fn, dim3(n_cta), dim3(threads), params,
                                     (size_t)pcg_shared_bytes(threads, args.wstride), st);
}

// The same launch through cudaLaunchKernelEx with the cooperative attribute, the form a graph's kernel
// node records (steps captured into a CUDA graph); no per-CTA timers.
cudaError_t launch_pcg_captured(const PcgArgs& a, int n_cta, int threads, cudaStream_t st) {
  PcgArgs args = a;
  args.wstride = (a.wstride > 0 && a.wstride < kPcgMaxEnvsPerCta) ? a.wstride : kPcgMaxEnvsPerCta;
  args.cta_ns = nullptr;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n_cta);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = (size_t)pcg_shared_bytes(threads, args.wstride);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return pcg_pipelined(threads) ? cudaLaunchKernelEx(&cfg, k_pcg<true, false>, args)
                                : cudaLaunchKernelEx(&cfg, k_pcg<false, false>, args);
}

}  // namespace sdx

