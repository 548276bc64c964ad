// Device code of the batched SQP solver: per-instance context, linearization, Schur assembly,
// the PCG variants, recovery, line search, and the forward / adjoint / rollout kernels.
// Included by k_sqp.cu, which is compiled once per launch configuration (DMPC_CFG).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "dual.cuh"
#include "layout.cuh"
#include "models.cuh"

namespace dmpc_impl {
namespace {
// ---------------------------------------------------------------- instance context
struct Inst {
  int model, nx, nu, N, K, scheme, pen, P, ld;
  double dt;
  const double *x0, *xf, *xref, *uref, *wx, *wu, *wf, *mp;
  double *A, *Bm, *C, *Qi, *Ri, *q, *r, *gam, *lam, *res, *t1, *xb, *ub, *xn, *un, *fv;
  double *th, *ph, *ti, *pm, *tmp, *li, *contrib;
  float* w32;  // scaled-basis off-diagonal blocks W_t (FP32, row stride ld)
};

// the kernels' dynamic shared memory, visible to device functions: pointers rebuilt
// from it let the compiler use shared-space loads instead of generic ones
extern __shared__ __align__(16) unsigned char g_dyn_smem[];

// g is the group's descriptor: G.g, or a view of it whose inputs/outputs point at one
// step of a closed-loop rollout.  `slot` is this CTA's workspace slot (not the instance's).
__device__ inline Inst make_inst(const DevGroup& G, const dmpc_group& g, int i, void* slot, float* smem_blocks) {
  Inst s;
  s.model = g.model;
  s.nx = g.nx;
  s.nu = g.nu;
  s.N = g.horizons ? g.horizons[i] : g.horizon;
  s.K = s.N + 1;
  s.scheme = g.scheme;
  s.pen = g.penalize_control_reference;
  s.P = g.n_model_params;
  s.ld = G.ld32;
  s.dt = g.dt[i];
  const int nx = g.nx, nu = g.nu, Kmax = G.K;
  s.x0 = g.initial_state + (size_t)i * nx;
  s.xf = g.final_state + (size_t)i * nx;
  s.xref = g.reference_state + (size_t)i * Kmax * nx;
  s.uref = g.reference_control + (size_t)i * Kmax * nu;
  s.wx = g.w_x + (size_t)i * nx;
  s.wu = g.w_u + (size_t)i * nu;
  s.wf = g.w_f + (size_t)i * nx;
  s.mp = g.model_params + (size_t)i * g.n_model_params;
  Layout L = make_layout(nx, nu, g.horizon, G.ld32, G.blocks_smem != 1, g.n_model_params);
  double* base = reinterpret_cast<double*>(slot);
  s.A = base + L.A;
  s.Bm = base + L.Bm;
  s.C = base + L.C;
  s.Qi = base + L.Qi;
  s.Ri = base + L.Ri;
  s.q = base + L.q;
  s.r = base + L.r;
  s.gam = base + L.gam;
  s.lam = base + L.lam;
  s.res = base + L.res;
  s.t1 = base + L.t1;
  s.xb = base + L.xb;
  s.ub = base + L.ub;
  s.xn = base + L.xn;
  s.un = base + L.un;
  s.fv = base + L.fv;
  s.th = base + L.th;
  s.ph = base + L.ph;
  s.ti = base + L.ti;
  s.pm = base + L.pm;
  s.tmp = base + L.tmp;
  s.li = base + L.li;
  s.contrib = base + L.contrib;
  const bool use_smem = G.blocks_smem == 1 ||
                        (G.blocks_smem == 2 && (uint64_t)s.K * nx * s.ld * sizeof(float) <= G.smem_block_budget);
  s.w32 = use_smem ? smem_blocks : reinterpret_cast<float*>(base + L.n_doubles);
  // the row PCG reads the FP64 W blocks at every residual replacement: keep them in
  // shared memory when the launch reserved room for them
  if (G.w64_off) s.pm = reinterpret_cast<double*>(g_dyn_smem + G.w64_off);
  return s;
}

// Linear model: integrator with the parameter matrices read from global memory.
// Parameter `pk` (or -1) carries the hyper-dual e2 direction.
template <class T>
__device__ __forceinline__ T pcoef(double v, bool hit) {
  return T(v);
}
template <>
__device__ __forceinline__ HDual pcoef<HDual>(double v, bool hit) {
  return HDual(v, 0.0, hit ? 1.0 : 0.0, 0.0);
}

template <class T>
__device__ void linear_state_dot_mem(const Inst& s, const T* x, const T* u, T* xd, int pk) {
  const int nx = s.nx, nu = s.nu;
  const double* A = s.mp;
  const double* B = A + nx * nx;
  const double* b = B + nx * nu;
  for (int i = 0; i < nx; ++i) {
    T a = 0.0;
    for (int j = 0; j < nx; ++j) a = a + pcoef<T>(A[i * nx + j], pk == i * nx + j) * x[j];
    T c = 0.0;
    for (int j = 0; j < nu; ++j) c = c + pcoef<T>(B[i * nu + j], pk == nx * nx + i * nu + j) * u[j];
    xd[i] = a + c + pcoef<T>(b[i], pk == nx * nx + nx * nu + i);
  }
}

template <class T>
__device__ void predict_next_state_linear(const Inst& s, const T* x, const T* u, T* xn, int pk = -1) {
  constexpr int MX = DMPC_MAX_NX;
  const int nx = s.nx;
  const double dt = s.dt;
  T k[MX], tmp[MX], acc[MX];
  linear_state_dot_mem(s, x, u, k, pk);
  for (int i = 0; i < nx; ++i) xn[i] = x[i] + dt * k[i];
  if (s.scheme == DMPC_MIDPOINT) {
    for (int i = 0; i < nx; ++i) tmp[i] = x[i] + 0.5 * dt * k[i];
    linear_state_dot_mem(s, tmp, u, acc, pk);
    for (int i = 0; i < nx; ++i) xn[i] = x[i] + dt * acc[i];
  } else if (s.scheme == DMPC_RK4) {
    for (int i = 0; i < nx; ++i) {
      acc[i] = k[i];
      tmp[i] = x[i] + 0.5 * dt * k[i];
    }
    linear_state_dot_mem(s, tmp, u, k, pk);
    for (int i = 0; i < nx; ++i) {
      acc[i] = acc[i] + 2.0 * k[i];
      tmp[i] = x[i] + 0.5 * dt * k[i];
    }
    linear_state_dot_mem(s, tmp, u, k, pk);
    for (int i = 0; i < nx; ++i) {
      acc[i] = acc[i] + 2.0 * k[i];
      tmp[i] = x[i] + dt * k[i];
    }
    linear_state_dot_mem(s, tmp, u, k, pk);
    for (int i = 0; i < nx; ++i) xn[i] = x[i] + ((1.0 / 6.0) * (acc[i] + k[i])) * dt;
  }
}

// ---------------------------------------------------------------- linearization
// One work item = (stage t, direction d): a Dual evaluation of the integrator
// gives column d of [A_t | B_t] (value_and_jacfwd, jax_utils.py:12-36).
template <int MODEL>
__device__ __noinline__ void linearize_item(const Inst& s, const double* xb, const double* ub, int t, int d) {
  constexpr int MX = ModelDims<MODEL>::NX, MU = ModelDims<MODEL>::NU;
  // fixed-size models have (nx, nu) == (MX, MU): compile-time trip counts keep the
  // dual arrays in registers
  const int nx = MODEL == DMPC_MODEL_LINEAR ? s.nx : MX, nu = MODEL == DMPC_MODEL_LINEAR ? s.nu : MU;
  Dual x[MX], u[MU], xn[MX];
  for (int j = 0; j < nx; ++j) x[j] = Dual(xb[t * nx + j], j == d ? 1.0 : 0.0);
  for (int j = 0; j < nu; ++j) u[j] = Dual(ub[t * nu + j], nx + j == d ? 1.0 : 0.0);
  if (MODEL == DMPC_MODEL_LINEAR) {
    // parameters as constants: read straight from memory to keep registers low
    predict_next_state_linear(s, x, u, xn);
  } else {
    Dual p[12];  // compile-time trip count keeps p in registers; unused slots are zero
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = Dual(k < s.P ? s.mp[k] : 0.0);
    predict_next_state<Dual, MODEL>(s.scheme, s.dt, nx, nu, x, u, p, xn);
  }
  if (d < nx) {
    for (int i = 0; i < nx; ++i) s.A[((size_t)t * nx + i) * nx + d] = xn[i].d;
  } else {
    for (int i = 0; i < nx; ++i) s.Bm[((size_t)t * nx + i) * nu + (d - nx)] = xn[i].d;
  }
  if (d == 0)
    for (int i = 0; i < nx; ++i) s.fv[t * nx + i] = xn[i].v;
}

// Plain FP64 integrator step for one stage (line search, constraint values).
__device__ __noinline__ void next_state_value(const Inst& s, const double* x, const double* u, double* xn) {
  switch (s.model) {
    case DMPC_MODEL_LINEAR: predict_next_state_linear<double>(s, x, u, xn); break;
    case DMPC_MODEL_QUADROTOR: predict_next_state<double, DMPC_MODEL_QUADROTOR>(s.scheme, s.dt, s.nx, s.nu, x, u, s.mp, xn); break;
    case DMPC_MODEL_SPACECRAFT: predict_next_state<double, DMPC_MODEL_SPACECRAFT>(s.scheme, s.dt, s.nx, s.nu, x, u, s.mp, xn); break;
    case DMPC_MODEL_ATTITUDE: predict_next_state<double, DMPC_MODEL_ATTITUDE>(s.scheme, s.dt, s.nx, s.nu, x, u, s.mp, xn); break;
    case DMPC_MODEL_CARTPOLE: predict_next_state<double, DMPC_MODEL_CARTPOLE>(s.scheme, s.dt, s.nx, s.nu, x, u, s.mp, xn); break;
  }
}

// A_t, B_t, f(x_t, u_t) for t < N, then C = [x0; -f + A x + B u]
// (optimal_control_problem.py:325-398).  As_next = -I is implicit.
__device__ __noinline__ void linearize_dynamics(const Inst& s, const double* xb, const double* ub) {
  const int nd = s.nx + s.nu;
  const int items = s.N * nd;
  for (int w = threadIdx.x; w < items; w += blockDim.x) {
    const int t = w / nd, d = w - t * nd;
    switch (s.model) {
      case DMPC_MODEL_LINEAR: linearize_item<DMPC_MODEL_LINEAR>(s, xb, ub, t, d); break;
      case DMPC_MODEL_QUADROTOR: linearize_item<DMPC_MODEL_QUADROTOR>(s, xb, ub, t, d); break;
      case DMPC_MODEL_SPACECRAFT: linearize_item<DMPC_MODEL_SPACECRAFT>(s, xb, ub, t, d); break;
      case DMPC_MODEL_ATTITUDE: linearize_item<DMPC_MODEL_ATTITUDE>(s, xb, ub, t, d); break;
      case DMPC_MODEL_CARTPOLE: linearize_item<DMPC_MODEL_CARTPOLE>(s, xb, ub, t, d); break;
    }
  }
  __syncthreads();
  const int nx = s.nx, nu = s.nu;
  for (int w = threadIdx.x; w < s.K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    if (t == 0) {
      s.C[i] = s.x0[i];
    } else {
      const int k = t - 1;
      const double* Ar = s.A + ((size_t)k * nx + i) * nx;
      const double* Br = s.Bm + ((size_t)k * nx + i) * nu;
      double a = 0.0, b = 0.0;
      for (int j = 0; j < nx; ++j) a += Ar[j] * xb[k * nx + j];
      for (int j = 0; j < nu; ++j) b += Br[j] * ub[k * nu + j];
      s.C[w] = -s.fv[k * nx + i] + a + b;
    }
  }
}

// Diagonal cost blocks (optimal_control_problem.py:249-323, sqp.py:160-197,243-244).
// The Hessian of the weighted-square cost is 2 diag(w); PSD projection clamps its
// eigenvalues at 1e-9 and q = J - x^T H uses the unprojected H.
__device__ void linearize_cost(const Inst& s, const double* xb, const double* ub) {
  const int nx = s.nx, nu = s.nu, N = s.N;
  for (int w = threadIdx.x; w < s.K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    double h, ref;
    if (t < N) {
      h = 2.0 * s.wx[i];
      ref = s.xref[t * nx + i];
    } else {
      h = 2.0 * (s.wx[i] + s.wf[i]);
      ref = s.xf[i];
    }
    const double x = xb[w];
    const double J = h * (x - ref);
    s.q[w] = J - x * h;
    s.Qi[w] = 1.0 / fmax(h, 1e-9);
  }
  for (int w = threadIdx.x; w < N * nu; w += blockDim.x) {
    const int t = w / nu, i = w - t * nu;
    const double h = 2.0 * s.wu[i];
    const double ref = s.pen ? s.uref[t * nu + i] : 0.0;
    const double u = ub[w];
    const double J = h * (u - ref);
    s.r[w] = J - u * h;
    s.Ri[w] = 1.0 / fmax(h, 1e-9);
  }
}

// ---------------------------------------------------------------- Schur assembly
// theta_0 = Q0^-1; theta_{t+1} = A_t Q_t^-1 A_t^T + B_t R_t^-1 B_t^T + Q_{t+1}^-1;
// phi_t = A_t Q_t^-1 An_{t-1}^T with An_{-1} = I, An = -I (pcg.py:182-196);
// theta^-1 in FP64; P_t = -theta_t^-1 phi_{t-1} theta_{t-1}^-1 (pcg.py:213-239).
// Writes FP64 blocks th/ph/ti/pm (row stride nx) and, for the mixed precision
// path, the scaled-basis blocks li (FP64) and w32 (FP32, row stride ld).
// Set when a theta block has no Cholesky factor in FP64; the QP solve then runs the
// FP64 recurrence instead of the scaled FP32 iterations.
__shared__ int sh_scaled_bad;

// Li_t = L_t^-1 for every knot (theta_t = L_t L_t^T, FP64): in registers by groups of 16
// lanes per block for the nx with a row PCG, else one warp per block in the workspace (tmp as the
// factorisation's working copy).  Sets sh_scaled_bad if a block has no factor.
template <int NX>
__device__ __noinline__ bool scaled_factors_regs(const Inst& s) {
  constexpr int nn = NX * NX;
  constexpr int W = NX <= 16 ? 16 : 32;  // lanes per block
  constexpr int G = 32 / W;              // blocks per warp at a time
  const int gid = (threadIdx.x >> 5) * G + ((threadIdx.x & 31) / W);
  const int ng = (blockDim.x >> 5) * G;
  bool ok = true;
  for (int base = 0; base < s.K; base += ng) {  // warp-uniform rounds
    const int t = base + gid;
    const bool active = t < s.K;
    const size_t o = (size_t)(active ? t : 0) * nn;
    ok = group_chol_inverse_regs<NX, W>(s.th + o, s.li + o, active) && ok;
  }
  return ok;
}

__device__ void scaled_factors(const Inst& s) {
  const int nx = s.nx, nn = nx * nx, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) sh_scaled_bad = 0;
  __syncthreads();
  bool ok = true;
  switch (nx) {
    case 3: ok = scaled_factors_regs<3>(s); break;
    case 4: ok = scaled_factors_regs<4>(s); break;
    case 6: ok = scaled_factors_regs<6>(s); break;
    case 7: ok = scaled_factors_regs<7>(s); break;
    case 8: ok = scaled_factors_regs<8>(s); break;
    case 12: ok = scaled_factors_regs<12>(s); break;
    case 13: ok = scaled_factors_regs<13>(s); break;
    default:
      for (int t = threadIdx.x >> 5; t < s.K; t += blockDim.x >> 5) {
        double* Lt = s.tmp + (size_t)t * nn;
        for (int e = lane; e < nn; e += 32) Lt[e] = s.th[(size_t)t * nn + e];
        __syncwarp();
        ok = warp_chol_inverse(Lt, s.li + (size_t)t * nn, nx) && ok;
      }
  }
  if (!ok && lane == 0) sh_scaled_bad = 1;
}

// NXT > 0: compile-time nx, so every inner product is unrolled and its loads (of blocks
// that live in L2) issue together; the triangular factors store exact zeros above the
// diagonal, so those products run over the full range.
template <int NXT>
__device__ __noinline__ void assemble_schur_t(const Inst& s, bool fp32_copy) {
  const int nx = NXT > 0 ? NXT : s.nx, nu = s.nu, N = s.N, K = s.K;
  const int nn = nx * nx;
  for (int w = threadIdx.x; w < K * nn; w += blockDim.x) {
    const int t = w / nn, e = w - t * nn, i = e / nx, j = e - i * nx;
    double v;
    if (t == 0) {
      v = (i == j) ? s.Qi[i] : 0.0;
    } else {
      const int k = t - 1;
      const double* Ai = s.A + ((size_t)k * nx + i) * nx;
      const double* Aj = s.A + ((size_t)k * nx + j) * nx;
      const double* Bi = s.Bm + ((size_t)k * nx + i) * nu;
      const double* Bj = s.Bm + ((size_t)k * nx + j) * nu;
      const double* D = s.Qi + k * nx;
      const double* E = s.Ri + k * nu;
      double a = 0.0, b = 0.0;
#pragma unroll
      for (int l = 0; l < nx; ++l) a += Ai[l] * D[l] * Aj[l];
      for (int l = 0; l < nu; ++l) b += Bi[l] * E[l] * Bj[l];
      v = a + b + ((i == j) ? s.Qi[t * nx + i] : 0.0);
    }
    s.th[w] = v;
    if (!fp32_copy) s.tmp[w] = v;  // working copy for the in-place Gauss-Jordan inverse
    if (t < N) {
      // phi_t = A_t D_t An_{t-1}^T : t == 0 -> A_0 D_0; t >= 1 -> -A_t D_t
      const double ph = s.A[((size_t)t * nx + i) * nx + j] * s.Qi[t * nx + j];
      s.ph[(size_t)t * nn + e] = (t == 0) ? ph : -ph;
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  if (!fp32_copy) {
    for (int t = warp; t < K; t += nwarp) warp_spd_inverse(s.tmp + (size_t)t * nn, s.ti + (size_t)t * nn, nx);
  } else {
    // Li_t = L_t^-1 with theta_t = L_t L_t^T.  The mixed path needs no theta^-1 or P: its
    // FP64 residual and fallback work in the scaled basis.  Without a factor (a theta block
    // that is not numerically SPD) it falls back to the reference recurrence, which needs them.
    scaled_factors(s);
    __syncthreads();
    if (sh_scaled_bad) {
      for (int t = warp; t < K; t += nwarp) {
        double* Lt = s.tmp + (size_t)t * nn;
        for (int e = (threadIdx.x & 31); e < nn; e += 32) Lt[e] = s.th[(size_t)t * nn + e];
        __syncwarp();
        warp_spd_inverse(Lt, s.ti + (size_t)t * nn, nx);
      }
    }
  }
  __syncthreads();
  // reference-basis Phi^-1 blocks (pcg.py:213-239): the FP64 path, or the mixed path without
  // Cholesky factors
  if (!fp32_copy || sh_scaled_bad) {
    // T_t = theta_t^-1 phi_{t-1}  (t = 1..N), stored in tmp block t
    for (int w = threadIdx.x; w < N * nn; w += blockDim.x) {
      const int k = w / nn, e = w - k * nn, i = e / nx, j = e - i * nx;
      const int t = k + 1;
      const double* Ti = s.ti + (size_t)t * nn + i * nx;
      const double* Pk = s.ph + (size_t)k * nn + j;
      double a = 0.0;
#pragma unroll
      for (int l = 0; l < nx; ++l) a += Ti[l] * Pk[l * nx];
      s.tmp[(size_t)t * nn + e] = a;
    }
    __syncthreads();
    // P_t = -T_t theta_{t-1}^-1, stored at index t-1
    for (int w = threadIdx.x; w < N * nn; w += blockDim.x) {
      const int k = w / nn, e = w - k * nn, i = e / nx, j = e - i * nx;
      const int t = k + 1;
      const double* Tr = s.tmp + (size_t)t * nn + i * nx;
      const double* Tm = s.ti + (size_t)k * nn + j;
      double a = 0.0;
#pragma unroll
      for (int l = 0; l < nx; ++l) a += Tr[l] * Tm[l * nx];
      s.pm[(size_t)k * nn + e] = -a;
    }
  }
  if (fp32_copy && !sh_scaled_bad) {
    // scaled basis: W_t = Li_t phi_{t-1} Li_{t-1}^T (t = 1..N) at block t-1, block N zero, in
    // FP32 (w32, row stride ld) for the FP32 iterations and in FP64 (pm, row stride nx) for
    // the FP64 residual and fallback
    __syncthreads();
    // T_t = Li_t phi_{t-1} (t = 1..N) in tmp block t
    for (int w = threadIdx.x; w < N * nn; w += blockDim.x) {
      const int k = w / nn, e = w - k * nn, i = e / nx, j = e - i * nx;
      const double* Lr = s.li + (size_t)(k + 1) * nn + i * nx;
      const double* Pk = s.ph + (size_t)k * nn + j;
      double a = 0.0;
#pragma unroll
      for (int l = 0; l < nx; ++l) a += Lr[l] * Pk[l * nx];
      s.tmp[(size_t)(k + 1) * nn + e] = a;
    }
    __syncthreads();
    const int ld = s.ld;
    const int nl = nx * ld;
    for (int w = threadIdx.x; w < K * nl; w += blockDim.x) {
      const int k = w / nl, e = w - k * nl, i = e / ld, j = e - i * ld;
      double v = 0.0;
      if (j < nx && k < N) {
        const double* Tr = s.tmp + (size_t)(k + 1) * nn + i * nx;
        const double* Lm = s.li + (size_t)k * nn + j * nx;  // (Li_{t-1}^T)[l][j] = Li_{t-1}[j][l]
#pragma unroll
        for (int l = 0; l < nx; ++l) v += Tr[l] * Lm[l];
      }
      s.w32[w] = (float)v;
      if (j < nx) s.pm[(size_t)k * nn + i * nx + j] = v;
    }
  }
  __syncthreads();
}

__device__ void assemble_schur(const Inst& s, bool fp32_copy) {
  switch (s.nx) {
    case 3: assemble_schur_t<3>(s, fp32_copy); break;
    case 4: assemble_schur_t<4>(s, fp32_copy); break;
    case 6: assemble_schur_t<6>(s, fp32_copy); break;
    case 7: assemble_schur_t<7>(s, fp32_copy); break;
    case 8: assemble_schur_t<8>(s, fp32_copy); break;
    case 12: assemble_schur_t<12>(s, fp32_copy); break;
    case 13: assemble_schur_t<13>(s, fp32_copy); break;
    default: assemble_schur_t<0>(s, fp32_copy);
  }
}

// gamma = C + [Q0^-1 q0; A Q^-1 q + B R^-1 r + An Q_next^-1 q_next] (pcg.py:245-288),
// with C == NULL meaning zeros (the adjoint, sqp.py:694-700).
__device__ void compute_gamma(const Inst& s, const double* C, const double* q, const double* r) {
  const int nx = s.nx, nu = s.nu;
  for (int w = threadIdx.x; w < s.K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    double g;
    if (t == 0) {
      g = s.Qi[i] * q[i];
    } else {
      const int k = t - 1;
      const double* Ar = s.A + ((size_t)k * nx + i) * nx;
      const double* Br = s.Bm + ((size_t)k * nx + i) * nu;
      double a = 0.0, b = 0.0;
      for (int j = 0; j < nx; ++j) a += Ar[j] * (s.Qi[k * nx + j] * q[k * nx + j]);
      for (int j = 0; j < nu; ++j) b += Br[j] * (s.Ri[k * nu + j] * r[k * nu + j]);
      g = a + b - s.Qi[w] * q[w];
    }
    s.gam[w] = (C ? C[w] : 0.0) + g;
  }
}

// CTA-wide sum: warp tree, one barrier, then every warp reduces the per-warp
// partials with the same shuffle tree (identical result in every thread).
__device__ __forceinline__ double block_sum2(double v, double* red, int& parity) {
  v = warp_sum(v);
  double* buf = red + (parity << 6);
  const int lane = threadIdx.x & 31;
  if (lane == 0) buf[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = (lane < (int)(blockDim.x >> 5)) ? buf[lane] : 0.0;
  parity ^= 1;
  return warp_sum(s);
}

// ---------------------------------------------------------------- compile-time-nx stencil
// FP64 blocks (workspace, row stride NX), dense vectors v[t*NX + j]
template <int NX>
__device__ __forceinline__ double stencil64(const double* __restrict__ Dg, const double* __restrict__ Off,
                                            const double* __restrict__ v, int t, int i, int N) {
  constexpr int BS = NX * NX;
  double a0 = 0.0, a1 = 0.0;
  const double* m = Dg + t * BS + i * NX;
  const double* x = v + t * NX;
#pragma unroll
  for (int j = 0; j < NX; ++j) a0 = fma(m[j], x[j], a0);
  if (t > 0) {
    const double* mo = Off + (t - 1) * BS + i * NX;
    const double* xo = v + (t - 1) * NX;
#pragma unroll
    for (int j = 0; j < NX; ++j) a1 = fma(mo[j], xo[j], a1);
  }
  if (t < N) {
    const double* c = Off + t * BS + i;
    const double* xp = v + (t + 1) * NX;
#pragma unroll
    for (int j = 0; j < NX; ++j) a0 = fma(c[j * NX], xp[j], a0);
  }
  return a0 + a1;
}

// ---------------------------------------------------------------- block-tridiagonal stencil
// y_t = Off_{t-1} v_{t-1} + Dg_t v_t + Off_t^T v_{t+1}  for row (t, i) = g.
template <class BT, class VT>
__device__ __forceinline__ double stencil_row(const BT* Dg, const BT* Off, int ld, int nx, int N, const VT* v, int g) {
  const int t = g / nx, i = g - t * nx;
  const size_t bs = (size_t)nx * ld;
  double acc;
  {
    const BT* row = Dg + t * bs + (size_t)i * ld;
    const VT* vt = v + t * nx;
    VT a = 0;
    for (int j = 0; j < nx; ++j) a += (VT)row[j] * vt[j];
    acc = (double)a;
  }
  if (t > 0) {
    const BT* row = Off + (t - 1) * bs + (size_t)i * ld;
    const VT* vm = v + (t - 1) * nx;
    VT a = 0;
    for (int j = 0; j < nx; ++j) a += (VT)row[j] * vm[j];
    acc += (double)a;
  }
  if (t < N) {
    const BT* col = Off + t * bs + i;
    const VT* vp = v + (t + 1) * nx;
    VT a = 0;
    for (int j = 0; j < nx; ++j) a += (VT)col[(size_t)j * ld] * vp[j];
    acc += (double)a;
  }
  return acc;
}

// ---------------------------------------------------------------- PCG, FP64 (reference recurrence)
struct PcgOut {
  int it;     // iterations (FP32 and FP64)
  double eta;
  int nrep;   // FP64 residual replacements of the FP32 PCG
  int it64;   // iterations of the FP64 recurrence
};

// Solves S lam = gam starting from lam (in/out, FP64 shared vector `lv`),
// pcg.py:350-436: r = gamma - S lam; rt = Phi^-1 r; p = rt; eta = r.rt; loop while
// (|eta| > eps && it <= max_iter - 1) || it < 1.
__device__ __noinline__ PcgOut pcg_fp64(const Inst& s, double* lv, double* rv, double* pv, double* tv, double* uv,
                           int max_iter, double eps, double* red, int& par) {
  const int n = s.K * s.nx, nx = s.nx, N = s.N;
  double part = 0.0;
  for (int g = threadIdx.x; g < n; g += blockDim.x)
    rv[g] = s.gam[g] + stencil_row<double, double>(s.th, s.ph, nx, nx, N, lv, g);  // S = -stencil
  __syncthreads();
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const double rt = stencil_row<double, double>(s.ti, s.pm, nx, nx, N, rv, g);
    tv[g] = rt;
    pv[g] = rt;
    part += rv[g] * rt;
  }
  double eta = block_sum(part, red, par);
  int it = 0;
  while ((fabs(eta) > eps && it <= max_iter - 1) || it < 1) {
    part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const double u = -stencil_row<double, double>(s.th, s.ph, nx, nx, N, pv, g);
      uv[g] = u;
      part += pv[g] * u;
    }
    const double vden = block_sum(part, red, par);
    const double alpha = eta / vden;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      lv[g] += alpha * pv[g];
      rv[g] -= alpha * uv[g];
    }
    __syncthreads();
    part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const double rt = stencil_row<double, double>(s.ti, s.pm, nx, nx, N, rv, g);
      tv[g] = rt;
      part += rv[g] * rt;
    }
    const double etap = block_sum(part, red, par);
    const double beta = etap / eta;
    for (int g = threadIdx.x; g < n; g += blockDim.x) pv[g] = tv[g] + beta * pv[g];
    eta = etap;
    ++it;
    __syncthreads();
  }
  return PcgOut{it, eta};
}

// (L_t^-1 v_t)_i = sum_{j <= i} Li_t[i][j] v_t[j]   (FP64 vector with row stride nx)
__device__ __forceinline__ double lower_row(const double* __restrict__ li, int nx, int t, int i,
                                            const double* __restrict__ v) {
  const double* m = li + ((size_t)t * nx + i) * nx;
  const double* x = v + (size_t)t * nx;
  double a = 0.0;
  for (int j = 0; j <= i; ++j) a = fma(m[j], x[j], a);
  return a;
}

// (L_t^-T v_t)_i = sum_{j >= i} Li_t[j][i] v_t[j]   (v_t: one FP32 vector segment)
__device__ __forceinline__ double lower_col(const double* __restrict__ li, int nx, int t, int i,
                                            const float* __restrict__ vt) {
  const double* m = li + (size_t)t * nx * nx + i;
  double a = 0.0;
  for (int j = i; j < nx; ++j) a = fma(m[(size_t)j * nx], (double)vt[j], a);
  return a;
}

// (L_t^-T v_t)_i for an FP64 vector with row stride nx
__device__ __forceinline__ double lower_col64(const double* __restrict__ li, int nx, int t, int i,
                                              const double* __restrict__ vt) {
  const double* m = li + (size_t)t * nx * nx + i;
  double a = 0.0;
  for (int j = i; j < nx; ++j) a = fma(m[(size_t)j * nx], vt[j], a);
  return a;
}

// (F^ v)_{t,i} in FP64 from the W blocks kept with row stride nx (block t-1 holds W_t, block
// N is zero) for an unpadded FP64 vector v with row stride nx.
__device__ __forceinline__ double fhat64_row(const double* __restrict__ w, int nx, int N, int t, int i,
                                             const double* __restrict__ v) {
  const int nn = nx * nx;
  double a = 0.0, c = 0.0;
  if (t > 0) {
    const double* lo = w + (size_t)(t - 1) * nn + i * nx;
    const double* vm = v + (size_t)(t - 1) * nx;
    for (int j = 0; j < nx; ++j) a = fma(lo[j], vm[j], a);
  }
  if (t < N) {
    const double* up = w + (size_t)t * nn + i;
    const double* vp = v + (size_t)(t + 1) * nx;
    for (int j = 0; j < nx; ++j) c = fma(up[(size_t)j * nx], vp[j], c);
  }
  return a + c;
}

// The FP64 fallback of the mixed path: the reference recurrence (pcg.py:350-436) in the
// scaled basis, i.e. PCG on S^ = -(I + F^) with the preconditioner I - F^ for the
// correction d^ from lam (r^ = L^-1 (gamma - S lam), lam += L^-T d^ at the end).  Its
// iterates, eta and stopping rule are the reference's in exact arithmetic.  Vectors in
// workspace regions free during the solve: r^ t1, p^ xn, u^ C, z^ tmp, d^ res.
__device__ __noinline__ PcgOut pcg_fp64_scaled(const Inst& s, double* lam, int max_iter, double eps, double* red,
                                               int& par) {
  const int nx = s.nx, N = s.N, n = s.K * nx;
  double *rh = s.t1, *pv = s.xn, *uv = s.C, *zv = s.tmp, *dv = s.res;
  const double* w = s.pm;  // FP64 W blocks
  for (int g = threadIdx.x; g < n; g += blockDim.x)
    s.res[g] = s.gam[g] + stencil_row<double, double>(s.th, s.ph, nx, nx, N, lam, g);
  __syncthreads();
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx;
    rh[g] = lower_row(s.li, nx, t, g - t * nx, s.res);
  }
  __syncthreads();
  double part = 0.0;
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx;
    const double z = rh[g] - fhat64_row(w, nx, N, t, g - t * nx, rh);
    pv[g] = z;
    dv[g] = 0.0;
    part += rh[g] * z;
  }
  double eta = block_sum(part, red, par);
  int it = 0;
  while ((fabs(eta) > eps && it <= max_iter - 1) || it < 1) {
    part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      const double u = -(pv[g] + fhat64_row(w, nx, N, t, g - t * nx, pv));
      uv[g] = u;
      part += pv[g] * u;
    }
    const double vden = block_sum(part, red, par);
    const double alpha = eta / vden;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      dv[g] += alpha * pv[g];
      rh[g] -= alpha * uv[g];
    }
    __syncthreads();
    part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      const double z = rh[g] - fhat64_row(w, nx, N, t, g - t * nx, rh);
      zv[g] = z;
      part += rh[g] * z;
    }
    const double etap = block_sum(part, red, par);
    const double beta = etap / eta;
    for (int g = threadIdx.x; g < n; g += blockDim.x) pv[g] = zv[g] + beta * pv[g];
    eta = etap;
    ++it;
    __syncthreads();
  }
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx;
    lam[g] += lower_col64(s.li, nx, t, g - t * nx, dv + (size_t)t * nx);
  }
  __syncthreads();
  return PcgOut{it, eta};
}

// The FP32 PCG is not paying off (a replacement shows the true residual stalled while the
// recursion fell, the recursion diverged or stalled, or the FP32 iterations used half of
// pcg.max_iter or max_refinement replacements).  Finish the solve with the FP64 recurrence (in
// the scaled basis, see pcg_fp64_scaled) from the current lam.  The recurrence gets the full
// pcg.max_iter budget of the reference's loop: the FP32 iterations before it are cheaper and
// not charged against it, so a QP's reported iteration count can reach 1.5 max_iter.
__device__ PcgOut fp64_finish(const Inst& s, double* lam, int it, int max_iter, double eps, double* red, int& par,
                              int nrep) {
  // without Cholesky factors (sh_scaled_bad) the reference-basis blocks theta^-1, P exist instead
  PcgOut o = sh_scaled_bad ? pcg_fp64(s, lam, s.res, s.t1, s.xn, s.C, max_iter, eps, red, par)
                           : pcg_fp64_scaled(s, lam, max_iter, eps, red, par);
  return PcgOut{it + o.it, o.eta, nrep, o.it};
}
// Residual-replacement PCGs (pcg_rows_scaled, pcg_mixed_scaled): the FP64 convergence test runs once the
// FP32 recursion's eta is below kCheckMargin * eps, and a replacement after which the
// FP64 eta fell by less than 1/kUpdateStagnation hands the solve to the FP64 recurrence.
constexpr double kCheckMargin = 0.1;
constexpr double kUpdateStagnation = 1e-2;
// A replaced residual whose eta exceeds the recursion's previous eta by this factor
// restarts the search direction.
constexpr double kRestartRatio = 10.0;
// The FP32 recursion's eta rising this far above its value at the last replacement
// triggers a replacement (and, without true progress, the FP64 recurrence).
constexpr double kDivergeRatio = 1e4;
// Stall detection: an FP32 segment (the iterations between two replacements) that runs past
// max(kStallGrowth x the previous segment, kStallMin) iterations (kStallMin for the first) is cut
// by a replacement, after which the FP32 PCG continues only if the true eta fell by the full
// inner_rel_tol factor since the last replacement: an FP32 recursion that has stopped falling on
// an ill-conditioned system, or falls far slower than before, goes to the FP64 recurrence after a
// few hundred iterations instead of half the budget.
constexpr int kStallMin = 200;
constexpr int kStallGrowth = 2;
__device__ __forceinline__ int next_stop(int it, int seg, int it_cap) {
  return min(it_cap, it + max(kStallGrowth * seg, kStallMin));
}

// ---------------------------------------------------------------- PCG, FP32 in a scaled basis + FP64 refinement
// Scaled basis.  With the FP64 Cholesky factors theta_t = L_t L_t^T (L block diagonal)
// and lam = L^-T lam^:
//   S^   = L^-1 S L^-T    = -(I + F^)
//   Phi^ = L^T Phi^-1 L   =   I - F^        (Phi^-1 = Theta^-1 - Theta^-1 F Theta^-1)
// where F is the off-diagonal part of -S (F_{t,t-1} = phi_{t-1}, F_{t,t+1} = phi_t^T) and
// F^ = L^-1 F L^-T has the blocks F^_{t,t-1} = W_t = L_t^-1 phi_{t-1} L_{t-1}^-T and
// F^_{t,t+1} = W_{t+1}^T.  PCG is invariant under this congruence (r^ = L^-1 r,
// z^ = L^T z, p^ = L^T p, S^ p^ = L^-1 S p), so r.z, p.Sp, alpha, beta and eta are those
// of the reference recurrence (pcg.py:350-436) in exact arithmetic, while an iteration
// reads only the W blocks: one off-diagonal block per stage instead of the six blocks
// per knot of S and Phi^-1, and the unit diagonal needs no storage.
//
// FP64 correction: residual replacement in both FP32 PCGs (pcg_rows_scaled for the nx with a
// compile-time row layout, pcg_mixed_scaled for any nx): one FP32 PCG whose recursively updated
// residual is replaced by the FP64 residual each time its eta has fallen by `inner_rel_tol`,
// keeping the search direction (reliable updates: no Krylov space is thrown away at a restart).
// The replacement residual is formed in the scaled basis from the FP64 W blocks,
// r^ = r^_0 + (I + F^) lam^; the stopping test always uses an exact gamma - S lam.


template <class T>
__device__ __forceinline__ T* as_shared(T* p) {
  const ptrdiff_t off = reinterpret_cast<const unsigned char*>(p) - g_dyn_smem;
  return reinterpret_cast<T*>(g_dyn_smem + off);
}

// Compile-time-nx FP64 helpers of the row PCGs: rows q + k TPK (k < R, TPK = ceil(NX / R)) of
// knot t for pcg_rows_scaled, rows R q + k for pcg_rows_t (CONTIG); a row past NX, or a thread
// without a knot (ok false), is skipped.  They stay out of line, so that their registers do not
// weigh on the allocation of the FP32 iteration loop that calls them on its cold path.
template <int NX, int R>
struct RowVals {
  double v[R];
};
template <int NX, int R, bool CONTIG>
__device__ __forceinline__ int row_of(int q, int k) {
  return CONTIG ? R * q + k : q + k * ((NX + R - 1) / R);
}

// res = gamma - S lam for the thread's rows and r^ = L^-1 res in t1 (one barrier between the
// passes; each thread reads back only its own t1 rows).
template <int NX, int R, bool CONTIG = false>
__device__ __noinline__ void exact_rhat_rows(const Inst& s, const double* lam, int t, int q, bool ok, int N) {
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int i = row_of<NX, R, CONTIG>(q, k);
    if (ok && i < NX) s.res[t * NX + i] = s.gam[t * NX + i] + stencil64<NX>(s.th, s.ph, lam, t, i, N);
  }
  __syncthreads();
  const double* x = s.res + t * NX;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int i = row_of<NX, R, CONTIG>(q, k);
    if (ok && i < NX) {
      const double* m = s.li + (size_t)(t * NX + i) * NX;
      double a = 0.0;
#pragma unroll
      for (int j = 0; j < NX; ++j)
        if (j <= i) a = fma(m[j], x[j], a);
      s.t1[t * NX + i] = a;
    }
  }
}

// (F^ v) for the thread's rows in FP64: W_t (block t-1 of w, row stride NX) times v_{t-1} plus
// W_{t+1}^T (block t) times v_{t+1}; block N is zero and stands in for W_0 and W_{N+1}.  v points
// at knot 0 of a vector with zero segments at knots -1 and K.  A row past NX repeats row q.
template <int NX, int R, bool CONTIG = false>
__device__ __noinline__ RowVals<NX, R> fhat64_rows(const double* __restrict__ w, int N, int t, int q,
                                                   const double* v) {
  constexpr int BS = NX * NX;
  const double* lo = w + (size_t)(t > 0 ? t - 1 : N) * BS;
  const double* up = w + (size_t)(t < N ? t : N) * BS;
  const double* vm = v + (t - 1) * NX;
  const double* vp = v + (t + 1) * NX;
  double a[R], b[R];
  int ii[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    a[k] = 0.0;
    b[k] = 0.0;
    ii[k] = (row_of<NX, R, CONTIG>(q, k) < NX) ? row_of<NX, R, CONTIG>(q, k) : q;
  }
#pragma unroll
  for (int j = 0; j < NX; ++j) {
    const double ym = vm[j], yp = vp[j];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      a[k] = fma(lo[ii[k] * NX + j], ym, a[k]);
      b[k] = fma(up[j * NX + ii[k]], yp, b[k]);
    }
  }
  RowVals<NX, R> o;
#pragma unroll
  for (int k = 0; k < R; ++k) o.v[k] = a[k] + b[k];
  return o;
}

// (L_t^-T v_t)_i for an FP64 vector segment v_t
template <int NX>
__device__ __forceinline__ double lower_col_t(const double* __restrict__ li, int t, int i, const double* vt) {
  const double* m = li + (size_t)t * NX * NX + i;
  double a = 0.0;
#pragma unroll
  for (int j = 0; j < NX; ++j)
    if (j >= i) a = fma(m[j * NX], vt[j], a);
  return a;
}

// (F^ v)_{t,i} = W_t[i,:] v_{t-1} + W_{t+1}[:,i] v_{t+1} for padded vectors (zero segments
// at t = -1 and t = K); block N of w is zero and stands in for W_0 and W_{N+1}.
__device__ __forceinline__ float fhat_row(const float* __restrict__ w, int nx, int ld, int N, int t, int i,
                                          const float* __restrict__ v) {
  const int bs = nx * ld;
  const float* lo = w + (t > 0 ? t - 1 : N) * bs + i * ld;
  const float* up = w + (t < N ? t : N) * bs + i;
  const float* vm = v + (t - 1) * ld;
  const float* vp = v + (t + 1) * ld;
  float a0 = 0.f, a1 = 0.f;
  for (int j = 0; j < nx; ++j) {
    a0 = fmaf(lo[j], vm[j], a0);
    a1 = fmaf(up[j * ld], vp[j], a1);
  }
  return a0 + a1;
}

// Any nx and horizon: thread rows g = tid + k*blockDim; five padded FP32 vectors r^, p^, z^, u^, d^
// (K + 2 segments of ld floats with zero end segments) in shared memory, the FP32 W blocks in
// shared or global memory.  One FP32 PCG with FP64 residual replacement, by the same rules as
// the compile-time row PCG (pcg_rows_scaled): the FP32 vectors carry the problem scaled by
// 1/sqrt(eta64) of the first residual; each time the recursion's eta has fallen by `upd_rel`
// (or rises 1e4-fold, or is not a number) the accumulated step goes into an FP64 sum lam^ (tmp),
// the true scaled residual r^ = r^_0 + (I + F^) lam^ from the FP64 W blocks replaces the
// recursive one and the search direction is kept; the convergence decision rests on an exact
// residual gamma - S lam (evaluated once the recursion is below 0.1 eps, or when the replaced
// residual is).  The FP64 recurrence finishes the solve (fp64_finish) when a replacement that the
// recursion's fall (or the stall detection) triggered shows a true fall of less than 100x, after
// max_ref replacements, after half the budget, or on a non-finite recursion.  FP64 vectors in workspace regions free
// during the solve: r^_0 t1, candidate r^ xn, z^ (FP64) C, lam^ tmp.
__device__ __noinline__ PcgOut pcg_mixed_scaled(const Inst& s, double* lam, float* vec, int max_iter, double eps,
                                                int max_ref, double upd_rel, double* red, int& par) {
  const int nx = s.nx, N = s.N, K = s.K, ld = s.ld, n = K * nx;
  const int span = (K + 2) * ld;
  for (int w = threadIdx.x; w < 5 * span; w += blockDim.x) vec[w] = 0.f;
  float* rv = vec + ld;
  float* pv = rv + span;
  float* zv = pv + span;
  float* uv = zv + span;
  float* dv = uv + span;
  const float* w32 = s.w32;
  const double* w64 = s.pm;  // FP64 W blocks (row stride nx, block N zero)
  double *rh0 = s.t1, *rhc = s.xn, *zh = s.C, *acc = s.tmp;
  const int w2 = warp_pow2();
  // res = gamma - S lam, r^_0 = L^-1 res (t1)
  auto exact = [&]() {
    for (int g = threadIdx.x; g < n; g += blockDim.x)
      s.res[g] = s.gam[g] + stencil_row<double, double>(s.th, s.ph, nx, nx, N, lam, g);
    __syncthreads();
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      rh0[g] = lower_row(s.li, nx, t, g - t * nx, s.res);
    }
    __syncthreads();
  };
  // z^ = r^ - F^ r^ in FP64 (zh) for an FP64 r^; returns eta64 = r^.z^
  auto eta_of = [&](const double* rh) -> double {
    double part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      const double z = rh[g] - fhat64_row(w64, nx, N, t, g - t * nx, rh);
      zh[g] = z;
      part += rh[g] * z;
    }
    return block_sum(part, red, par);
  };
  // lam += L^-T lam^, lam^ = 0
  auto flush = [&]() {
    __syncthreads();
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      zh[g] = lower_col64(s.li, nx, t, g - t * nx, acc + (size_t)t * nx);
    }
    __syncthreads();
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      lam[g] += zh[g];
      acc[g] = 0.0;
    }
    __syncthreads();
  };
  // scaled FP32 copies of an FP64 r^ (and of zh)
  auto load32 = [&](const double* rh, double scale) {
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx, x = t * ld + (g - t * nx);
      rv[x] = (float)(scale * rh[g]);
      zv[x] = (float)(scale * zh[g]);
    }
  };
  for (int g = threadIdx.x; g < n; g += blockDim.x) acc[g] = 0.0;
  exact();
  double eta64 = eta_of(rh0);
  int it = 0;
  if (!(eta64 == eta64)) return PcgOut{it, eta64};  // the reference loop always runs an iteration
  const double scale = (eta64 > 0.0) ? rsqrt(eta64) : 1.0, back = (eta64 > 0.0) ? sqrt(eta64) : 1.0;
  const double s2 = scale * scale, check_at = eps * s2 * kCheckMargin;
  double prev64 = eta64, eta_upd = eta64 * s2, eta = eta64 * s2;
  int nupd = 0, seg0 = 0;
  const int it_cap = max_iter / 2;  // FP32 share of the budget; the rest is kept for fp64_finish
  int it_stop = min(it_cap, kStallMin);  // stall detection: the current segment ends here at the latest
  load32(rh0, scale);
  __syncthreads();
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx, x = t * ld + (g - t * nx);
    pv[x] = zv[x];
  }
  double trig = fmax(check_at, upd_rel * eta), hi = kDivergeRatio * eta;
  __syncthreads();
  for (;;) {
    double vden, etap;
    for (;;) {
      // u^ = S^ p^ = -(p^ + F^ p^)
      float part = 0.f;
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, i = g - t * nx, x = t * ld + i;
        const float u = -(pv[x] + fhat_row(w32, nx, ld, N, t, i, pv));
        uv[x] = u;
        part = fmaf(pv[x], u, part);
      }
      vden = block_sum_f32w(part, red, par, w2);
      const float alpha = quot32(eta, vden);
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, x = t * ld + (g - t * nx);
        dv[x] = fmaf(alpha, pv[x], dv[x]);
        rv[x] = fmaf(-alpha, uv[x], rv[x]);
      }
      __syncthreads();
      // z^ = Phi^ r^ = r^ - F^ r^
      part = 0.f;
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, i = g - t * nx, x = t * ld + i;
        const float z = rv[x] - fhat_row(w32, nx, ld, N, t, i, rv);
        zv[x] = z;
        part = fmaf(rv[x], z, part);
      }
      etap = block_sum_f32w(part, red, par, w2);
      ++it;
      if (!(etap > trig) || etap > hi || it >= it_stop || !(vden == vden)) break;
      const float beta = quot32(etap, eta);
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, x = t * ld + (g - t * nx);
        pv[x] = fmaf(beta, pv[x], zv[x]);
      }
      eta = etap;
      __syncthreads();
    }
    // Residual replacement (see above); a non-finite segment is dropped.
    const bool bad = !(etap == etap) || !(vden == vden);
    const bool at_check = etap <= check_at;
    const bool fell = etap <= upd_rel * eta_upd || etap > hi;
    const bool cut = !fell && it >= it_stop && it < it_cap;  // ended by the stall detection
    const bool progressed = fell || cut;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx, x = t * ld + (g - t * nx);
      if (!bad) acc[g] += back * (double)dv[x];
      dv[x] = 0.f;
    }
    __syncthreads();
    bool exact_now = bad || at_check || it >= it_cap;
    const double* rh = rh0;
    if (!exact_now) {
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx;
        rhc[g] = rh0[g] + acc[g] + fhat64_row(w64, nx, N, t, g - t * nx, acc);
      }
      __syncthreads();
      eta64 = eta_of(rhc);
      rh = rhc;
      exact_now = !(eta64 > eps);
    }
    if (exact_now) {
      flush();
      exact();
      eta64 = eta_of(rh0);
      rh = rh0;
    }
    ++nupd;
    if (!(fabs(eta64) > eps && it <= max_iter - 1) || !(eta64 == eta64)) {
      if (!exact_now) flush();
      break;
    }
    const double etas = eta64 * s2;
    if (bad || nupd >= max_ref || it >= it_cap || !(etas > 0.0) ||
        (progressed && !at_check && eta64 > (cut ? upd_rel : kUpdateStagnation) * prev64)) {
      if (!exact_now) flush();
      return fp64_finish(s, lam, it, max_iter, eps, red, par, nupd);
    }
    prev64 = eta64;
    eta_upd = etas;
    it_stop = next_stop(it, it - seg0, it_cap);
    seg0 = it;
    load32(rh, scale);
    const bool restart = etas > kRestartRatio * eta;  // a stale direction: restart it
    const float beta = restart ? 0.f : quot32(etas, eta);
    __syncthreads();
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx, x = t * ld + (g - t * nx);
      pv[x] = fmaf(beta, pv[x], zv[x]);
    }
    eta = etas;
    trig = fmax(check_at, upd_rel * etas);
    hi = kDivergeRatio * etas;
    __syncthreads();
  }
  return PcgOut{it, eta64, nupd};
}

// Compile-time nx, K ceil(nx / R) <= blockDim.  Thread (t, q) = (tid mod K, tid div K) owns the
// rows i_k = q + k TPK (k < R, i_k < nx; TPK = ceil(nx / R) threads per knot) of block row t and
// keeps their W coefficients (W_t rows i_k and W_{t+1} columns i_k: 2 R nx floats) in registers
// for the whole FP32 segment.  Both operators then read only the vector segments t-1 and t+1
// from shared memory, each loaded once for all R rows.  Lanes run over t for a fixed q, so a half
// warp's 64-bit segment loads (ld/2 odd) hit distinct banks.  Threads past the last knot
// (tid >= TPK K) idle on knot 0, row q = 0, which keeps every address in range; they take part
// in the barriers and reductions with zeros.
//
// The recursion's two dot products per iteration are summed in FP32 over each thread's rows and
// each warp and in FP64 over the warps (block_sum_f32w), and its step lengths alpha, beta are
// FP32 quotients (quot32).  Its vectors are FP32 already, and the exact FP64 residual of every
// replacement decides convergence; both shorten the CTA-wide reductions that bound an
// iteration's latency.
//
// Registers.  The W coefficients (2 R nx floats) dominate a thread's registers, so they are
// loaded from the workspace at the start of every FP32 segment and are dead across the FP64
// residual replacement that ends it, and the two neighbour segments of a stencil are read one
// after the other.  This keeps the iteration loop free of register spills with the 168 registers
// a thread of a CTA of at most 384 threads can have (kCfgRows384); at most 256 threads (kCfgRows,
// up to 255 registers) it also leaves the compiler room to schedule the stencil's loads early
// (2.8 K instead of 3.3 K cycles per iteration for the quadrotor, N=60).
template <int NX, int R>
__device__ __noinline__ PcgOut pcg_rows_scaled(const Inst& s, double* lam, float* vec, int max_iter, double eps,
                                               int max_ref, double upd_rel, double* red, int& par) {
  constexpr int LD = pad_ld(NX);
  constexpr int BS = NX * LD;
  constexpr int TPK = (NX + R - 1) / R;
  constexpr int NP = (NX + 1) / 2;  // float2 pairs per padded segment
  const int K = s.K, N = s.N;
  float* rbase = as_shared(vec);  // (K + 2) segments: [0][v_0 .. v_N][0]
  float* pbase = as_shared(vec + (K + 2) * LD);
  float* rv = rbase + LD;
  float* pv = pbase + LD;
  red = as_shared(red);
  const int qq = threadIdx.x / K;
  const bool ok = qq < TPK;
  const int q = ok ? qq : 0;
  const int tc = ok ? threadIdx.x - qq * K : 0;
  auto row = [&](int k) { return q + k * TPK; };
  auto has = [&](int k) { return ok && q + k * TPK < NX; };
  const int seg = tc * LD;  // segment t in the padded vectors
  for (int w = threadIdx.x; w < (K + 2) * LD; w += blockDim.x) {
    if (w < LD || w >= (K + 1) * LD || (w % LD) >= NX) {
      rbase[w] = 0.f;
      pbase[w] = 0.f;
    }
  }
  // F^ v for the thread's rows: W_t v_{t-1} (wl), then W_{t+1}^T v_{t+1} (wu)
  auto fhat = [&](const float (&wl)[R][NX], const float (&wu)[R][NX], const float* v, float* f) {
    float a[R], b[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      a[k] = 0.f;
      b[k] = 0.f;
    }
    {
      const float2* vm = reinterpret_cast<const float2*>(v + seg - LD);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        const float2 y = vm[j];
#pragma unroll
        for (int k = 0; k < R; ++k) {
          a[k] = fmaf(wl[k][2 * j], y.x, a[k]);
          if (2 * j + 1 < NX) b[k] = fmaf(wl[k][2 * j + 1], y.y, b[k]);
        }
      }
    }
    {
      const float2* vp = reinterpret_cast<const float2*>(v + seg + LD);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        const float2 x = vp[j];
#pragma unroll
        for (int k = 0; k < R; ++k) {
          a[k] = fmaf(wu[k][2 * j], x.x, a[k]);
          if (2 * j + 1 < NX) b[k] = fmaf(wu[k][2 * j + 1], x.y, b[k]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) f[k] = a[k] + b[k];
  };
  auto store = [&](float* v, const float* x) {
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (has(k)) v[seg + row(k)] = x[k];
  };
  // the thread's FP32 share of a dot product
  auto dot32 = [&](const float* a, const float* b) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (has(k)) acc = fmaf(a[k], b[k], acc);
    return acc;
  };
  const int w2 = warp_pow2();
  // FP64 exchange vector (knots -1..K) in the shared vector slots the row path leaves free,
  // followed by the solve's constants (cst).  Everything the residual replacements need is
  // re-derived there from s, vec and cst, so that none of it occupies registers of the
  // iteration loop.
  auto x64_of = [&]() { return reinterpret_cast<double*>(as_shared(vec + 2 * (K + 2) * LD)) + NX; };
  {
    double* x64 = x64_of();
    for (int w = threadIdx.x; w < NX; w += blockDim.x) {
      x64[w - NX] = 0.0;
      x64[K * NX + w] = 0.0;
    }
  }
  // r^ rows (rh) -> z^ = r^ - F^ r^ rows (zh); returns the thread's share of eta = r^.z^
  auto eta_of = [&](const double* rh, double* zh) -> double {
    double* x64 = x64_of();
    __syncthreads();
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (has(k)) x64[tc * NX + row(k)] = rh[k];
    __syncthreads();
    const RowVals<NX, R> h = fhat64_rows<NX, R>(s.pm, N, tc, q, x64);
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      zh[k] = rh[k] - h.v[k];
      if (has(k)) e += rh[k] * zh[k];
    }
    return e;
  };
  // lam += L^-T acc, acc = 0 (acc: lam^ accumulated since the last exact residual, FP64 in tmp)
  auto flush = [&]() {
    double* acc = s.tmp;
    __syncthreads();
    double l[R];
#pragma unroll
    for (int k = 0; k < R; ++k) l[k] = lower_col_t<NX>(s.li, tc, has(k) ? row(k) : q, acc + tc * NX);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (has(k)) {
        lam[tc * NX + row(k)] += l[k];
        acc[tc * NX + row(k)] = 0.0;
      }
    __syncthreads();
  };
  float r[R], p[R], d[R], f[R];
  int it = 0;
  double eta;
  float trig, hi;
  {
    double rh[R], zh[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      d[k] = 0.f;
      if (has(k)) s.tmp[tc * NX + row(k)] = 0.0;
    }
    exact_rhat_rows<NX, R>(s, lam, tc, q, ok, N);
#pragma unroll
    for (int k = 0; k < R; ++k) rh[k] = has(k) ? s.t1[tc * NX + row(k)] : 0.0;
    const double eta64 = block_sum2(eta_of(rh, zh), red, par);
    if (!(eta64 == eta64)) return PcgOut{it, eta64};
    // The FP32 vectors carry the problem scaled by 1/sqrt(eta64) of the first residual
    // (eta starts at 1) and keep that scale through every replacement.  cst: scale,
    // sqrt(eta64_0), scale^2, the convergence-check level, eta64 and the scaled eta at the
    // last replacement, eps, upd_rel, max_ref, the replacement count, max_iter, the first
    // iteration of the current FP32 segment.
    const double scale = (eta64 > 0.0) ? rsqrt(eta64) : 1.0;
    double* cst = x64_of() + (K + 1) * NX;
    if (threadIdx.x == 0) {
      cst[0] = scale;
      cst[1] = (eta64 > 0.0) ? sqrt(eta64) : 1.0;
      cst[2] = scale * scale;
      cst[3] = eps * scale * scale * kCheckMargin;
      cst[4] = eta64;
      cst[5] = eta64 * scale * scale;
      cst[6] = eps;
      cst[7] = upd_rel;
      cst[8] = (double)max_ref;
      cst[9] = 0.0;
      cst[10] = (double)max_iter;
      cst[11] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
      r[k] = (float)(scale * rh[k]);
      p[k] = (float)(scale * zh[k]);
    }
    eta = eta64 * scale * scale;
    // a replacement is due once the recursion's eta is at or below trig, above hi (the
    // recursion diverges: FP32 cannot resolve this system) or not a number
    trig = (float)fmax(eps * scale * scale * kCheckMargin, upd_rel * eta);
    hi = (float)(kDivergeRatio * eta);
  }
  // the FP32 segment ends at it_stop at the latest (stall detection; max_iter / 2, the FP32 share
  // of the budget, bounds it: the rest is kept for fp64_finish)
  int it_stop = min(max_iter / 2, kStallMin);
  int nrep_out;  // set where the loop ends
  store(pv, p);
  __syncthreads();
  double eta64 = 0.0;
  const int lo_blk = (tc > 0 ? tc - 1 : N) * BS;  // block N is zero
  const int up_blk = (tc < N ? tc : N) * BS;
  for (;;) {
    // FP32 iterations until a replacement is due (a tight loop of its own)
    double vden, etap;
    float z[R];
    {
      float wl[R][NX], wu[R][NX];
      {
        const float* w = s.w32;
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const int i = has(k) ? row(k) : q;
#pragma unroll
          for (int j = 0; j < NX; ++j) {
            wl[k][j] = has(k) ? w[lo_blk + i * LD + j] : 0.f;
            wu[k][j] = has(k) ? w[up_blk + j * LD + i] : 0.f;
          }
        }
      }
      for (;;) {
        // u^ = S^ p^ = -(p^ + F^ p^)
        float u[R];
        fhat(wl, wu, pv, f);
#pragma unroll
        for (int k = 0; k < R; ++k) u[k] = -(p[k] + f[k]);
        vden = block_sum_f32w(dot32(p, u), red, par, w2);
        const float alpha = quot32(eta, vden);
#pragma unroll
        for (int k = 0; k < R; ++k) {
          d[k] = fmaf(alpha, p[k], d[k]);
          r[k] = fmaf(-alpha, u[k], r[k]);
        }
        store(rv, r);
        __syncthreads();
        // z^ = Phi^ r^ = r^ - F^ r^
        fhat(wl, wu, rv, f);
#pragma unroll
        for (int k = 0; k < R; ++k) z[k] = r[k] - f[k];
        etap = block_sum_f32w(dot32(r, z), red, par, w2);
        ++it;
        const float etaf = (float)etap;
        if (!(etaf > trig) || etaf > hi || it >= it_stop || !(vden == vden)) break;
        const float beta = quot32(etap, eta);
#pragma unroll
        for (int k = 0; k < R; ++k) p[k] = fmaf(beta, p[k], z[k]);
        store(pv, p);
        eta = etap;
        __syncthreads();
      }
    }
    {
      // Residual replacement.  acc += sqrt(eta64_0) d^ (FP64); the true scaled residual
      // r^ = r^_0 + (I + F^) acc (r^_0 = t1, the residual at the last exact evaluation)
      // replaces the recursively updated one and the search direction is kept.  The
      // convergence decision always rests on an exact residual gamma - S lam.
      double* cst = x64_of() + (K + 1) * NX;
      double* acc = s.tmp;
      const double scale = cst[0], back = cst[1], s2 = cst[2], check_at = cst[3], prev64 = cst[4],
                   eta_upd = cst[5], c_eps = cst[6], c_upd = cst[7];
      const int c_maxref = (int)cst[8], nupd = (int)cst[9] + 1, c_maxit = (int)cst[10], it_cap = c_maxit / 2;
      const bool bad = !(etap == etap) || !(vden == vden);
      const bool at_check = etap <= check_at;
      // a segment cut by the stall detection counts as progress for the stagnation rule
      const bool fell = etap <= c_upd * eta_upd || (float)etap > hi;
      const bool cut = !fell && it >= it_stop && it < it_cap;  // ended by the stall detection
      const bool progressed = fell || cut;
      // a non-finite segment is dropped: lam keeps the last finite update
      double a[R];
#pragma unroll
      for (int k = 0; k < R; ++k) {
        a[k] = has(k) ? acc[tc * NX + row(k)] : 0.0;
        if (!bad) {
          a[k] += back * (double)d[k];
          if (has(k)) acc[tc * NX + row(k)] = a[k];
        }
        d[k] = 0.f;
      }
      double rh[R], zh[R];
      bool exact = bad || at_check || it >= it_cap;
      if (!exact) {
        double* x64 = x64_of();
        __syncthreads();
#pragma unroll
        for (int k = 0; k < R; ++k)
          if (has(k)) x64[tc * NX + row(k)] = a[k];
        __syncthreads();
        const RowVals<NX, R> h = fhat64_rows<NX, R>(s.pm, N, tc, q, x64);
#pragma unroll
        for (int k = 0; k < R; ++k) rh[k] = has(k) ? s.t1[tc * NX + row(k)] + a[k] + h.v[k] : 0.0;
        eta64 = block_sum2(eta_of(rh, zh), red, par);
        exact = !(eta64 > c_eps);
      }
      if (exact) {
        flush();
        exact_rhat_rows<NX, R>(s, lam, tc, q, ok, N);
#pragma unroll
        for (int k = 0; k < R; ++k) rh[k] = has(k) ? s.t1[tc * NX + row(k)] : 0.0;
        eta64 = block_sum2(eta_of(rh, zh), red, par);
      }
      if (!(fabs(eta64) > c_eps && it <= c_maxit - 1) || !(eta64 == eta64)) {
        if (!exact) flush();
        nrep_out = nupd;
        break;
      }
      const double etas = eta64 * s2;
      if (bad || nupd >= c_maxref || it >= it_cap || !(etas > 0.0) ||
          (progressed && !at_check && eta64 > (cut ? c_upd : kUpdateStagnation) * prev64)) {
        if (!exact) flush();
        return fp64_finish(s, lam, it, c_maxit, c_eps, red, par, nupd);
      }
      it_stop = next_stop(it, it - (int)cst[11], it_cap);
      __syncthreads();
      if (threadIdx.x == 0) {
        cst[4] = eta64;
        cst[5] = etas;
        cst[9] = (double)nupd;
        cst[11] = (double)it;
      }
#pragma unroll
      for (int k = 0; k < R; ++k) {
        r[k] = (float)(scale * rh[k]);
        z[k] = (float)(scale * zh[k]);
      }
      // a true residual far above the recursion's means a stale direction: restart
      if (etas > kRestartRatio * eta) {
#pragma unroll
        for (int k = 0; k < R; ++k) p[k] = 0.f;
      }
      etap = etas;
      trig = (float)fmax(check_at, c_upd * etas);
      hi = (float)(kDivergeRatio * etas);
    }
    const float beta = quot32(etap, eta);
#pragma unroll
    for (int k = 0; k < R; ++k) p[k] = fmaf(beta, p[k], z[k]);
    store(pv, p);
    eta = etap;
    __syncthreads();
  }
  return PcgOut{it, eta64, nrep_out};
}

// Two CTAs per SM (kCfgDual: 256 threads, 128 registers a thread).  Compile-time nx, TPK threads
// per knot (TPK = 1, 2, 4 for nx <= 4, 8, 16), K TPK <= blockDim.  Thread (t, q) = (tid div TPK,
// tid mod TPK) owns rows 4q .. 4q + 3 of block row t and keeps those rows of W_t, padded to
// PD = 4 TPK columns, in registers: 4 PD floats (64 for the quadrotor), ONE copy of each W block
// instead of the row layout's two (W_t rows and W_{t+1} columns), which is what lets two
// instances share an SM.  Both products of F^ v come from those registers:
//   lower  (W_t v_{t-1})_i      = sum_j W_t[i, j] v_{t-1, j}: the thread's rows, v_{t-1} from
//                                 shared memory;
//   upper  (W_t^T v_t)_j        = sum_i W_t[i, j] v_{t, i}: the thread's share from its own v_t
//                                 rows (registers), summed over the knot's TPK lanes by a
//                                 reduce-scatter of warp shuffles (log2 TPK rounds), after
//                                 which lane q holds columns 4q .. 4q + 3.  They are knot t-1's
//                                 upper term and go to shared memory (segment t-1 of `up`) in
//                                 the same barrier interval as v_t itself.
// So that the reduce-scatter needs no selects, lane q keeps its W columns in an order that puts
// the columns it sends in the first half of its registers at each round: register group g holds
// column group g ^ (TPK - 1 - q).  The lower product reads v_{t-1} in that order (float4 loads).
// Threads past the last knot idle on knot 0 (their F^ v reads knot K, zero) with zero
// coefficients, store nothing and add zeros to the reductions.  Everything else (scaling, FP64
// residual replacement, stall detection, hand-over to the FP64 recurrence, stopping test) follows
// pcg_rows_scaled line by line.
template <int NX, int TPK>
__device__ __noinline__ PcgOut pcg_rows_t(const Inst& s, double* lam, float* vec, int max_iter, double eps,
                                          int max_ref, double upd_rel, double* red, int& par_io) {
  int par = par_io;  // the reduction parity in a register; written back on every return
  constexpr int R = 4;
  constexpr int PD = R * TPK;  // padded rows / columns of a knot, the segment stride of the vectors
  constexpr int LD = pad_ld(NX);
  constexpr int BS = NX * LD;
  static_assert(NX <= PD && (TPK == 1 || TPK == 2 || TPK == 4), "row layout");
  const int K = s.K, N = s.N;
  const int span = (K + 2) * PD;
  float* rbase = as_shared(vec);  // four vectors of K + 2 segments: knots -1 .. K
  float* rv = rbase + PD;
  float* pv = rv + span;
  float* upr = pv + span;  // upr / upp segment t: (W_{t+1}^T v_{t+1}) for knot t's rows
  float* upp = upr + span;
  red = as_shared(red);
  const int lane_q = threadIdx.x % TPK;
  const bool ok = (int)threadIdx.x < TPK * K;
  const int q = ok ? lane_q : 0;
  const int tc = ok ? (int)threadIdx.x / TPK : 0;
  // the knot an idle thread's F^ reads: K, whose upper-term segment is never written (zero), and
  // whose lower term meets the thread's zero coefficients, so its F^ v is zero without a select
  const int tp = ok ? tc : K;
  auto row = [&](int k) { return R * q + k; };
  auto has = [&](int k) { return ok && R * q + k < NX; };
  auto cgrp = [&](int g) { return g ^ (TPK - 1 - lane_q); };  // column group of register group g
  for (int w = threadIdx.x; w < 4 * span; w += blockDim.x) rbase[w] = 0.f;
  // v_t rows (own) -> v store and the upper term for knot t-1 (before the barrier)
  auto push = [&](const float (&w)[R][PD], const float* x, float* v, float* up) {
    float c[PD];
#pragma unroll
    for (int m = 0; m < PD; ++m) c[m] = 0.f;
#pragma unroll
    for (int k = 0; k < R; ++k)
#pragma unroll
      for (int m = 0; m < PD; ++m) c[m] = fmaf(w[k][m], x[k], c[m]);
    float y[R];
    if constexpr (TPK == 4) {
      float h[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) h[j] = c[8 + j] + __shfl_xor_sync(DMPC_FULL_MASK, c[j], 2);
#pragma unroll
      for (int j = 0; j < 4; ++j) y[j] = h[4 + j] + __shfl_xor_sync(DMPC_FULL_MASK, h[j], 1);
    } else if constexpr (TPK == 2) {
#pragma unroll
      for (int j = 0; j < 4; ++j) y[j] = c[4 + j] + __shfl_xor_sync(DMPC_FULL_MASK, c[j], 1);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) y[j] = c[j];
    }
    if (ok) {
      *reinterpret_cast<float4*>(v + tc * PD + R * q) = make_float4(x[0], x[1], x[2], x[3]);
      *reinterpret_cast<float4*>(up + (tc - 1) * PD + R * q) = make_float4(y[0], y[1], y[2], y[3]);
    }
  };
  // (F^ v) for the thread's rows after the barrier: lower term from v_{t-1}, upper from `up`
  auto pull = [&](const float (&w)[R][PD], const float* v, const float* up, float* f) {
    float a[R], b[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      a[k] = 0.f;
      b[k] = 0.f;
    }
    const float* vm = v + (tp - 1) * PD;
#pragma unroll
    for (int g = 0; g < TPK; ++g) {
      const float4 y = *reinterpret_cast<const float4*>(vm + 4 * cgrp(g));
#pragma unroll
      for (int k = 0; k < R; ++k) {
        a[k] = fmaf(w[k][4 * g], y.x, a[k]);
        b[k] = fmaf(w[k][4 * g + 1], y.y, b[k]);
        a[k] = fmaf(w[k][4 * g + 2], y.z, a[k]);
        b[k] = fmaf(w[k][4 * g + 3], y.w, b[k]);
      }
    }
    const float4 u = *reinterpret_cast<const float4*>(up + tp * PD + R * q);
    f[0] = a[0] + b[0] + u.x;
    f[1] = a[1] + b[1] + u.y;
    f[2] = a[2] + b[2] + u.z;
    f[3] = a[3] + b[3] + u.w;
  };
  // rows past NX and idle threads hold exact zeros in every FP32 vector (set so at the start and
  // kept by the recurrences, whose operator terms vanish there), so a dot product needs no mask
  auto dot32 = [&](const float* a, const float* b) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < R; ++k) acc = fmaf(a[k], b[k], acc);
    return acc;
  };
  // FP64 exchange vector (knots -1..K) after the four FP32 vectors, then the solve's constants
  auto x64_of = [&]() { return reinterpret_cast<double*>(as_shared(vec + 4 * span)) + NX; };
  {
    double* x64 = x64_of();
    for (int w = threadIdx.x; w < NX; w += blockDim.x) {
      x64[w - NX] = 0.0;
      x64[K * NX + w] = 0.0;
    }
  }
  auto eta_of = [&](const double* rh, double* zh) -> double {
    double* x64 = x64_of();
    __syncthreads();
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (has(k)) x64[tc * NX + row(k)] = rh[k];
    __syncthreads();
    const RowVals<NX, R> h = fhat64_rows<NX, R, true>(s.pm, N, tc, q, x64);
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      zh[k] = rh[k] - h.v[k];
      if (has(k)) e += rh[k] * zh[k];
    }
    return e;
  };
  auto flush = [&]() {
    double* acc = s.tmp;
    __syncthreads();
    double l[R];
#pragma unroll
    for (int k = 0; k < R; ++k) l[k] = lower_col_t<NX>(s.li, tc, has(k) ? row(k) : q, acc + tc * NX);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (has(k)) {
        lam[tc * NX + row(k)] += l[k];
        acc[tc * NX + row(k)] = 0.0;
      }
    __syncthreads();
  };
  // W_t rows 4q..4q+3 in register-group order (block t-1 of w32; block N is zero and stands in
  // for W_0); zero past NX and on idle threads
  auto load_w = [&](float (&w)[R][PD]) {
    const float* wb = s.w32 + (tc > 0 ? tc - 1 : N) * BS;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int i = R * q + k;
#pragma unroll
      for (int g = 0; g < TPK; ++g)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const int c = 4 * cgrp(g) + kk;
          w[k][4 * g + kk] = (ok && i < NX && c < NX) ? wb[i * LD + c] : 0.f;
        }
    }
  };
  float r[R], p[R], d[R], f[R];
  int it = 0;
  double eta;
  float trig, hi;
  {
    double rh[R], zh[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      d[k] = 0.f;
      if (has(k)) s.tmp[tc * NX + row(k)] = 0.0;
    }
    exact_rhat_rows<NX, R, true>(s, lam, tc, q, ok, N);
#pragma unroll
    for (int k = 0; k < R; ++k) rh[k] = has(k) ? s.t1[tc * NX + row(k)] : 0.0;
    const double eta64 = block_sum2(eta_of(rh, zh), red, par);
    if (!(eta64 == eta64)) {
      par_io = par;
      return PcgOut{it, eta64};
    }
    const double scale = (eta64 > 0.0) ? rsqrt(eta64) : 1.0;
    double* cst = x64_of() + (K + 1) * NX;
    if (threadIdx.x == 0) {
      cst[0] = scale;
      cst[1] = (eta64 > 0.0) ? sqrt(eta64) : 1.0;
      cst[2] = scale * scale;
      cst[3] = eps * scale * scale * kCheckMargin;
      cst[4] = eta64;
      cst[5] = eta64 * scale * scale;
      cst[6] = eps;
      cst[7] = upd_rel;
      cst[8] = (double)max_ref;
      cst[9] = 0.0;
      cst[10] = (double)max_iter;
      cst[11] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
      r[k] = has(k) ? (float)(scale * rh[k]) : 0.f;
      p[k] = has(k) ? (float)(scale * zh[k]) : 0.f;
    }
    eta = eta64 * scale * scale;
    trig = (float)fmax(eps * scale * scale * kCheckMargin, upd_rel * eta);
    hi = (float)(kDivergeRatio * eta);
  }
  int it_stop = min(max_iter / 2, kStallMin);
  int nrep_out;
  double eta64 = 0.0;
  for (;;) {
    double vden, etap;
    float z[R];
    {
      float w[R][PD];
      load_w(w);
      // p^ and its upper term: the first segment's, or p after a replacement
      __syncthreads();
      push(w, p, pv, upp);
      __syncthreads();
      for (;;) {
        // u^ = S^ p^ = -(p^ + F^ p^)
        float u[R];
        pull(w, pv, upp, f);
#pragma unroll
        for (int k = 0; k < R; ++k) u[k] = -(p[k] + f[k]);
        vden = block_sum_f32b(dot32(p, u), red, par);
        const float alpha = quot32(eta, vden);
#pragma unroll
        for (int k = 0; k < R; ++k) {
          d[k] = fmaf(alpha, p[k], d[k]);
          r[k] = fmaf(-alpha, u[k], r[k]);
        }
        push(w, r, rv, upr);
        __syncthreads();
        // z^ = Phi^ r^ = r^ - F^ r^
        pull(w, rv, upr, f);
#pragma unroll
        for (int k = 0; k < R; ++k) z[k] = r[k] - f[k];
        etap = block_sum_f32b(dot32(r, z), red, par);
        ++it;
        const float etaf = (float)etap;
        if (!(etaf > trig) || etaf > hi || it >= it_stop || !(vden == vden)) break;
        const float beta = quot32(etap, eta);
#pragma unroll
        for (int k = 0; k < R; ++k) p[k] = fmaf(beta, p[k], z[k]);
        push(w, p, pv, upp);
        eta = etap;
        __syncthreads();
      }
    }
    {
      // Residual replacement, as in pcg_rows_scaled.
      double* cst = x64_of() + (K + 1) * NX;
      double* acc = s.tmp;
      const double scale = cst[0], back = cst[1], s2 = cst[2], check_at = cst[3], prev64 = cst[4],
                   eta_upd = cst[5], c_eps = cst[6], c_upd = cst[7];
      const int c_maxref = (int)cst[8], nupd = (int)cst[9] + 1, c_maxit = (int)cst[10], it_cap = c_maxit / 2;
      const bool bad = !(etap == etap) || !(vden == vden);
      const bool at_check = etap <= check_at;
      const bool fell = etap <= c_upd * eta_upd || (float)etap > hi;
      const bool cut = !fell && it >= it_stop && it < it_cap;
      const bool progressed = fell || cut;
      double a[R];
#pragma unroll
      for (int k = 0; k < R; ++k) {
        a[k] = has(k) ? acc[tc * NX + row(k)] : 0.0;
        if (!bad) {
          a[k] += back * (double)d[k];
          if (has(k)) acc[tc * NX + row(k)] = a[k];
        }
        d[k] = 0.f;
      }
      double rh[R], zh[R];
      bool exact = bad || at_check || it >= it_cap;
      if (!exact) {
        double* x64 = x64_of();
        __syncthreads();
#pragma unroll
        for (int k = 0; k < R; ++k)
          if (has(k)) x64[tc * NX + row(k)] = a[k];
        __syncthreads();
        const RowVals<NX, R> h = fhat64_rows<NX, R, true>(s.pm, N, tc, q, x64);
#pragma unroll
        for (int k = 0; k < R; ++k) rh[k] = has(k) ? s.t1[tc * NX + row(k)] + a[k] + h.v[k] : 0.0;
        eta64 = block_sum2(eta_of(rh, zh), red, par);
        exact = !(eta64 > c_eps);
      }
      if (exact) {
        flush();
        exact_rhat_rows<NX, R, true>(s, lam, tc, q, ok, N);
#pragma unroll
        for (int k = 0; k < R; ++k) rh[k] = has(k) ? s.t1[tc * NX + row(k)] : 0.0;
        eta64 = block_sum2(eta_of(rh, zh), red, par);
      }
      if (!(fabs(eta64) > c_eps && it <= c_maxit - 1) || !(eta64 == eta64)) {
        if (!exact) flush();
        nrep_out = nupd;
        break;
      }
      const double etas = eta64 * s2;
      if (bad || nupd >= c_maxref || it >= it_cap || !(etas > 0.0) ||
          (progressed && !at_check && eta64 > (cut ? c_upd : kUpdateStagnation) * prev64)) {
        if (!exact) flush();
        par_io = par;
        return fp64_finish(s, lam, it, c_maxit, c_eps, red, par_io, nupd);
      }
      it_stop = next_stop(it, it - (int)cst[11], it_cap);
      __syncthreads();
      if (threadIdx.x == 0) {
        cst[4] = eta64;
        cst[5] = etas;
        cst[9] = (double)nupd;
        cst[11] = (double)it;
      }
#pragma unroll
      for (int k = 0; k < R; ++k) {
        r[k] = has(k) ? (float)(scale * rh[k]) : 0.f;
        z[k] = has(k) ? (float)(scale * zh[k]) : 0.f;
      }
      if (etas > kRestartRatio * eta) {
#pragma unroll
        for (int k = 0; k < R; ++k) p[k] = 0.f;
      }
      etap = etas;
      trig = (float)fmax(check_at, c_upd * etas);
      hi = (float)(kDivergeRatio * etas);
    }
    const float beta = quot32(etap, eta);
#pragma unroll
    for (int k = 0; k < R; ++k) p[k] = fmaf(beta, p[k], z[k]);
    eta = etap;
  }
  par_io = par;
  return PcgOut{it, eta64, nrep_out};
}


// ---------------------------------------------------------------- recovery (pcg.py:290-348)
// x_t = -Qi_t (q_t + An_{t-1}^T lam_t + A_t^T lam_{t+1}), An_{-1} = I, An = -I;
// u_t = -Ri_t (r_t + B_t^T lam_{t+1}); u_N = 0.
__device__ void recover(const Inst& s, const double* lam, const double* q, const double* r, double* xo,
                        double* uo, int ustride_rows) {
  const int nx = s.nx, nu = s.nu, N = s.N;
  for (int w = threadIdx.x; w < s.K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    double a = q[w] + ((t == 0) ? lam[w] : -lam[w]);
    if (t < N) {
      const double* Ac = s.A + (size_t)t * nx * nx + i;
      const double* ln = lam + (t + 1) * nx;
      double b = 0.0;
      for (int j = 0; j < nx; ++j) b += Ac[(size_t)j * nx] * ln[j];
      a += b;
    }
    xo[w] = -s.Qi[w] * a;
  }
  for (int w = threadIdx.x; w < ustride_rows * nu; w += blockDim.x) {
    const int t = w / nu, i = w - t * nu;
    if (t >= N) {
      uo[w] = 0.0;
      continue;
    }
    const double* Bc = s.Bm + (size_t)t * nx * nu + i;
    const double* ln = lam + (t + 1) * nx;
    double b = 0.0;
    for (int j = 0; j < nx; ++j) b += Bc[(size_t)j * nu] * ln[j];
    uo[w] = -s.Ri[w] * (r[w] + b);
  }
}

// ---------------------------------------------------------------- line search (sqp.py:301-411)
__device__ double stage_cost(const Inst& s, const double* x, const double* u) {
  // per-thread partial of the reference cost (optimal_control_problem.py:208-247)
  const int nx = s.nx, nu = s.nu, N = s.N;
  double c = 0.0;
  for (int w = threadIdx.x; w < s.K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    double d, wt;
    if (t < N) {
      d = x[w] - s.xref[t * nx + i];
      wt = s.wx[i];
    } else {
      d = x[w] - s.xf[i];
      wt = s.wx[i] + s.wf[i];
    }
    c += wt * d * d;
  }
  for (int w = threadIdx.x; w < N * nu; w += blockDim.x) {
    const int t = w / nu, i = w - t * nu;
    const double d = u[w] - (s.pen ? s.uref[t * nu + i] : 0.0);
    c += s.wu[i] * d * d;
  }
  return c;
}

// returns the chosen alpha and overwrites xn/un with x + alpha (xn - x)
__device__ __noinline__ double linesearch(const Inst& s, const dmpc_solver_params& P, const double* xb, const double* ub,
                             double* xn, double* un, double* red, int& par, double* sh_dv) {
  const int nx = s.nx, nu = s.nu, N = s.N, K = s.K;
  // cost, directional derivative and constraint l1 at the current iterate
  double c = stage_cost(s, xb, ub);
  double cd = 0.0;
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    const double h = (t < N) ? 2.0 * s.wx[i] : 2.0 * (s.wx[i] + s.wf[i]);
    const double ref = (t < N) ? s.xref[t * nx + i] : s.xf[i];
    cd += h * (xb[w] - ref) * (xn[w] - xb[w]);
  }
  for (int w = threadIdx.x; w < N * nu; w += blockDim.x) {
    const int t = w / nu, i = w - t * nu;
    const double ref = s.pen ? s.uref[t * nu + i] : 0.0;
    cd += 2.0 * s.wu[i] * (ub[w] - ref) * (un[w] - ub[w]);
  }
  double l1 = 0.0;
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    l1 += fabs((t == 0) ? (xb[i] - s.x0[i]) : (s.fv[(t - 1) * nx + i] - xb[w]));
  }
  const double cost = block_sum(c, red, par);
  const double cdz = block_sum(cd, red, par);
  const double l1n = block_sum(l1, red, par);
  const double mu_min = cdz / (0.5 * l1n);
  const double mu = (mu_min != mu_min) ? mu_min : fmax(0.1, mu_min);
  const double merit = cost + mu * l1n;
  const double merit_d = cdz + -mu * l1n;
  const int na = P.n_alphas;
  for (int a = 0; a < na; ++a) {
    const double alpha = P.alphas[a];
    double cc = 0.0, ll = 0.0;
    // candidate cost
    for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
      const int t = w / nx, i = w - t * nx;
      const double x = xb[w] + alpha * (xn[w] - xb[w]);
      const double d = x - ((t < N) ? s.xref[t * nx + i] : s.xf[i]);
      cc += ((t < N) ? s.wx[i] : (s.wx[i] + s.wf[i])) * d * d;
      if (t == 0) ll += fabs(x - s.x0[i]);
    }
    for (int w = threadIdx.x; w < N * nu; w += blockDim.x) {
      const int t = w / nu, i = w - t * nu;
      const double u = ub[w] + alpha * (un[w] - ub[w]);
      const double d = u - (s.pen ? s.uref[t * nu + i] : 0.0);
      cc += s.wu[i] * d * d;
    }
    // candidate dynamics defects: one integrator step per stage
    for (int t = threadIdx.x; t < N; t += blockDim.x) {
      double x[DMPC_MAX_NX], u[DMPC_MAX_NU], f[DMPC_MAX_NX];
      for (int i = 0; i < nx; ++i) x[i] = xb[t * nx + i] + alpha * (xn[t * nx + i] - xb[t * nx + i]);
      for (int i = 0; i < nu; ++i) u[i] = ub[t * nu + i] + alpha * (un[t * nu + i] - ub[t * nu + i]);
      next_state_value(s, x, u, f);
      for (int i = 0; i < nx; ++i) {
        const int w = (t + 1) * nx + i;
        ll += fabs(f[i] - (xb[w] + alpha * (xn[w] - xb[w])));
      }
    }
    const double ccs = block_sum(cc, red, par);
    const double lls = block_sum(ll, red, par);
    if (threadIdx.x == 0) sh_dv[a] = ccs + mu * lls - (merit + P.linesearch_eta * alpha * merit_d);
  }
  __syncthreads();
  // while_loop from index n+1 downwards with clamped gathers (sqp.py:389-403)
  auto clampi = [&](int i) { return i < 0 ? 0 : (i > na - 1 ? na - 1 : i); };
  double amax = P.alphas[0];
  for (int a = 1; a < na; ++a) amax = fmax(amax, P.alphas[a]);
  int i = na + 1;
  double alpha = amax;
  while (!(sh_dv[clampi(i)] < 0.0 || i == 0)) {
    i = i - 1;
    alpha = P.alphas[clampi(i)];
  }
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) xn[w] = xb[w] + alpha * (xn[w] - xb[w]);
  for (int w = threadIdx.x; w < K * nu; w += blockDim.x) un[w] = ub[w] + alpha * (un[w] - ub[w]);
  __syncthreads();
  return alpha;
}

// ---------------------------------------------------------------- persistent work distribution
#if DMPC_CFG == 3
#define DMPC_SQP_BOUNDS __launch_bounds__(384, 1)
#elif DMPC_CFG == 2
#define DMPC_SQP_BOUNDS __launch_bounds__(256, 2)
#elif DMPC_CFG == 1
#define DMPC_SQP_BOUNDS __launch_bounds__(256, 1)
#else
#define DMPC_SQP_BOUNDS __launch_bounds__(512, 1)
#endif

// Group and instance of work item `item` (groups occupy contiguous ranges of the work order).
__device__ inline bool locate(const DevArgs& args, int item, int& gi, int& ii) {
  for (int g = 0; g < args.n_groups; ++g) {
    const int first = args.grp[g].first_item;
    if (item >= first && item < first + args.grp[g].g.batch) {
      gi = g;
      ii = item - first;
      return true;
    }
  }
  return false;
}

// The next work item of this CTA from the launch's counter (the first word of the workspace,
// zeroed on the stream before the launch), broadcast to the CTA; false once every item is
// handed out.  Starts with a barrier, so the previous item is finished by every thread before
// its shared state is reused.
__device__ inline bool next_item(const DevArgs& args, void* ws, int& gi, int& ii) {
  __shared__ int sh_item;
  __syncthreads();
  if (threadIdx.x == 0) sh_item = (int)atomicAdd(reinterpret_cast<unsigned int*>(ws), 1u);
  __syncthreads();
  const int item = sh_item;
  if (item >= args.total_items) return false;
  return locate(args, item, gi, ii);
}

// This CTA's workspace slot.
__device__ inline void* slot_of(const DevArgs& args, void* ws) {
  return reinterpret_cast<unsigned char*>(ws) + kQueueBytes + (size_t)blockIdx.x * args.slot_stride;
}

__device__ inline double nan0(double v) {
  // jnp.nan_to_num: NaN -> 0, +-inf -> +-max double
  if (v != v) return 0.0;
  if (v == __longlong_as_double(0x7ff0000000000000ll)) return 1.7976931348623157e308;
  if (v == __longlong_as_double(0xfff0000000000000ll)) return -1.7976931348623157e308;
  return v;
}

struct SmemView {
  double* red;
  double* dvals;  // line-search decrease values
  void* vec;      // PCG vectors
  float* blocks;  // FP32 blocks (if in smem)
};

__device__ inline SmemView carve_smem(unsigned char* sm, int nx, int K, int precision) {
  SmemView v;
  v.red = reinterpret_cast<double*>(sm);
  v.dvals = v.red + 128;
  unsigned char* p = sm + 136 * sizeof(double);
  v.vec = p;
  v.blocks = reinterpret_cast<float*>(p + pcg_vec_bytes(nx, K, precision, DMPC_CFG));
  return v;
}

// Solve the QP assembled in the workspace; lam (FP64 vector) in/out.
__device__ PcgOut solve_qp(const Inst& s, const dmpc_solver_params& P, SmemView& sv, double* lam, int& par) {
  const int n = s.K * s.nx;
  if (P.precision == DMPC_PREC_FP64) {
    double* v = reinterpret_cast<double*>(sv.vec);
    double *lv = v, *rv = v + n, *pv = v + 2 * n, *tv = v + 3 * n, *uv = v + 4 * n;
    for (int g = threadIdx.x; g < n; g += blockDim.x) lv[g] = lam[g];
    __syncthreads();
    PcgOut o = pcg_fp64(s, lv, rv, pv, tv, uv, P.pcg_max_iter, P.pcg_tol_epsilon, sv.red, par);
    for (int g = threadIdx.x; g < n; g += blockDim.x) lam[g] = lv[g];
    __syncthreads();
    o.it64 = o.it;
    return o;
  }
  float* v = reinterpret_cast<float*>(sv.vec);
  if (sh_scaled_bad) return fp64_finish(s, lam, 0, P.pcg_max_iter, P.pcg_tol_epsilon, sv.red, par, 0);
#if DMPC_CFG == 2
  // two CTAs per SM: the row PCG with one register copy of each W block
  if (s.K * rows_tpk(s.nx) <= (int)blockDim.x) {
    switch (s.nx) {
#define DMPC_ROWS_T(NXV)                                                                                   \
  case NXV:                                                                                                \
    return pcg_rows_t<NXV, rows_tpk(NXV)>(s, lam, v, P.pcg_max_iter, P.pcg_tol_epsilon, P.max_refinement, \
                                          P.inner_rel_tol, sv.red, par);
      DMPC_ROWS_T(3)
      DMPC_ROWS_T(4)
      DMPC_ROWS_T(6)
      DMPC_ROWS_T(7)
      DMPC_ROWS_T(8)
      DMPC_ROWS_T(12)
      DMPC_ROWS_T(13)
#undef DMPC_ROWS_T
      default: break;
    }
  }
#else
  if (s.K * ((s.nx + 3) / 4) <= (int)blockDim.x) {
    switch (s.nx) {
#define DMPC_ROWS(NXV)                                                                                   \
  case NXV:                                                                                              \
    return pcg_rows_scaled<NXV, 4>(s, lam, v, P.pcg_max_iter, P.pcg_tol_epsilon, P.max_refinement,       \
                                   P.inner_rel_tol, sv.red, par);
      DMPC_ROWS(3)
      DMPC_ROWS(4)
      DMPC_ROWS(6)
      DMPC_ROWS(7)
      DMPC_ROWS(8)
      DMPC_ROWS(12)
      DMPC_ROWS(13)
#undef DMPC_ROWS
      default: break;
    }
  }
#endif
  return pcg_mixed_scaled(s, lam, v, P.pcg_max_iter, P.pcg_tol_epsilon, P.max_refinement, P.inner_rel_tol,
                          sv.red, par);
}

// ---------------------------------------------------------------- forward kernel
// The SQP loop of one instance (sqp.py:436-560): initial guess from g's states/controls/
// dual, solution, status and histories back into g.  Called once per CTA by k_sqp_fwd and
// once per simulation step by k_rollout_fwd.
__device__ __forceinline__ void sqp_forward(const DevGroup& G, const dmpc_group& g, int ii,
                                            const dmpc_solver_params& P, void* ws, unsigned char* smem) {
  SmemView sv = carve_smem(smem, g.nx, G.K, P.precision);
  __shared__ Inst sh_inst;  // per-instance context in shared memory: keeps ~70 pointer registers free
  if (threadIdx.x == 0) sh_inst = make_inst(G, g, ii, ws, sv.blocks);
  __syncthreads();
  const Inst& s = sh_inst;
  if (s.N < 1 || s.N > g.horizon) {
    // per-instance horizon outside [1, horizon]: reported, not solved (the host does not read
    // the horizons back, so the check lives here)
    if (threadIdx.x == 0) {
      g.status[ii] = DMPC_STATUS_ERROR;
      g.num_iter[ii] = 0;
      g.convergence_error[ii] = __longlong_as_double(0x7ff8000000000000ll);
    }
    return;
  }
  const int nx = s.nx, nu = s.nu, Kmax = G.K, K = s.K;
  const int maxit = P.num_scp_iteration_max;
  double* gx = g.states + (size_t)ii * Kmax * nx;
  double* gu = g.controls + (size_t)ii * Kmax * nu;
  double* gl = g.dual + (size_t)ii * Kmax * nx;
  int par = 0;
  // initial guess -> workspace
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    s.xb[w] = gx[w];
    s.lam[w] = gl[w];
  }
  for (int w = threadIdx.x; w < K * nu; w += blockDim.x) s.ub[w] = gu[w];
  __syncthreads();
  double conv_err = g.convergence_error[ii];
  int num_iter = 0;
  const double tol = P.tol_convergence;
  while ((num_iter < maxit && conv_err > tol) || num_iter < 1) {
    // remember the linearization point of this iteration (used by the adjoint)
    for (int w = threadIdx.x; w < K * nx; w += blockDim.x) g.lin_states[(size_t)ii * Kmax * nx + w] = s.xb[w];
    for (int w = threadIdx.x; w < K * nu; w += blockDim.x) g.lin_controls[(size_t)ii * Kmax * nu + w] = s.ub[w];
    linearize_dynamics(s, s.xb, s.ub);
    linearize_cost(s, s.xb, s.ub);
    __syncthreads();
    assemble_schur(s, P.precision != DMPC_PREC_FP64);
    compute_gamma(s, s.C, s.q, s.r);
    __syncthreads();
    PcgOut o = solve_qp(s, P, sv, s.lam, par);
    recover(s, s.lam, s.q, s.r, s.xn, s.un, K);
    __syncthreads();
    double alpha = 0.0;
    if (P.linesearch) alpha = linesearch(s, P, s.xb, s.ub, s.xn, s.un, sv.red, par, sv.dvals);
    double e = 0.0;
    for (int w = threadIdx.x; w < K * nx; w += blockDim.x) e = fmax(e, fabs(s.xn[w] - s.xb[w]));
    for (int w = threadIdx.x; w < K * nu; w += blockDim.x) e = fmax(e, fabs(s.un[w] - s.ub[w]));
    // NaN-propagating max like jnp.max
    {
      double ee = 0.0;
      bool nan = false;
      for (int w = threadIdx.x; w < K * nx; w += blockDim.x) nan |= (s.xn[w] != s.xn[w]) || (s.xb[w] != s.xb[w]);
      for (int w = threadIdx.x; w < K * nu; w += blockDim.x) nan |= (s.un[w] != s.un[w]) || (s.ub[w] != s.ub[w]);
      ee = nan ? __longlong_as_double(0x7ff8000000000000ll) : e;
      conv_err = block_max(ee, sv.red, par);
    }
    if (threadIdx.x == 0 && num_iter < maxit) {
      g.convergence_errors[(size_t)ii * maxit + num_iter] = conv_err;
      g.num_pcg_iters[(size_t)ii * maxit + num_iter] = o.it;
      if (g.num_pcg_corrections) g.num_pcg_corrections[(size_t)ii * maxit + num_iter] = o.nrep;
      if (g.num_pcg_fp64_iters) g.num_pcg_fp64_iters[(size_t)ii * maxit + num_iter] = o.it64;
      if (P.linesearch) g.linesearch_alphas[(size_t)ii * maxit + num_iter] = alpha;
    }
    for (int w = threadIdx.x; w < K * nx; w += blockDim.x) s.xb[w] = s.xn[w];
    for (int w = threadIdx.x; w < K * nu; w += blockDim.x) s.ub[w] = s.un[w];
    ++num_iter;
    __syncthreads();
  }
  // status + nan_to_num (sqp.py:535-559)
  bool nan = false;
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) nan |= (s.xb[w] != s.xb[w]);
  for (int w = threadIdx.x; w < K * nu; w += blockDim.x) nan |= (s.ub[w] != s.ub[w]);
  const int anynan = __syncthreads_or(nan ? 1 : 0);
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    gx[w] = nan0(s.xb[w]);
    gl[w] = nan0(s.lam[w]);
  }
  for (int w = threadIdx.x; w < K * nu; w += blockDim.x) gu[w] = nan0(s.ub[w]);
  if (threadIdx.x == 0) {
    g.status[ii] = (anynan || conv_err > tol || conv_err != conv_err) ? DMPC_STATUS_ERROR : DMPC_STATUS_SUCCESS;
    g.num_iter[ii] = num_iter;
    g.convergence_error[ii] = conv_err;
  }
}

__global__ void DMPC_SQP_BOUNDS k_sqp_fwd(const __grid_constant__ DevArgs args, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  void* slot = slot_of(args, ws);
  int gi, ii;
  while (next_item(args, ws, gi, ii)) {
    const DevGroup& G = args.grp[gi];
    sqp_forward(G, G.g, ii, args.p, slot, smem);
  }
}

// ---------------------------------------------------------------- closed-loop rollout
// One integrator step of the instance's model as the rollout's simulator (s.scheme: Euler
// for DMPC_SIM_MODEL, the group's scheme for DMPC_SIM_MODEL_SCHEME): sum_i lam_i d(x+_i)/dz_d
// for the direction z_d of (x, u) (d < nx: state, else control), by one Dual evaluation.
template <int MODEL>
__device__ __noinline__ double sim_vjp_item(const Inst& s, const double* x, const double* u, const double* lam, int d) {
  constexpr int MX = ModelDims<MODEL>::NX, MU = ModelDims<MODEL>::NU;
  const int nx = MODEL == DMPC_MODEL_LINEAR ? s.nx : MX, nu = MODEL == DMPC_MODEL_LINEAR ? s.nu : MU;
  Dual xd[MX], ud[MU], xn[MX];
  for (int j = 0; j < nx; ++j) xd[j] = Dual(x[j], j == d ? 1.0 : 0.0);
  for (int j = 0; j < nu; ++j) ud[j] = Dual(u[j], nx + j == d ? 1.0 : 0.0);
  if (MODEL == DMPC_MODEL_LINEAR) {
    predict_next_state_linear(s, xd, ud, xn);
  } else {
    Dual p[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = Dual(k < s.P ? s.mp[k] : 0.0);
    predict_next_state<Dual, MODEL>(s.scheme, s.dt, nx, nu, xd, ud, p, xn);
  }
  double acc = 0.0;
  for (int i = 0; i < nx; ++i) acc += lam[i] * xn[i].d;
  return acc;
}

__device__ double sim_vjp(const Inst& s, const double* x, const double* u, const double* lam, int d) {
  switch (s.model) {
    case DMPC_MODEL_LINEAR: return sim_vjp_item<DMPC_MODEL_LINEAR>(s, x, u, lam, d);
    case DMPC_MODEL_QUADROTOR: return sim_vjp_item<DMPC_MODEL_QUADROTOR>(s, x, u, lam, d);
    case DMPC_MODEL_SPACECRAFT: return sim_vjp_item<DMPC_MODEL_SPACECRAFT>(s, x, u, lam, d);
    case DMPC_MODEL_ATTITUDE: return sim_vjp_item<DMPC_MODEL_ATTITUDE>(s, x, u, lam, d);
    case DMPC_MODEL_CARTPOLE: return sim_vjp_item<DMPC_MODEL_CARTPOLE>(s, x, u, lam, d);
  }
  return 0.0;
}

// The group as seen by simulation step k: initial state x_k, and solution, linearization
// point, status and histories in step k's slices of the rollout arrays.
__device__ inline dmpc_group rollout_step_view(const dmpc_group& g0, const dmpc_rollout& ra, int k, int Kmax, int mi) {
  const size_t B = g0.batch;
  const size_t sx = B * Kmax * g0.nx, su = B * Kmax * g0.nu, sh = B * mi;
  dmpc_group v = g0;
  v.initial_state = ra.step_initial_state + (size_t)k * B * g0.nx;
  v.states = ra.step_states + k * sx;
  v.controls = ra.step_controls + k * su;
  v.dual = ra.step_dual + k * sx;
  v.lin_states = ra.step_lin_states + k * sx;
  v.lin_controls = ra.step_lin_controls + k * su;
  v.status = ra.step_status + (size_t)k * B;
  v.num_iter = ra.step_num_iter + (size_t)k * B;
  v.convergence_error = ra.step_convergence_error + (size_t)k * B;
  v.convergence_errors = ra.step_convergence_errors + k * sh;
  v.linesearch_alphas = ra.step_linesearch_alphas + k * sh;
  v.num_pcg_iters = ra.step_num_pcg_iters + k * sh;
  v.num_pcg_corrections = nullptr;
  v.num_pcg_fp64_iters = nullptr;
  return v;
}

// benchmark_diffmpc.py:140-175 (lax.scan of rollout_step, vmapped over instances), one CTA
// per instance for all simulation steps: solve the MPC from x_k (warm-started from step
// k-1's solution, or from the initial guess), apply u_k = controls[0], simulate x_{k+1}
// (x_{k+1} = A x_k + B u_k + b, or an integrator step of the model as in
// spacecraft/benchmark_diffmpc.py:87-89) and add the weighted squared deviations of x_{k+1}
// and u_k.  Every
// step's solution and last linearization point are kept for the adjoint sweep.
__device__ __noinline__ void rollout_fwd_instance(const DevArgs& args, const dmpc_rollout& ra, int ii, void* ws,
                                                  unsigned char* smem) {
  const DevGroup& G = args.grp[0];
  const dmpc_group& g0 = G.g;
  const int nx = g0.nx, nu = g0.nu, Kmax = G.K, B = g0.batch;
  const int mi = args.p.num_scp_iteration_max;
  const size_t sx = (size_t)B * Kmax * nx, su = (size_t)B * Kmax * nu, sh = (size_t)B * mi;
  const size_t ox = (size_t)ii * Kmax * nx, ou = (size_t)ii * Kmax * nu, oh = (size_t)ii * mi;
  __shared__ dmpc_group sh_g;  // the group as seen by step k
  __shared__ double sh_cost;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) ra.step_initial_state[(size_t)ii * nx + i] = g0.initial_state[(size_t)ii * nx + i];
  if (threadIdx.x == 0) sh_cost = 0.0;
  for (int k = 0; k < ra.num_steps; ++k) {
    if (threadIdx.x == 0) sh_g = rollout_step_view(g0, ra, k, Kmax, mi);
    __syncthreads();
    // guess of step k: step k-1's solution (warm start) or the initial guess; the SQP
    // counter restarts either way (sqp.py:530-532)
    const bool warm = ra.warm_start && k > 0;
    const double* gsx = warm ? ra.step_states + (k - 1) * sx : g0.states;
    const double* gsu = warm ? ra.step_controls + (k - 1) * su : g0.controls;
    const double* gsl = warm ? ra.step_dual + (k - 1) * sx : g0.dual;
    for (int w = threadIdx.x; w < Kmax * nx; w += blockDim.x) {
      sh_g.states[ox + w] = gsx[ox + w];
      sh_g.dual[ox + w] = gsl[ox + w];
    }
    for (int w = threadIdx.x; w < Kmax * nu; w += blockDim.x) sh_g.controls[ou + w] = gsu[ou + w];
    const double* hce = warm ? ra.step_convergence_errors + (k - 1) * sh : g0.convergence_errors;
    const double* hal = warm ? ra.step_linesearch_alphas + (k - 1) * sh : g0.linesearch_alphas;
    const int32_t* hpc = warm ? ra.step_num_pcg_iters + (k - 1) * sh : g0.num_pcg_iters;
    for (int w = threadIdx.x; w < mi; w += blockDim.x) {
      sh_g.convergence_errors[oh + w] = hce[oh + w];
      sh_g.linesearch_alphas[oh + w] = hal[oh + w];
      sh_g.num_pcg_iters[oh + w] = hpc[oh + w];
    }
    if (threadIdx.x == 0)
      sh_g.convergence_error[ii] = warm ? ra.step_convergence_error[(size_t)(k - 1) * B + ii] : g0.convergence_error[ii];
    __syncthreads();
    sqp_forward(G, sh_g, ii, args.p, ws, smem);
    __syncthreads();
    // simulator step and running cost (the negated reward)
    const double* x = ra.step_initial_state + ((size_t)k * B + ii) * nx;
    const double* u = sh_g.controls + ou;  // controls[0]
    double* xn = ra.step_initial_state + ((size_t)(k + 1) * B + ii) * nx;
    if (ra.simulator != DMPC_SIM_LINEAR) {
      if (threadIdx.x == 0) {
        Inst se = make_inst(G, sh_g, ii, ws, nullptr);
        if (ra.simulator == DMPC_SIM_MODEL) se.scheme = DMPC_EULER;
        next_state_value(se, x, u, xn);
      }
    } else {
      const double* A = ra.sim_A + (size_t)ii * nx * nx;
      const double* Bm = ra.sim_B + (size_t)ii * nx * nu;
      for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        double a = ra.sim_b[(size_t)ii * nx + i];
        for (int j = 0; j < nx; ++j) a += A[i * nx + j] * x[j];
        for (int j = 0; j < nu; ++j) a += Bm[i * nu + j] * u[j];
        xn[i] = a;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double c = 0.0;
      for (int i = 0; i < nx; ++i) {
        const double d = xn[i] - (ra.cost_state_ref ? ra.cost_state_ref[i] : 0.0);
        c += ra.cost_state_weights[i] * d * d;
      }
      for (int j = 0; j < nu; ++j) {
        const double d = u[j] - (ra.cost_control_ref ? ra.cost_control_ref[j] : 0.0);
        c += ra.cost_control_weights[j] * d * d;
      }
      sh_cost += c;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) ra.running_cost[ii] = sh_cost;
}

__global__ void DMPC_SQP_BOUNDS k_rollout_fwd(const __grid_constant__ DevArgs args,
                                              const __grid_constant__ dmpc_rollout ra, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  void* slot = slot_of(args, ws);
  int gi, ii;
  while (next_item(args, ws, gi, ii)) rollout_fwd_instance(args, ra, ii, slot, smem);
}

// ---------------------------------------------------------------- adjoint kernel
// Hyper-dual evaluation for model-parameter gradients: the e1e2 part of
// lam*_{t+1} . F(z*_t + z~_t e1, theta + e_k e2) and the e2 part against lam~_{t+1}.
template <int MODEL>
__device__ __noinline__ double param_grad_item(const Inst& s, const double* xs, const double* us, const double* xt,
                                  const double* ut, const double* lstar, const double* ltil, int t, int k) {
  constexpr int MX = ModelDims<MODEL>::NX, MU = ModelDims<MODEL>::NU;
  const int nx = MODEL == DMPC_MODEL_LINEAR ? s.nx : MX, nu = MODEL == DMPC_MODEL_LINEAR ? s.nu : MU;
  HDual x[MX], u[MU], f[MX];
  for (int j = 0; j < nx; ++j) x[j] = HDual(xs[t * nx + j], xt[t * nx + j], 0.0, 0.0);
  for (int j = 0; j < nu; ++j) u[j] = HDual(us[t * nu + j], ut[t * nu + j], 0.0, 0.0);
  if (MODEL == DMPC_MODEL_LINEAR) {
    predict_next_state_linear<HDual>(s, x, u, f, k);
  } else {
    HDual p[12];  // compile-time trip count keeps p in registers; unused slots are zero
#pragma unroll
    for (int q = 0; q < 12; ++q) p[q] = HDual(q < s.P ? s.mp[q] : 0.0, 0.0, q == k ? 1.0 : 0.0, 0.0);
    predict_next_state<HDual, MODEL>(s.scheme, s.dt, nx, nu, x, u, p, f);
  }
  double acc = 0.0;
  for (int i = 0; i < nx; ++i) acc += lstar[(t + 1) * nx + i] * f[i].ab + ltil[(t + 1) * nx + i] * f[i].b;
  return acc;
}

// The adjoint of one instance's solve (sqp.py:668-798) at the linearization point saved in
// g.  With `acc`, the parameter gradients are added to the outputs (the rollout's sweep
// over its steps) instead of stored; a null dl_dstates stands for zeros.
__device__ __forceinline__ void sqp_adjoint(const DevGroup& G, const dmpc_group& g, const dmpc_adjoint& a, int ii,
                                            const dmpc_solver_params& P, void* ws, unsigned char* smem, bool acc) {
  SmemView sv = carve_smem(smem, g.nx, G.K, P.precision);
  __shared__ Inst sh_inst;  // per-instance context in shared memory: keeps ~70 pointer registers free
  if (threadIdx.x == 0) sh_inst = make_inst(G, g, ii, ws, sv.blocks);
  __syncthreads();
  const Inst& s = sh_inst;
  if (s.N < 1 || s.N > g.horizon) return;  // invalid horizon: the forward marked it ERROR
  const int nx = s.nx, nu = s.nu, Kmax = G.K, K = s.K, N = s.N;
  const size_t ox = (size_t)ii * Kmax * nx, ou = (size_t)ii * Kmax * nu;
  int par = 0;
  // linearization point of the last SQP iteration (sqp.py:761-763)
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) s.xb[w] = g.lin_states[ox + w];
  for (int w = threadIdx.x; w < K * nu; w += blockDim.x) s.ub[w] = g.lin_controls[ou + w];
  __syncthreads();
  linearize_dynamics(s, s.xb, s.ub);
  linearize_cost(s, s.xb, s.ub);
  // q = -dl/dx, r = -dl/du[:-1] (sqp.py:682-683)
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) s.q[w] = a.dl_dstates ? -a.dl_dstates[ox + w] : -0.0;
  for (int w = threadIdx.x; w < N * nu; w += blockDim.x) s.r[w] = -a.dl_dcontrols[ou + w];
  __syncthreads();
  assemble_schur(s, P.precision != DMPC_PREC_FP64);
  compute_gamma(s, nullptr, s.q, s.r);
  const bool warm = P.warm_start_backward && a.dual_backward_guess;
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) s.lam[w] = warm ? a.dual_backward_guess[ox + w] : 0.0;
  __syncthreads();
  PcgOut o = solve_qp(s, P, sv, s.lam, par);
  // adjoint states/controls (x~, u~)
  recover(s, s.lam, s.q, s.r, s.xn, s.un, K);
  __syncthreads();
  const double* xs = g.states + ox;  // z*, lambda* (post nan_to_num)
  const double* us = g.controls + ou;
  const double* ls = g.dual + ox;
  const double* xt = s.xn;
  const double* ut = s.un;
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    a.dual_backward[ox + w] = s.lam[w];
    if (a.adj_states) a.adj_states[ox + w] = xt[w];
  }
  if (a.adj_controls)
    for (int w = threadIdx.x; w < K * nu; w += blockDim.x) a.adj_controls[ou + w] = ut[w];
  if (threadIdx.x == 0) {
    if (a.num_pcg_iter) a.num_pcg_iter[ii] = o.it;
    if (a.num_pcg_corrections) a.num_pcg_corrections[ii] = o.nrep;
    if (a.num_pcg_fp64_iter) a.num_pcg_fp64_iter[ii] = o.it64;
  }
  // closed-form gradients of the cost-related parameters (sqp.py:605-666,724-739)
  const int j = threadIdx.x;
  if (j < nx) {
    double gwx = 0.0;
    for (int t = 0; t < N; ++t) gwx += 2.0 * (xs[t * nx + j] - s.xref[t * nx + j]) * xt[t * nx + j];
    const double dN = xs[N * nx + j] - s.xf[j];
    const double xtN = xt[N * nx + j];
    gwx += 2.0 * dN * xtN;
    const size_t o = (size_t)ii * nx + j;
    if (a.g_w_x) a.g_w_x[o] = (acc ? a.g_w_x[o] : 0.0) - gwx;
    if (a.g_w_f) a.g_w_f[o] = (acc ? a.g_w_f[o] : 0.0) - 2.0 * dN * xtN;
    if (a.g_initial_state) a.g_initial_state[o] = (acc ? a.g_initial_state[o] : 0.0) + s.lam[j];
    if (a.g_final_state) a.g_final_state[o] = (acc ? a.g_final_state[o] : 0.0) + 2.0 * (s.wx[j] + s.wf[j]) * xtN;
  } else if (j < nx + nu) {
    const int k = j - nx;
    double gwu = 0.0;
    for (int t = 0; t < N; ++t)
      gwu += 2.0 * (us[t * nu + k] - (s.pen ? s.uref[t * nu + k] : 0.0)) * ut[t * nu + k];
    const size_t o = (size_t)ii * nu + k;
    if (a.g_w_u) a.g_w_u[o] = (acc ? a.g_w_u[o] : 0.0) - gwu;
  }
  if (a.g_reference_state)
    for (int w = threadIdx.x; w < Kmax * nx; w += blockDim.x) {
      const int t = w / nx, i = w - t * nx;
      a.g_reference_state[ox + w] = (acc ? a.g_reference_state[ox + w] : 0.0) + ((t < N) ? 2.0 * s.wx[i] * xt[w] : 0.0);
    }
  if (a.g_reference_control)
    for (int w = threadIdx.x; w < Kmax * nu; w += blockDim.x) {
      const int t = w / nu, i = w - t * nu;
      a.g_reference_control[ou + w] = (acc ? a.g_reference_control[ou + w] : 0.0) + ((t < N && s.pen) ? 2.0 * s.wu[i] * ut[w] : 0.0);
    }
  // model parameters: hyper-dual mixed partials through the integrator
  const int ng = a.n_param_grads;
  if (ng > 0 && a.g_model_params) {
    for (int w = threadIdx.x; w < N * ng; w += blockDim.x) {
      const int t = w / ng, q = w - t * ng;
      const int k = G.pg_idx[q];
      double v = 0.0;
      switch (s.model) {
        case DMPC_MODEL_LINEAR: v = param_grad_item<DMPC_MODEL_LINEAR>(s, xs, us, xt, ut, ls, s.lam, t, k); break;
        case DMPC_MODEL_QUADROTOR: v = param_grad_item<DMPC_MODEL_QUADROTOR>(s, xs, us, xt, ut, ls, s.lam, t, k); break;
        case DMPC_MODEL_SPACECRAFT: v = param_grad_item<DMPC_MODEL_SPACECRAFT>(s, xs, us, xt, ut, ls, s.lam, t, k); break;
        case DMPC_MODEL_ATTITUDE: v = param_grad_item<DMPC_MODEL_ATTITUDE>(s, xs, us, xt, ut, ls, s.lam, t, k); break;
        case DMPC_MODEL_CARTPOLE: v = param_grad_item<DMPC_MODEL_CARTPOLE>(s, xs, us, xt, ut, ls, s.lam, t, k); break;
      }
      s.contrib[(size_t)q * K + t] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < ng; q += blockDim.x) {
      double sum = 0.0;
      for (int t = 0; t < N; ++t) sum += s.contrib[(size_t)q * K + t];
      a.g_model_params[(size_t)ii * ng + q] = (acc ? a.g_model_params[(size_t)ii * ng + q] : 0.0) - sum;
    }
  }
}

__global__ void DMPC_SQP_BOUNDS k_sqp_adj(const __grid_constant__ DevArgs args, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  void* slot = slot_of(args, ws);
  int gi, ii;
  while (next_item(args, ws, gi, ii)) {
    const DevGroup& G = args.grp[gi];
    sqp_adjoint(G, G.g, G.a, ii, args.p, slot, smem, false);
  }
}

// Reverse sweep of the rollout's gradient (what jax.grad of the reference's scan computes):
// with lam_T = c dcost/dx_T (c = dL/d running cost), F the simulator step, for k = T-1 .. 0
//   dl/du_0 of step k  = c dcost/du_k + (dF/du)^T lam_{k+1}
//   adjoint of step k's solve, parameter gradients accumulated into adj's outputs
//   lam_k = (dF/dx)^T lam_{k+1} + c dcost/dx_k (k >= 1) [+ the solve's dL/dx_0 if through_state]
// (dF/dz)^T lam is formed by one Dual evaluation per direction for the model simulator.
// and dL/dx_0 = lam_0.  One CTA per instance, all steps in one launch.
__device__ __noinline__ void rollout_adj_instance(const DevArgs& args, const dmpc_rollout& ra,
                                                  const dmpc_rollout_adjoint& rr, int ii, void* ws,
                                                  unsigned char* smem) {
  const DevGroup& G = args.grp[0];
  const dmpc_group& g0 = G.g;
  const int nx = g0.nx, nu = g0.nu, Kmax = G.K, B = g0.batch;
  const int mi = args.p.num_scp_iteration_max;
  const size_t ox = (size_t)ii * Kmax * nx, ou = (size_t)ii * Kmax * nu;
  __shared__ dmpc_group sh_g;
  __shared__ dmpc_adjoint sh_a;
  __shared__ double sh_lam[DMPC_MAX_NX], sh_vjp[DMPC_MAX_NX + DMPC_MAX_NU];
  const double c = rr.cost_cotangent[ii];
  const int T = ra.num_steps;
  // d cost / dx_k and d cost / du_k of the running cost's terms
  auto dcx = [&](const double* x, int i) {
    return 2.0 * c * ra.cost_state_weights[i] * (x[i] - (ra.cost_state_ref ? ra.cost_state_ref[i] : 0.0));
  };
  auto dcu = [&](const double* u, int j) {
    return 2.0 * c * ra.cost_control_weights[j] * (u[j] - (ra.cost_control_ref ? ra.cost_control_ref[j] : 0.0));
  };
  for (int i = threadIdx.x; i < nx; i += blockDim.x) sh_lam[i] = dcx(ra.step_initial_state + ((size_t)T * B + ii) * nx, i);
  for (int w = threadIdx.x; w < Kmax * nu; w += blockDim.x) rr.scratch_dl_dcontrols[ou + w] = 0.0;
  __syncthreads();
  for (int k = T - 1; k >= 0; --k) {
    if (threadIdx.x == 0) {
      sh_g = rollout_step_view(g0, ra, k, Kmax, mi);
      dmpc_adjoint a = G.a;
      a.dl_dstates = nullptr;
      a.dl_dcontrols = rr.scratch_dl_dcontrols;
      a.dual_backward_guess = nullptr;  // the carried solution's backward guess is zero
      a.dual_backward = rr.scratch_dual;
      a.num_pcg_iter = nullptr;
      a.num_pcg_corrections = nullptr;
      a.num_pcg_fp64_iter = nullptr;
      a.g_initial_state = nullptr;
      a.adj_states = nullptr;
      a.adj_controls = nullptr;
      sh_a = a;
    }
    __syncthreads();
    const double* u = sh_g.controls + ou;  // u_k = controls[0]
    const double* x = ra.step_initial_state + ((size_t)k * B + ii) * nx;
    // sh_vjp = [dx_{k+1}/dx_k, dx_{k+1}/du_k]^T lam_{k+1}
    if (ra.simulator != DMPC_SIM_LINEAR) {
      for (int d = threadIdx.x; d < nx + nu; d += blockDim.x) {
        Inst se = make_inst(G, sh_g, ii, ws, nullptr);
        if (ra.simulator == DMPC_SIM_MODEL) se.scheme = DMPC_EULER;
        sh_vjp[d] = sim_vjp(se, x, u, sh_lam, d);
      }
    } else {
      const double* A = ra.sim_A + (size_t)ii * nx * nx;
      const double* Bm = ra.sim_B + (size_t)ii * nx * nu;
      for (int d = threadIdx.x; d < nx + nu; d += blockDim.x) {
        double v = 0.0;
        if (d < nx)
          for (int j = 0; j < nx; ++j) v += A[j * nx + d] * sh_lam[j];
        else
          for (int i = 0; i < nx; ++i) v += Bm[i * nu + (d - nx)] * sh_lam[i];
        sh_vjp[d] = v;
      }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nu; j += blockDim.x) rr.scratch_dl_dcontrols[ou + j] = dcu(u, j) + sh_vjp[nx + j];
    __syncthreads();
    sqp_adjoint(G, sh_g, sh_a, ii, args.p, ws, smem, true);
    __syncthreads();
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      double v = sh_vjp[i];
      if (rr.through_state) v += rr.scratch_dual[ox + i];  // the solve's dL/dx_0 = lam~_0
      if (k >= 1) v += dcx(x, i);
      sh_lam[i] = v;
    }
    __syncthreads();
  }
  if (rr.g_initial_state)
    for (int i = threadIdx.x; i < nx; i += blockDim.x) rr.g_initial_state[(size_t)ii * nx + i] = sh_lam[i];
}

__global__ void DMPC_SQP_BOUNDS k_rollout_adj(const __grid_constant__ DevArgs args,
                                              const __grid_constant__ dmpc_rollout ra,
                                              const __grid_constant__ dmpc_rollout_adjoint rr, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  void* slot = slot_of(args, ws);
  int gi, ii;
  while (next_item(args, ws, gi, ii)) rollout_adj_instance(args, ra, rr, ii, slot, smem);
}

// dmpc_linearize: dense As, Bs, Cs, Qinv, qvec, Rinv, rvec of one group
#if DMPC_CFG == 0
__global__ void __launch_bounds__(256) k_linearize(const __grid_constant__ DevArgs args, void* ws, double* As,
                                                   double* Bs, double* Cs, double* Qinv, double* qv, double* Rinv,
                                                   double* rv) {
  void* slot = slot_of(args, ws);
  int gi, ii;
  while (next_item(args, ws, gi, ii)) {
  const DevGroup& G = args.grp[gi];
  const dmpc_group& g = G.g;
  Inst s = make_inst(G, g, ii, slot, nullptr);
  const int nx = s.nx, nu = s.nu, N = G.g.horizon, K = N + 1;
  const double* xb = g.states + (size_t)ii * K * nx;
  const double* ub = g.controls + (size_t)ii * K * nu;
  linearize_dynamics(s, xb, ub);
  linearize_cost(s, xb, ub);
  __syncthreads();
  for (int w = threadIdx.x; w < N * nx * nx; w += blockDim.x) As[(size_t)ii * N * nx * nx + w] = s.A[w];
  for (int w = threadIdx.x; w < N * nx * nu; w += blockDim.x) Bs[(size_t)ii * N * nx * nu + w] = s.Bm[w];
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    Cs[(size_t)ii * K * nx + w] = s.C[w];
    qv[(size_t)ii * K * nx + w] = s.q[w];
  }
  for (int w = threadIdx.x; w < K * nx * nx; w += blockDim.x) {
    const int t = w / (nx * nx), e = w - t * nx * nx, i = e / nx, j = e - i * nx;
    Qinv[(size_t)ii * K * nx * nx + w] = (i == j) ? s.Qi[t * nx + i] : 0.0;
  }
  for (int w = threadIdx.x; w < N * nu * nu; w += blockDim.x) {
    const int t = w / (nu * nu), e = w - t * nu * nu, i = e / nu, j = e - i * nu;
    Rinv[(size_t)ii * N * nu * nu + w] = (i == j) ? s.Ri[t * nu + i] : 0.0;
  }
  for (int w = threadIdx.x; w < N * nu; w += blockDim.x) rv[(size_t)ii * N * nu + w] = s.r[w];
  }
}
#endif

}  // namespace
}  // namespace dmpc_impl
