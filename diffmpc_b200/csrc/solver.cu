// Batched SQP + Schur-complement PCG solver and its adjoint for sm_100a.
//
// One CTA solves one instance from start to finish: the SQP loop of
// diffmpc/solvers/sqp.py:436-560 (linearize -> assemble S, Phi^-1, gamma ->
// PCG -> recover (x, u) -> optional line search -> convergence test) runs
// entirely on the device with per-instance early exit, and the adjoint
// (sqp.py:668-798) reuses the same building blocks.  The grid holds every
// instance of every group, so one launch solves a ragged, mixed-model batch and
// the hardware block scheduler balances uneven instances across the 148 SMs.
//
// Precision.  DMPC_PREC_FP64 runs the reference's FP64 PCG recurrence.
// DMPC_PREC_MIXED runs the PCG iterations in FP32 (dot products accumulated in
// FP64) in the basis scaled by the Cholesky factors of the diagonal blocks, where
// S and the block preconditioner Phi^-1 both reduce to the identity plus or minus
// one off-diagonal block per stage (see pcg_pair_scaled), and wraps them in FP64
// iterative refinement: the residual gamma - S lambda and the stopping test
// eta = r^T Phi^-1 r <= eps use the FP64 blocks, so the reference's absolute
// stopping rule (pcg.py:397-403) is applied in FP64.
//
// Storage of the Schur system (compact, symmetric block-tridiagonal):
//   S row t      = -[phi_{t-1}, theta_t, phi_t^T]          (pcg.py:198-211)
//   Phi^-1 row t =  [P_t, theta_t^-1, P_{t+1}^T],  P_t = -theta_t^-1 phi_{t-1} theta_{t-1}^-1
//                                                           (pcg.py:213-239)
// so each operator is one diagonal block per knot and one off-diagonal block per
// stage; the reference's third column block of Phi^-1 equals P_{t+1}^T because
// the theta blocks are symmetric.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../include/dmpc.h"
#include "common.cuh"
#include "dual.cuh"
#include "models.cuh"

namespace {

constexpr int kMaxGroups = 8;

struct DevGroup {
  dmpc_group g;
  dmpc_adjoint a;
  int32_t first_block;  // first grid block of this group
  int32_t K;            // horizon + 1
  int32_t ld32;         // row stride of FP32 blocks and padded vectors (pad_ld)
  int32_t blocks_smem;  // FP32 blocks: 0 workspace, 1 shared memory, 2 per instance (shared if they fit)
  uint64_t smem_block_budget;  // mode 2: shared-memory bytes available for one instance's blocks
  uint32_t w64_off;      // mixed row-pair path: shared-memory byte offset of the FP64 W blocks (0: workspace)
  size_t ws_offset;     // byte offset of instance 0 in the workspace
  size_t ws_stride;     // bytes per instance
  int32_t pg_idx[DMPC_MAX_PARAM_GRADS];
};

struct DevArgs {
  int32_t n_groups;
  int32_t total_blocks;
  dmpc_solver_params p;
  DevGroup grp[kMaxGroups];
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------- workspace layout
struct Layout {
  // offsets in doubles
  size_t A, Bm, C, Qi, Ri, q, r, gam, lam, res, t1, xb, ub, xn, un, fv, th, ph, ti, pm, tmp, li, contrib;
  size_t n_doubles;
  size_t f32;  // float offset (in floats) after the doubles, FP32 blocks when not in smem
  size_t n_floats;
  size_t bytes;
};

__host__ __device__ inline Layout make_layout(int nx, int nu, int N, int ld32, bool blocks_global,
                                              int n_param_grads) {
  Layout L;
  const size_t K = N + 1;
  size_t o = 0;
  auto take = [&](size_t n) {
    size_t r = o;
    o += align_up(n, 4);
    return r;
  };
  L.A = take((size_t)N * nx * nx);
  L.Bm = take((size_t)N * nx * nu);
  L.C = take(K * nx);
  L.Qi = take(K * nx);
  L.Ri = take(K * nu);
  L.q = take(K * nx);
  L.r = take(K * nu);
  L.gam = take(K * nx);
  L.lam = take(K * nx);
  L.res = take(K * nx);
  L.t1 = take(K * nx);
  L.xb = take(K * nx);
  L.ub = take(K * nu);
  L.xn = take(K * nx);
  L.un = take(K * nu);
  L.fv = take(K * nx);
  L.th = take(K * nx * nx);
  L.ph = take((size_t)N * nx * nx + nx * nx);
  L.ti = take(K * nx * nx);
  L.pm = take((size_t)N * nx * nx + nx * nx);
  L.tmp = take(K * nx * nx);
  L.li = take(K * nx * nx);
  L.contrib = take((size_t)(n_param_grads > 0 ? (n_param_grads < DMPC_MAX_PARAM_GRADS ? n_param_grads : DMPC_MAX_PARAM_GRADS) : 1) * K);
  L.n_doubles = o;
  L.f32 = 0;
  L.n_floats = blocks_global ? align_up((size_t)K * nx * ld32, 8) : 0;
  L.bytes = align_up(L.n_doubles * 8 + L.n_floats * 4, 256);
  return L;
}

// Row stride of the FP32 blocks and padded PCG vectors: the smallest ld >= nx with
// ld = 2 (mod 4).  ld/2 is odd, so 64-bit shared loads of 16 consecutive rows hit
// distinct banks, and ld is even, so every row starts 8-byte aligned.
__host__ __device__ constexpr int pad_ld(int nx) { return nx + ((6 - nx % 4) % 4); }

// shared memory bytes of one CTA: 2x32 reduction doubles + PCG vectors (+ FP32 blocks)
__host__ __device__ inline size_t smem_bytes_for(int nx, int N, int precision, bool blocks_smem) {
  const size_t K = N + 1;
  size_t b = 136 * sizeof(double);  // 2 x 64 reduction doubles + 8 line-search values
  if (precision == DMPC_PREC_FP64) {
    b += 5 * K * nx * sizeof(double);
  } else {
    b += align_up(5 * (K + 2) * pad_ld(nx) * sizeof(float), 16);
    if (blocks_smem) b += (size_t)K * nx * pad_ld(nx) * sizeof(float);
  }
  return align_up(b, 16);
}

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
// step of a closed-loop rollout.
__device__ inline Inst make_inst(const DevGroup& G, const dmpc_group& g, int i, void* ws, float* smem_blocks) {
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
  double* base = reinterpret_cast<double*>(reinterpret_cast<char*>(ws) + G.ws_offset + (size_t)i * G.ws_stride);
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
  // the row-pair PCG reads the FP64 W blocks at every residual replacement: keep them in
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
// lanes per block for the nx with a row-pair PCG, else one warp per block in the workspace (tmp as the
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
  int it;
  double eta;
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

// FP32 refinement is not paying off: a refinement step cut eta64 by less than 1e4 (the
// residual norm by less than 100x: kappa * eps32 is too close to 1 for the FP32 iterations
// to reach their target in the true residual), or the FP32 iterations have used half of
// pcg.max_iter.  Finish the solve with the FP64 recurrence (in the scaled basis, see
// pcg_fp64_scaled).  The recurrence
// gets the full pcg.max_iter budget of the reference's loop: the FP32 iterations before it
// are cheaper and restart at every refinement, so they are not charged against it, and a
// QP's reported iteration count can reach 1.5 max_iter.
__device__ PcgOut fp64_finish(const Inst& s, double* lam, int it, int max_iter, double eps, double* red, int& par) {
  // without Cholesky factors (sh_scaled_bad) the reference-basis blocks theta^-1, P exist instead
  PcgOut o = sh_scaled_bad ? pcg_fp64(s, lam, s.res, s.t1, s.xn, s.C, max_iter, eps, red, par)
                           : pcg_fp64_scaled(s, lam, max_iter, eps, red, par);
  return PcgOut{it + o.it, o.eta};
}
constexpr double kStagnation = 1e-4;
// Residual-replacement PCG (pcg_pair_scaled): the FP64 convergence test runs once the
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
// FP64 correction, two forms.
// * Any nx (pcg_mixed_scaled): iterative refinement.  res = gamma - S lam and
//   eta64 = res^T Phi^-1 res in FP64; stop like the reference on eta64 (pcg.py:397-403);
//   otherwise run the FP32 PCG on S^ d^ = L^-1 res / sqrt(eta64) to a relative eta
//   reduction of `inner_rel_tol` (and to 0.01 eps in absolute terms) and update
//   lam += sqrt(eta64) L^-T d^.  A refinement that cuts eta64 by less than 1e4, or the
//   max_ref-th refinement, hands the solve to the FP64 recurrence (fp64_finish).
// * Row pairs (pcg_pair_scaled): one FP32 PCG whose recursively updated residual is
//   replaced by the FP64 residual each time its eta has fallen by `inner_rel_tol`, keeping
//   the search direction (reliable updates: no Krylov space is thrown away at a restart).
//   The replacement residual is formed in the scaled basis from the FP64 W blocks,
//   r^ = r^_0 + (I + F^) lam^; the stopping test always uses an exact gamma - S lam.


template <class T>
__device__ __forceinline__ T* as_shared(T* p) {
  const ptrdiff_t off = reinterpret_cast<const unsigned char*>(p) - g_dyn_smem;
  return reinterpret_cast<T*>(g_dyn_smem + off);
}

// Compile-time-nx FP64 helpers of the row-pair PCG (pcg_pair_scaled), rows i0, i1 of knot
// t.  Both stay out of line, so that their registers do not weigh on the allocation of the
// FP32 iteration loop that calls them on its cold path.
//
// res = gamma - S lam for the thread's rows and r^ = L^-1 res in t1 (one barrier between
// the passes; each thread reads back only its own t1 rows).
template <int NX>
__device__ __noinline__ void exact_rhat(const Inst& s, const double* lam, int t, int i0, int i1, bool ok0,
                                        bool ok1, int N) {
  const int g0 = t * NX + i0, g1 = t * NX + i1;
  if (ok0) s.res[g0] = s.gam[g0] + stencil64<NX>(s.th, s.ph, lam, t, i0, N);
  if (ok1) s.res[g1] = s.gam[g1] + stencil64<NX>(s.th, s.ph, lam, t, i1, N);
  __syncthreads();
  const double* m0 = s.li + (size_t)g0 * NX;
  const double* m1 = s.li + (size_t)g1 * NX;
  const double* x = s.res + t * NX;
  double a0 = 0.0, a1 = 0.0;
#pragma unroll
  for (int j = 0; j < NX; ++j) {
    const double xj = x[j];
    if (j <= i0) a0 = fma(m0[j], xj, a0);
    if (j <= i1) a1 = fma(m1[j], xj, a1);
  }
  if (ok0) s.t1[g0] = a0;
  if (ok1) s.t1[g1] = a1;
}

// (F^ v) for the two rows in FP64: W_t (block t-1 of w, row stride NX) times v_{t-1} plus
// W_{t+1}^T (block t) times v_{t+1}; block N is zero and stands in for W_0 and W_{N+1}.
// v points at knot 0 of a vector with zero segments at knots -1 and K.
template <int NX>
__device__ __noinline__ double2 fhat64_pair(const double* __restrict__ w, int N, int t, int i0, int i1,
                                            const double* v) {
  constexpr int BS = NX * NX;
  const double* lo = w + (size_t)(t > 0 ? t - 1 : N) * BS;
  const double* up = w + (size_t)(t < N ? t : N) * BS;
  const double* vm = v + (t - 1) * NX;
  const double* vp = v + (t + 1) * NX;
  double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
  for (int j = 0; j < NX; ++j) {
    const double ym = vm[j], yp = vp[j];
    a0 = fma(lo[i0 * NX + j], ym, a0);
    a1 = fma(lo[i1 * NX + j], ym, a1);
    b0 = fma(up[j * NX + i0], yp, b0);
    b1 = fma(up[j * NX + i1], yp, b1);
  }
  return make_double2(a0 + b0, a1 + b1);
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

// Any nx and horizon: thread rows g = tid + k*blockDim; five padded FP32 vectors
// (K + 2 segments of ld floats with zero end segments) in shared memory, the W blocks
// in shared or global memory.
__device__ __noinline__ PcgOut pcg_mixed_scaled(const Inst& s, double* lam, float* vec, int max_iter, double eps,
                                                int max_ref, double inner_rel, double* red, int& par) {
  const int nx = s.nx, N = s.N, K = s.K, ld = s.ld, n = K * nx;
  const int span = (K + 2) * ld;
  for (int w = threadIdx.x; w < 5 * span; w += blockDim.x) vec[w] = 0.f;
  float* rv = vec + ld;
  float* pv = rv + span;
  float* zv = pv + span;
  float* uv = zv + span;
  float* dv = uv + span;
  const float* w32 = s.w32;
  int it = 0;
  const int it_cap = max_iter / 2;  // FP32 share of the budget; the rest is kept for fp64_finish
  double eta64 = 0.0, prev64 = 0.0;
  for (int ref = 0;; ++ref) {
    // res = gamma - S lam, r^ = L^-1 res (t1), eta64 = r^T (I - F^) r^ = res^T Phi^-1 res
    for (int g = threadIdx.x; g < n; g += blockDim.x)
      s.res[g] = s.gam[g] + stencil_row<double, double>(s.th, s.ph, nx, nx, N, lam, g);
    __syncthreads();
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      s.t1[g] = lower_row(s.li, nx, t, g - t * nx, s.res);
    }
    __syncthreads();
    double part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx;
      part += s.t1[g] * (s.t1[g] - fhat64_row(s.pm, nx, N, t, g - t * nx, s.t1));
    }
    eta64 = block_sum(part, red, par);
    const bool cont = (fabs(eta64) > eps && it <= max_iter - 1) || it < 1;
    if (!cont || !(eta64 == eta64)) break;
    if (ref >= max_ref || it >= it_cap || (ref > 0 && eta64 > kStagnation * prev64))
      return fp64_finish(s, lam, it, max_iter, eps, red, par);
    prev64 = eta64;
    const double scale = (eta64 > 0.0) ? rsqrt(eta64) : 1.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx, i = g - t * nx, x = t * ld + i;
      rv[x] = (float)(scale * s.t1[g]);
      dv[x] = 0.f;
    }
    __syncthreads();
    part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx, i = g - t * nx, x = t * ld + i;
      const float z = rv[x] - fhat_row(w32, nx, ld, N, t, i, rv);
      pv[x] = z;
      part += (double)rv[x] * (double)z;
    }
    double eta = block_sum(part, red, par);
    const double target = fmax(inner_rel * eta, eps * scale * scale * 0.01);
    int inner = 0;
    while ((eta > target && it < it_cap) || inner < 1) {
      part = 0.0;
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, i = g - t * nx, x = t * ld + i;
        const float u = -(pv[x] + fhat_row(w32, nx, ld, N, t, i, pv));
        uv[x] = u;
        part += (double)pv[x] * (double)u;
      }
      const double vden = block_sum(part, red, par);
      const float alpha = (float)(eta / vden);
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, x = t * ld + (g - t * nx);
        dv[x] = fmaf(alpha, pv[x], dv[x]);
        rv[x] = fmaf(-alpha, uv[x], rv[x]);
      }
      __syncthreads();
      part = 0.0;
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, i = g - t * nx, x = t * ld + i;
        const float z = rv[x] - fhat_row(w32, nx, ld, N, t, i, rv);
        zv[x] = z;
        part += (double)rv[x] * (double)z;
      }
      const double etap = block_sum(part, red, par);
      const float beta = (float)(etap / eta);
      for (int g = threadIdx.x; g < n; g += blockDim.x) {
        const int t = g / nx, x = t * ld + (g - t * nx);
        pv[x] = fmaf(beta, pv[x], zv[x]);
      }
      eta = etap;
      ++it;
      ++inner;
      __syncthreads();
      if (!(eta == eta) || !(vden == vden)) break;
    }
    const double back = (eta64 > 0.0) ? sqrt(eta64) : 1.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const int t = g / nx, i = g - t * nx;
      lam[g] += back * lower_col(s.li, nx, t, i, dv + t * ld);
    }
    __syncthreads();
  }
  return PcgOut{it, eta64};
}

// Compile-time nx, K * ceil(nx/2) <= blockDim.  Thread (t, q) = (tid mod K, tid div K) owns
// the rows i0 = q and i1 = q + H (H = ceil(nx/2); i1 exists when q + H < nx) of block row t
// and keeps their W coefficients (W_t rows i0, i1 and W_{t+1} columns i0, i1: 4 nx floats)
// in registers for the whole QP solve.  Both operators then read only the vector
// segments t-1 and t+1 from shared memory, each loaded once for both rows.  Lanes run
// over t for a fixed q, so a half warp's 64-bit segment loads (ld/2 odd) hit distinct
// banks.  Threads past the last pair (tid >= H K) idle on row 0 of block 0, which keeps
// every address in range; they take part in the barriers and reductions with zeros.
template <int NX>
__device__ __noinline__ PcgOut pcg_pair_scaled(const Inst& s, double* lam, float* vec, int max_iter, double eps,
                                               int max_ref, double upd_rel, double* red, int& par) {
  constexpr int LD = pad_ld(NX);
  constexpr int BS = NX * LD;
  constexpr int H = (NX + 1) / 2;
  constexpr int NP = (NX + 1) / 2;  // float2 pairs per padded segment
  const int K = s.K, N = s.N;
  float* rbase = as_shared(vec);  // (K + 2) segments: [0][v_0 .. v_N][0]
  float* pbase = as_shared(vec + (K + 2) * LD);
  float* rv = rbase + LD;
  float* pv = pbase + LD;
  const int qq = threadIdx.x / K;
  const bool ok0 = qq < H;
  const int q = ok0 ? qq : 0;
  const int tc = ok0 ? threadIdx.x - qq * K : 0;
  const bool ok1 = ok0 && (q + H < NX);
  const int i0 = q, i1 = ok1 ? q + H : q;
  const int lo_blk = (tc > 0 ? tc - 1 : N) * BS;  // block N is zero
  const int up_blk = (tc < N ? tc : N) * BS;
  float wl0[NX], wl1[NX], wu0[NX], wu1[NX];
  {
    const float* w = s.w32;
#pragma unroll
    for (int j = 0; j < NX; ++j) {
      wl0[j] = w[lo_blk + i0 * LD + j];
      wl1[j] = w[lo_blk + i1 * LD + j];
      wu0[j] = w[up_blk + j * LD + i0];
      wu1[j] = w[up_blk + j * LD + i1];
    }
  }
  const int seg = tc * LD;  // segment t in the padded vectors
  for (int w = threadIdx.x; w < (K + 2) * LD; w += blockDim.x) {
    if (w < LD || w >= (K + 1) * LD || (w % LD) >= NX) {
      rbase[w] = 0.f;
      pbase[w] = 0.f;
    }
  }
  // F^ v for the two rows
  auto fhat = [&](const float* v, float& f0, float& f1) {
    const float2* vm = reinterpret_cast<const float2*>(v + seg - LD);
    const float2* vp = reinterpret_cast<const float2*>(v + seg + LD);
    float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const float2 y = vm[j], x = vp[j];
      const int j0 = 2 * j, j1 = 2 * j + 1;
      a0 = fmaf(wl0[j0], y.x, a0);
      a1 = fmaf(wl1[j0], y.x, a1);
      a0 = fmaf(wu0[j0], x.x, a0);
      a1 = fmaf(wu1[j0], x.x, a1);
      if (j1 < NX) {
        b0 = fmaf(wl0[j1], y.y, b0);
        b1 = fmaf(wl1[j1], y.y, b1);
        b0 = fmaf(wu0[j1], x.y, b0);
        b1 = fmaf(wu1[j1], x.y, b1);
      }
    }
    f0 = a0 + b0;
    f1 = a1 + b1;
  };
  // FP64 exchange vector (knots -1..K) in the shared vector slots the pair path leaves free,
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
  auto eta_of = [&](double rh0, double rh1, double& zh0, double& zh1) -> double {
    double* x64 = x64_of();
    __syncthreads();
    if (ok0) x64[tc * NX + i0] = rh0;
    if (ok1) x64[tc * NX + i1] = rh1;
    __syncthreads();
    const double2 h = fhat64_pair<NX>(s.pm, N, tc, i0, i1, x64);
    zh0 = rh0 - h.x;
    zh1 = rh1 - h.y;
    return (ok0 ? rh0 * zh0 : 0.0) + (ok1 ? rh1 * zh1 : 0.0);
  };
  // lam += L^-T acc, acc = 0 (acc: lam^ accumulated since the last exact residual, FP64 in tmp)
  auto flush = [&]() {
    double* acc = s.tmp;
    __syncthreads();
    const double l0 = lower_col_t<NX>(s.li, tc, i0, acc + tc * NX);
    const double l1 = lower_col_t<NX>(s.li, tc, i1, acc + tc * NX);
    __syncthreads();
    if (ok0) {
      lam[tc * NX + i0] += l0;
      acc[tc * NX + i0] = 0.0;
    }
    if (ok1) {
      lam[tc * NX + i1] += l1;
      acc[tc * NX + i1] = 0.0;
    }
    __syncthreads();
  };
  float r0, r1, p0, p1, d0 = 0.f, d1 = 0.f, f0, f1;
  int it = 0;
  double eta, trig, hi;
  {
    const int g0 = tc * NX + i0, g1 = tc * NX + i1;
    if (ok0) s.tmp[g0] = 0.0;
    if (ok1) s.tmp[g1] = 0.0;
    double zh0, zh1;
    exact_rhat<NX>(s, lam, tc, i0, i1, ok0, ok1, N);
    const double rh0 = ok0 ? s.t1[g0] : 0.0, rh1 = ok1 ? s.t1[g1] : 0.0;
    const double eta64 = block_sum2(eta_of(rh0, rh1, zh0, zh1), red, par);
    if (!(eta64 == eta64)) return PcgOut{it, eta64};
    // The FP32 vectors carry the problem scaled by 1/sqrt(eta64) of the first residual
    // (eta starts at 1) and keep that scale through every replacement.  cst: scale,
    // sqrt(eta64_0), scale^2, the convergence-check level, eta64 and the scaled eta at the
    // last replacement, eps, upd_rel, max_ref, the replacement count, max_iter.
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
    }
    r0 = (float)(scale * rh0);
    r1 = (float)(scale * rh1);
    p0 = (float)(scale * zh0);
    p1 = (float)(scale * zh1);
    eta = eta64 * scale * scale;
    // a replacement is due once the recursion's eta is at or below trig, above hi (the
    // recursion diverges: FP32 cannot resolve this system) or not a number
    trig = fmax(eps * scale * scale * kCheckMargin, upd_rel * eta);
    hi = kDivergeRatio * eta;
  }
  const int it_cap = max_iter / 2;  // FP32 share of the budget; the rest is kept for fp64_finish
  if (ok0) pv[seg + i0] = p0;
  if (ok1) pv[seg + i1] = p1;
  __syncthreads();
  double eta64 = 0.0;
  for (;;) {
    // FP32 iterations until a replacement is due (a tight loop of its own)
    double vden, etap;
    float z0, z1;
    for (;;) {
      // u^ = S^ p^ = -(p^ + F^ p^)
      fhat(pv, f0, f1);
      const float u0 = -(p0 + f0), u1 = -(p1 + f1);
      double part = (ok0 ? (double)p0 * (double)u0 : 0.0) + (ok1 ? (double)p1 * (double)u1 : 0.0);
      vden = block_sum2(part, red, par);
      const float alpha = (float)(eta / vden);
      d0 = fmaf(alpha, p0, d0);
      d1 = fmaf(alpha, p1, d1);
      r0 = fmaf(-alpha, u0, r0);
      r1 = fmaf(-alpha, u1, r1);
      if (ok0) rv[seg + i0] = r0;
      if (ok1) rv[seg + i1] = r1;
      __syncthreads();
      // z^ = Phi^ r^ = r^ - F^ r^
      fhat(rv, f0, f1);
      z0 = r0 - f0;
      z1 = r1 - f1;
      part = (ok0 ? (double)r0 * (double)z0 : 0.0) + (ok1 ? (double)r1 * (double)z1 : 0.0);
      etap = block_sum2(part, red, par);
      ++it;
      if (!(etap > trig) || etap > hi || it >= it_cap || !(vden == vden)) break;
      const float beta = (float)(etap / eta);
      p0 = fmaf(beta, p0, z0);
      p1 = fmaf(beta, p1, z1);
      if (ok0) pv[seg + i0] = p0;
      if (ok1) pv[seg + i1] = p1;
      eta = etap;
      __syncthreads();
    }
    {
      // Residual replacement.  acc += sqrt(eta64_0) d^ (FP64); the true scaled residual
      // r^ = r^_0 + (I + F^) acc (r^_0 = t1, the residual at the last exact evaluation)
      // replaces the recursively updated one and the search direction is kept.  The
      // convergence decision always rests on an exact residual gamma - S lam.
      double* cst = x64_of() + (K + 1) * NX;
      double* acc = s.tmp;
      const int g0 = tc * NX + i0, g1 = tc * NX + i1;
      const double scale = cst[0], back = cst[1], s2 = cst[2], check_at = cst[3], prev64 = cst[4],
                   eta_upd = cst[5], c_eps = cst[6], c_upd = cst[7];
      const int c_maxref = (int)cst[8], nupd = (int)cst[9] + 1, c_maxit = (int)cst[10];
      const bool bad = !(etap == etap) || !(vden == vden);
      const bool at_check = etap <= check_at;
      const bool progressed = etap <= c_upd * eta_upd || etap > hi;
      // a non-finite segment is dropped: lam keeps the last finite update
      double a0 = ok0 ? acc[g0] : 0.0, a1 = ok1 ? acc[g1] : 0.0;
      if (!bad) {
        a0 += back * (double)d0;
        a1 += back * (double)d1;
        if (ok0) acc[g0] = a0;
        if (ok1) acc[g1] = a1;
      }
      d0 = 0.f;
      d1 = 0.f;
      double rh0, rh1, zh0, zh1;
      bool exact = bad || at_check || it >= it_cap;
      if (!exact) {
        double* x64 = x64_of();
        __syncthreads();
        if (ok0) x64[g0] = a0;
        if (ok1) x64[g1] = a1;
        __syncthreads();
        const double2 h = fhat64_pair<NX>(s.pm, N, tc, i0, i1, x64);
        rh0 = ok0 ? s.t1[g0] + a0 + h.x : 0.0;
        rh1 = ok1 ? s.t1[g1] + a1 + h.y : 0.0;
        eta64 = block_sum2(eta_of(rh0, rh1, zh0, zh1), red, par);
        exact = !(eta64 > c_eps);
      }
      if (exact) {
        flush();
        exact_rhat<NX>(s, lam, tc, i0, i1, ok0, ok1, N);
        rh0 = ok0 ? s.t1[g0] : 0.0;
        rh1 = ok1 ? s.t1[g1] : 0.0;
        eta64 = block_sum2(eta_of(rh0, rh1, zh0, zh1), red, par);
      }
      if (!(fabs(eta64) > c_eps && it <= c_maxit - 1) || !(eta64 == eta64)) {
        if (!exact) flush();
        break;
      }
      const double etas = eta64 * s2;
      if (bad || nupd >= c_maxref || it >= it_cap || !(etas > 0.0) ||
          (progressed && !at_check && eta64 > kUpdateStagnation * prev64)) {
        if (!exact) flush();
        return fp64_finish(s, lam, it, c_maxit, c_eps, red, par);
      }
      if (threadIdx.x == 0) {
        cst[4] = eta64;
        cst[5] = etas;
        cst[9] = (double)nupd;
      }
      r0 = (float)(scale * rh0);
      r1 = (float)(scale * rh1);
      z0 = (float)(scale * zh0);
      z1 = (float)(scale * zh1);
      // a true residual far above the recursion's means a stale direction: restart
      if (etas > kRestartRatio * eta) {
        p0 = 0.f;
        p1 = 0.f;
      }
      etap = etas;
      trig = fmax(check_at, c_upd * etas);
      hi = kDivergeRatio * etas;
    }
    const float beta = (float)(etap / eta);
    p0 = fmaf(beta, p0, z0);
    p1 = fmaf(beta, p1, z1);
    if (ok0) pv[seg + i0] = p0;
    if (ok1) pv[seg + i1] = p1;
    eta = etap;
    __syncthreads();
  }
  return PcgOut{it, eta64};
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

// ---------------------------------------------------------------- grid mapping
__device__ inline bool locate(const DevArgs& args, int b, int& gi, int& ii) {
  for (int g = args.n_groups - 1; g >= 0; --g) {
    if (b >= args.grp[g].first_block) {
      gi = g;
      ii = b - args.grp[g].first_block;
      return ii < args.grp[g].g.batch;
    }
  }
  return false;
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
  size_t vb = (precision == DMPC_PREC_FP64) ? 5 * (size_t)K * nx * sizeof(double)
                                            : align_up(5 * (size_t)(K + 2) * pad_ld(nx) * sizeof(float), 16);
  v.blocks = reinterpret_cast<float*>(p + vb);
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
    return o;
  }
  float* v = reinterpret_cast<float*>(sv.vec);
  if (sh_scaled_bad) return fp64_finish(s, lam, 0, P.pcg_max_iter, P.pcg_tol_epsilon, sv.red, par);
  if (s.K * ((s.nx + 1) / 2) <= (int)blockDim.x) {
    switch (s.nx) {
#define DMPC_PAIR(NXV)                                                                                   \
  case NXV:                                                                                              \
    return pcg_pair_scaled<NXV>(s, lam, v, P.pcg_max_iter, P.pcg_tol_epsilon, P.max_refinement,          \
                                P.inner_rel_tol, sv.red, par);
      DMPC_PAIR(3)
      DMPC_PAIR(4)
      DMPC_PAIR(6)
      DMPC_PAIR(7)
      DMPC_PAIR(8)
      DMPC_PAIR(12)
      DMPC_PAIR(13)
#undef DMPC_PAIR
      default: break;
    }
  }
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

__global__ void __launch_bounds__(512, 1) k_sqp_fwd(const __grid_constant__ DevArgs args, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  int gi, ii;
  if (!locate(args, blockIdx.x, gi, ii)) return;
  const DevGroup& G = args.grp[gi];
  sqp_forward(G, G.g, ii, args.p, ws, smem);
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
  return v;
}

// benchmark_diffmpc.py:140-175 (lax.scan of rollout_step, vmapped over instances), one CTA
// per instance for all simulation steps: solve the MPC from x_k (warm-started from step
// k-1's solution, or from the initial guess), apply u_k = controls[0], simulate x_{k+1}
// (x_{k+1} = A x_k + B u_k + b, or an integrator step of the model as in
// spacecraft/benchmark_diffmpc.py:87-89) and add the weighted squared deviations of x_{k+1}
// and u_k.  Every
// step's solution and last linearization point are kept for the adjoint sweep.
__global__ void __launch_bounds__(512, 1) k_rollout_fwd(const __grid_constant__ DevArgs args,
                                                        const __grid_constant__ dmpc_rollout ra, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DevGroup& G = args.grp[0];
  const dmpc_group& g0 = G.g;
  const int ii = blockIdx.x;
  if (ii >= g0.batch) return;
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
  if (threadIdx.x == 0 && a.num_pcg_iter) a.num_pcg_iter[ii] = o.it;
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

__global__ void __launch_bounds__(512, 1) k_sqp_adj(const __grid_constant__ DevArgs args, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  int gi, ii;
  if (!locate(args, blockIdx.x, gi, ii)) return;
  const DevGroup& G = args.grp[gi];
  sqp_adjoint(G, G.g, G.a, ii, args.p, ws, smem, false);
}

// Reverse sweep of the rollout's gradient (what jax.grad of the reference's scan computes):
// with lam_T = c dcost/dx_T (c = dL/d running cost), F the simulator step, for k = T-1 .. 0
//   dl/du_0 of step k  = c dcost/du_k + (dF/du)^T lam_{k+1}
//   adjoint of step k's solve, parameter gradients accumulated into adj's outputs
//   lam_k = (dF/dx)^T lam_{k+1} + c dcost/dx_k (k >= 1) [+ the solve's dL/dx_0 if through_state]
// (dF/dz)^T lam is formed by one Dual evaluation per direction for the model simulator.
// and dL/dx_0 = lam_0.  One CTA per instance, all steps in one launch.
__global__ void __launch_bounds__(512, 1) k_rollout_adj(const __grid_constant__ DevArgs args,
                                                        const __grid_constant__ dmpc_rollout ra,
                                                        const __grid_constant__ dmpc_rollout_adjoint rr, void* ws) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DevGroup& G = args.grp[0];
  const dmpc_group& g0 = G.g;
  const int ii = blockIdx.x;
  if (ii >= g0.batch) return;
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

// ---------------------------------------------------------------- dense-layout parity kernels
// dmpc_linearize: dense As, Bs, Cs, Qinv, qvec, Rinv, rvec of one group
__global__ void __launch_bounds__(256) k_linearize(const __grid_constant__ DevArgs args, void* ws, double* As,
                                                   double* Bs, double* Cs, double* Qinv, double* qv, double* Rinv,
                                                   double* rv) {
  int gi, ii;
  if (!locate(args, blockIdx.x, gi, ii)) return;
  const DevGroup& G = args.grp[gi];
  const dmpc_group& g = G.g;
  Inst s = make_inst(G, g, ii, ws, nullptr);
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

// dmpc_schur_assemble: general QP data (any As_next, dense Qinv / Rinv), FP64
__global__ void __launch_bounds__(256) k_schur_dense(int N, int nx, int nu, const double* As_next, const double* As,
                                                     const double* Bs, const double* Cs, const double* Qinv,
                                                     const double* qvec, const double* Rinv, const double* rvec,
                                                     double* S, double* Phiinv, double* gamma, double* ws) {
  const int b = blockIdx.x, K = N + 1, nn = nx * nx;
  const double* An = As_next + (size_t)b * N * nn;
  const double* A = As + (size_t)b * N * nn;
  const double* B = Bs + (size_t)b * N * nx * nu;
  const double* Qi = Qinv + (size_t)b * K * nn;
  const double* Ri = Rinv + (size_t)b * N * nu * nu;
  double* th = ws + (size_t)b * 4 * K * nn;
  double* ph = th + K * nn;
  double* ti = ph + K * nn;
  double* tm = ti + K * nn;
  // theta, phi
  for (int w = threadIdx.x; w < K * nn; w += blockDim.x) {
    const int t = w / nn, e = w - t * nn, i = e / nx, j = e - i * nx;
    double v;
    if (t == 0) {
      v = Qi[e];
    } else {
      const int k = t - 1;
      const double* Ak = A + (size_t)k * nn;
      const double* Ank = An + (size_t)k * nn;
      const double* Bk = B + (size_t)k * nx * nu;
      const double* Q0 = Qi + (size_t)k * nn;
      const double* Q1 = Qi + (size_t)(k + 1) * nn;
      const double* R0 = Ri + (size_t)k * nu * nu;
      v = 0.0;
      for (int l = 0; l < nx; ++l)
        for (int m = 0; m < nx; ++m) v += Ak[i * nx + l] * Q0[l * nx + m] * Ak[j * nx + m];
      for (int l = 0; l < nu; ++l)
        for (int m = 0; m < nu; ++m) v += Bk[i * nu + l] * R0[l * nu + m] * Bk[j * nu + m];
      for (int l = 0; l < nx; ++l)
        for (int m = 0; m < nx; ++m) v += Ank[i * nx + l] * Q1[l * nx + m] * Ank[j * nx + m];
    }
    th[w] = v;
    tm[w] = v;
    if (t < N) {
      // phi_t = A_t Qinv_t Anext_{t-1}^T, Anext_{-1} = I
      const double* Ak = A + (size_t)t * nn;
      const double* Q0 = Qi + (size_t)t * nn;
      double p = 0.0;
      for (int l = 0; l < nx; ++l)
        for (int m = 0; m < nx; ++m) {
          const double anp = (t == 0) ? ((j == m) ? 1.0 : 0.0) : An[(size_t)(t - 1) * nn + j * nx + m];
          p += Ak[i * nx + l] * Q0[l * nx + m] * anp;
        }
      ph[(size_t)t * nn + e] = p;
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int t = warp; t < K; t += nwarp) warp_spd_inverse(tm + (size_t)t * nn, ti + (size_t)t * nn, nx);
  __syncthreads();
  // S and Phiinv rows (pcg.py:198-239)
  const int rw = 3 * nx;
  for (int w = threadIdx.x; w < K * nx * rw; w += blockDim.x) {
    const int t = w / (nx * rw), e = w - t * nx * rw, i = e / rw, c = e - i * rw;
    const int blk = c / nx, j = c - blk * nx;
    double sv = 0.0, pv = 0.0;
    if (blk == 1) {
      sv = -th[(size_t)t * nn + i * nx + j];
      pv = ti[(size_t)t * nn + i * nx + j];
    } else if (blk == 0 && t > 0) {
      const double* phm = ph + (size_t)(t - 1) * nn;
      sv = -phm[i * nx + j];
      // -theta_t^-1 phi_{t-1} theta_{t-1}^-1
      const double* Ti = ti + (size_t)t * nn;
      const double* Tm = ti + (size_t)(t - 1) * nn;
      double acc = 0.0;
      for (int l = 0; l < nx; ++l) {
        double m = 0.0;
        for (int o = 0; o < nx; ++o) m += Ti[i * nx + o] * phm[o * nx + l];
        acc += m * Tm[l * nx + j];
      }
      pv = -acc;
    } else if (blk == 2 && t < N) {
      const double* pht = ph + (size_t)t * nn;
      sv = -pht[j * nx + i];
      // -theta_t^-1 phi_t^T theta_{t+1}^-1
      const double* Ti = ti + (size_t)t * nn;
      const double* Tp = ti + (size_t)(t + 1) * nn;
      double acc = 0.0;
      for (int l = 0; l < nx; ++l) {
        double m = 0.0;
        for (int o = 0; o < nx; ++o) m += Ti[i * nx + o] * pht[l * nx + o];
        acc += m * Tp[l * nx + j];
      }
      pv = -acc;
    }
    S[(size_t)b * K * nx * rw + w] = sv;
    Phiinv[(size_t)b * K * nx * rw + w] = pv;
  }
  // gamma
  const double* q = qvec + (size_t)b * K * nx;
  const double* r = rvec + (size_t)b * N * nu;
  for (int w = threadIdx.x; w < K * nx; w += blockDim.x) {
    const int t = w / nx, i = w - t * nx;
    double gv = 0.0;
    if (t == 0) {
      for (int l = 0; l < nx; ++l) gv += Qi[i * nx + l] * q[l];
    } else {
      const int k = t - 1;
      const double* Ak = A + (size_t)k * nn;
      const double* Ank = An + (size_t)k * nn;
      const double* Bk = B + (size_t)k * nx * nu;
      const double* Q0 = Qi + (size_t)k * nn;
      const double* Q1 = Qi + (size_t)t * nn;
      const double* R0 = Ri + (size_t)k * nu * nu;
      for (int l = 0; l < nx; ++l) {
        double a0 = 0.0, a1 = 0.0;
        for (int m = 0; m < nx; ++m) {
          a0 += Q0[l * nx + m] * q[k * nx + m];
          a1 += Q1[l * nx + m] * q[t * nx + m];
        }
        gv += Ak[i * nx + l] * a0 + Ank[i * nx + l] * a1;
      }
      for (int l = 0; l < nu; ++l) {
        double a0 = 0.0;
        for (int m = 0; m < nu; ++m) a0 += R0[l * nu + m] * r[k * nu + m];
        gv += Bk[i * nu + l] * a0;
      }
    }
    gamma[(size_t)b * K * nx + w] = Cs[(size_t)b * K * nx + w] + gv;
  }
}

// dense 3-block stencil row: y = M_t [v_{t-1}; v_t; v_{t+1}]
__device__ inline double dense_row(const double* M, const double* v, int nx, int N, int g) {
  const int t = g / nx, i = g - t * nx;
  const double* row = M + ((size_t)t * nx + i) * 3 * nx;
  double a = 0.0;
  for (int blk = 0; blk < 3; ++blk) {
    const int tt = t + blk - 1;
    if (tt < 0 || tt > N) continue;
    for (int j = 0; j < nx; ++j) a += row[blk * nx + j] * v[tt * nx + j];
  }
  return a;
}

// x_t = -Qinv_t (q_t + An_{t-1}^T lam_t + A_t^T lam_{t+1}), An_{-1} = I,
// x_N = -Qinv_N (q_N + An_{N-1}^T lam_N), u_t = -Rinv_t (r_t + B_t^T lam_{t+1}), u_N = 0
// (pcg.py:290-348), general dense matrices.  `tv` is K*nx scratch.
__device__ void dense_recover(int b, int N, int nx, int nu, const double* lv, double* tv, const double* As_next,
                              const double* As, const double* Bs, const double* Qinv, const double* qvec,
                              const double* Rinv, const double* rvec, double* xs, double* us) {
  const int K = N + 1, n = K * nx, nn = nx * nx;
  const double* An = As_next + (size_t)b * N * nn;
  const double* A = As + (size_t)b * N * nn;
  const double* B = Bs + (size_t)b * N * nx * nu;
  const double* Qi = Qinv + (size_t)b * K * nn;
  const double* Ri = Rinv + (size_t)b * N * nu * nu;
  const double* q = qvec + (size_t)b * n;
  const double* r = rvec + (size_t)b * N * nu;
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx, i = g - t * nx;
    double a = q[g];
    if (t == 0) {
      a += lv[i];
    } else {
      const double* Ap = An + (size_t)(t - 1) * nn;
      for (int j = 0; j < nx; ++j) a += Ap[j * nx + i] * lv[t * nx + j];
    }
    if (t < N) {
      const double* At = A + (size_t)t * nn;
      for (int j = 0; j < nx; ++j) a += At[j * nx + i] * lv[(t + 1) * nx + j];
    }
    tv[g] = a;
  }
  __syncthreads();
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx, i = g - t * nx;
    const double* Qt = Qi + (size_t)t * nn + i * nx;
    double a = 0.0;
    for (int j = 0; j < nx; ++j) a += Qt[j] * tv[t * nx + j];
    xs[(size_t)b * n + g] = -a;
  }
  for (int g = threadIdx.x; g < K * nu; g += blockDim.x) {
    const int t = g / nu, i = g - t * nu;
    double val = 0.0;
    if (t < N) {
      const double* Bt = B + (size_t)t * nx * nu;
      const double* Rt = Ri + (size_t)t * nu * nu + i * nu;
      for (int m = 0; m < nu; ++m) {
        double c = r[t * nu + m];
        for (int j = 0; j < nx; ++j) c += Bt[j * nu + m] * lv[(t + 1) * nx + j];
        val += Rt[m] * c;
      }
      val = -val;
    }
    us[(size_t)b * K * nu + g] = val;
  }
}

__global__ void __launch_bounds__(256) k_recover_dense(int N, int nx, int nu, const double* lam, const double* As_next,
                                                       const double* As, const double* Bs, const double* Qinv,
                                                       const double* qvec, const double* Rinv, const double* rvec,
                                                       double* xs, double* us) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int b = blockIdx.x, n = (N + 1) * nx;
  double* lv = reinterpret_cast<double*>(smem);
  double* tv = lv + n;
  for (int g = threadIdx.x; g < n; g += blockDim.x) lv[g] = lam[(size_t)b * n + g];
  __syncthreads();
  dense_recover(b, N, nx, nu, lv, tv, As_next, As, Bs, Qinv, qvec, Rinv, rvec, xs, us);
}

// gamma from the premultiplied matrices (pcg.py:245-288)
__global__ void __launch_bounds__(256) k_gamma_dense(int N, int nx, int nu, const double* AQ, const double* AnQ,
                                                     const double* BR, const double* Cs, const double* Q0inv,
                                                     const double* qs, const double* rs, double* gamma) {
  const int b = blockIdx.x, K = N + 1, n = K * nx, nn = nx * nx;
  const double* q = qs + (size_t)b * n;
  const double* r = rs + (size_t)b * N * nu;
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const int t = g / nx, i = g - t * nx;
    double v = 0.0;
    if (t == 0) {
      const double* Q0 = Q0inv + (size_t)b * nn + i * nx;
      for (int j = 0; j < nx; ++j) v += Q0[j] * q[j];
    } else {
      const int k = t - 1;
      const double* a = AQ + ((size_t)b * N + k) * nn + i * nx;
      const double* an = AnQ + ((size_t)b * N + k) * nn + i * nx;
      const double* br = BR + ((size_t)b * N + k) * nx * nu + i * nu;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      for (int j = 0; j < nx; ++j) s0 += a[j] * q[k * nx + j];
      for (int j = 0; j < nu; ++j) s1 += br[j] * r[k * nu + j];
      for (int j = 0; j < nx; ++j) s2 += an[j] * q[t * nx + j];
      v = s0 + s1 + s2;
    }
    gamma[(size_t)b * n + g] = Cs[(size_t)b * n + g] + v;
  }
}

// dmpc_pcg_solve: solve_KKT_Schur on the dense layout (pcg.py:350-445), FP64
__global__ void __launch_bounds__(256) k_pcg_dense(int N, int nx, int nu, const double* S, const double* Phi,
                                                   const double* gamma, const double* lam0, const double* As_next,
                                                   const double* As, const double* Bs, const double* Qinv,
                                                   const double* qvec, const double* Rinv, const double* rvec,
                                                   int max_iter, double eps, double* lam_out, double* xs,
                                                   double* us, int32_t* iters, double* etas) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int b = blockIdx.x, K = N + 1, n = K * nx;
  double* red = reinterpret_cast<double*>(smem);
  double* lv = red + 128;
  double *rv = lv + n, *pv = rv + n, *tv = pv + n, *uv = tv + n;
  const double* Sb = S + (size_t)b * K * nx * 3 * nx;
  const double* Pb = Phi + (size_t)b * K * nx * 3 * nx;
  const double* gb = gamma + (size_t)b * n;
  int par = 0;
  for (int g = threadIdx.x; g < n; g += blockDim.x) lv[g] = lam0[(size_t)b * n + g];
  __syncthreads();
  for (int g = threadIdx.x; g < n; g += blockDim.x) rv[g] = gb[g] - dense_row(Sb, lv, nx, N, g);
  __syncthreads();
  double part = 0.0;
  for (int g = threadIdx.x; g < n; g += blockDim.x) {
    const double rt = dense_row(Pb, rv, nx, N, g);
    tv[g] = rt;
    pv[g] = rt;
    part += rv[g] * rt;
  }
  double eta = block_sum(part, red, par);
  int it = 0;
  while ((fabs(eta) > eps && it <= max_iter - 1) || it < 1) {
    part = 0.0;
    for (int g = threadIdx.x; g < n; g += blockDim.x) {
      const double u = dense_row(Sb, pv, nx, N, g);
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
      const double rt = dense_row(Pb, rv, nx, N, g);
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
  for (int g = threadIdx.x; g < n; g += blockDim.x) lam_out[(size_t)b * n + g] = lv[g];
  __syncthreads();
  dense_recover(b, N, nx, nu, lv, tv, As_next, As, Bs, Qinv, qvec, Rinv, rvec, xs, us);
  if (threadIdx.x == 0) {
    iters[b] = it;
    etas[b] = eta;
  }
}

// ---------------------------------------------------------------- FP32 FMA throughput probe
// Eight independent FMA chains per thread; used only to measure the FP32 CUDA-core
// peak that serves as the roofline denominator of the (shared-memory resident) PCG.
__global__ void __launch_bounds__(256) k_fma_probe(int iters, float seed, float* out) {
  float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
  float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
  const float m = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
    }
  }
  const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 12345.678f) out[blockIdx.x] = r;  // keeps the chains live
}

// ---------------------------------------------------------------- host side
// Last CUDA error seen by an entry point on this thread (dmpc_last_cuda_error).
thread_local cudaError_t g_last_cuda_error = cudaSuccess;
int cuda_rc(cudaError_t e) {
  if (e == cudaSuccess) return DMPC_OK;
  g_last_cuda_error = e;
  return DMPC_ERR_CUDA;
}

// Static shared memory of the SQP kernels: the per-instance context (sh_inst), the
// scaled-basis flag and, in the rollout kernels, the step views and the state cotangent.  It counts against the same per-CTA opt-in limit as the dynamic
// request, so every dynamic size is checked against optin - kStaticSmemReserve.  A fixed
// reserve (checked at compile time) keeps the size logic free of runtime queries.
constexpr size_t kStaticSmemReserve = 2048;
// (the rollout kernels also keep the per-step group and adjoint views and the state
// cotangent there)
static_assert(sizeof(Inst) + sizeof(dmpc_group) + sizeof(dmpc_adjoint) + (2 * DMPC_MAX_NX + DMPC_MAX_NU) * sizeof(double) +
                      2 * sizeof(double) + 64 <= kStaticSmemReserve,
              "static shared memory reserve too small");

// nx with a row-pair specialisation of the scaled FP32 PCG (pcg_pair_scaled)
bool pair_nx(int nx) { return nx == 3 || nx == 4 || nx == 6 || nx == 7 || nx == 8 || nx == 12 || nx == 13; }

// Threads per CTA (256..512; 512 is the kernels' launch bound).  Mixed precision: one thread
// per row pair when K * ceil(nx/2) fits, else one thread per row up to 512 threads (several
// rows per thread beyond that).
int choose_threads(const dmpc_solver_params* p, int nx, int K) {
  if (p && p->threads_per_block > 0) return p->threads_per_block;
  int rows = K * nx;
  if (p && p->precision == DMPC_PREC_MIXED && pair_nx(nx) && K * ((nx + 1) / 2) <= 512) rows = K * ((nx + 1) / 2);
  int t = ((rows + 31) / 32) * 32;
  // at least 256: the FP64 setup phases (assembly, factorisations) spread over all threads,
  // and short horizons leave too few rows to keep them busy (measured: nx=8, 40 knots runs
  // 17 % faster at 256 threads than at its 160 row pairs)
  if (t < 256) t = 256;
  if (t > 512) t = 512;
  return t;
}

int fill_args(int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj, const dmpc_solver_params* p,
              DevArgs* args, size_t* ws_total, size_t* smem_max, int* threads) {
  if (n_groups < 1 || n_groups > kMaxGroups || !groups || !p) return DMPC_ERR_INVALID;
  if (p->precision != DMPC_PREC_FP64 && p->precision != DMPC_PREC_MIXED) return DMPC_ERR_INVALID;
  if (p->n_alphas < 1 || p->n_alphas > DMPC_MAX_ALPHAS) return DMPC_ERR_INVALID;
  if (p->threads_per_block != 0 &&
      (p->threads_per_block < 64 || p->threads_per_block > 512 || (p->threads_per_block & 31) != 0))
    return DMPC_ERR_INVALID;
  if (p->num_scp_iteration_max < 1 || p->pcg_max_iter < 1 || p->max_refinement < 1) return DMPC_ERR_INVALID;
  memset(args, 0, sizeof(DevArgs));
  args->n_groups = n_groups;
  args->p = *p;
  size_t off = 0, smax = 0;
  int blocks = 0, thr = 0;
  int dev = 0;
  int smem_optin = 0;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem_optin <= 0) smem_optin = 227 * 1024;
  const size_t smem_cap = (size_t)smem_optin - kStaticSmemReserve;
  for (int k = 0; k < n_groups; ++k) {
    const dmpc_group& g = groups[k];
    if (!model_dims_ok(g.model, g.nx, g.nu)) return DMPC_ERR_UNSUPPORTED;
    if (g.horizon < 1 || g.batch < 0 || g.scheme < 0 || g.scheme > 2) return DMPC_ERR_INVALID;
    if (g.n_model_params != model_param_count(g.model, g.nx, g.nu)) return DMPC_ERR_INVALID;
    DevGroup& G = args->grp[k];
    G.g = g;
    if (adj) G.a = adj[k];
    G.first_block = blocks;
    G.K = g.horizon + 1;
    G.ld32 = pad_ld(g.nx);
    // FP32 blocks: all instances in shared memory (1); ragged group whose longest
    // instance does not fit: each instance checks its own size at run time (2); else
    // workspace (0).  Per-instance horizons live in device memory, hence mode 2.
    const size_t need_all = smem_bytes_for(g.nx, g.horizon, p->precision, true);
    const size_t base = smem_bytes_for(g.nx, g.horizon, p->precision, false);
    int mode = 0;
    if (p->precision == DMPC_PREC_MIXED && p->blocks_in_smem != 0) {
      if (need_all <= smem_cap)
        mode = 1;
      else if (g.horizons && base + (size_t)2 * g.nx * pad_ld(g.nx) * sizeof(float) <= smem_cap)
        mode = 2;
    }
    if (p->blocks_in_smem == 1 && p->precision == DMPC_PREC_MIXED && mode != 1) return DMPC_ERR_UNSUPPORTED;
    size_t sm = mode == 1 ? need_all : (mode == 2 ? smem_cap : base);
    // Row-pair path (the FP32 W blocks live in registers during the iterations): the FP64
    // W blocks of its residual replacements go to shared memory, ahead of the FP32 copy,
    // which the pair path reads only once per QP.
    G.w64_off = 0;
    const int pairs = G.K * ((g.nx + 1) / 2);
    if (p->precision == DMPC_PREC_MIXED && p->blocks_in_smem != 0 && pair_nx(g.nx) && pairs <= 512 &&
        (p->threads_per_block == 0 || pairs <= p->threads_per_block)) {
      const size_t w64b = (size_t)G.K * g.nx * g.nx * sizeof(double);
      if (mode != 2 && align_up(sm, 16) + w64b <= smem_cap) {
        G.w64_off = (uint32_t)align_up(sm, 16);
      } else if (mode == 1 && p->blocks_in_smem != 1 && align_up(base, 16) + w64b <= smem_cap) {
        mode = 0;
        G.w64_off = (uint32_t)align_up(base, 16);
      }
      if (G.w64_off) sm = G.w64_off + w64b;
    }
    G.blocks_smem = mode;
    G.smem_block_budget = mode == 2 ? (uint64_t)(smem_cap - base) : 0;
    if (sm > smem_cap) return DMPC_ERR_UNSUPPORTED;
    if (sm > smax) smax = sm;
    int ng = 0;
    if (adj) {
      ng = adj[k].n_param_grads;
      if (ng < 0 || ng > g.n_model_params || ng > DMPC_MAX_PARAM_GRADS) return DMPC_ERR_INVALID;
      for (int q = 0; q < ng; ++q) {
        const int idx = adj[k].param_grad_index[q];
        if (idx < 0 || idx >= g.n_model_params) return DMPC_ERR_INVALID;
        G.pg_idx[q] = idx;
      }
    } else {
      ng = g.n_model_params;  // size the workspace for any later adjoint call
    }
    Layout L = make_layout(g.nx, g.nu, g.horizon, G.ld32, mode != 1, g.n_model_params);
    G.ws_offset = off;
    G.ws_stride = L.bytes;
    off += L.bytes * (size_t)g.batch;
    blocks += g.batch;
    const int t = choose_threads(p, g.nx, G.K);
    if (t > thr) thr = t;
  }
  args->total_blocks = blocks;
  *ws_total = off;
  *smem_max = smax;
  *threads = thr;
  return DMPC_OK;
}

}  // namespace

// Fixed scratch for dmpc_solve_fwd_noalloc.  It is part of this library's device
// module, so every GPU that loads the library holds these bytes until the process
// exits.  Host code must not pass `g_noalloc_scratch` itself to a kernel: on the host
// the name stands for a host-side shadow, not a device address.  The device address
// is looked up once per device with cudaGetSymbolAddress and cached below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[DMPC_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_device_ptr[kNoallocMaxDevices] = {};
}  // namespace

extern "C" {

int dmpc_abi_version(void) { return DMPC_ABI_VERSION; }

const char* dmpc_last_cuda_error(void) { return cudaGetErrorName(g_last_cuda_error); }

const char* dmpc_error_string(int code) {
  switch (code) {
    case DMPC_OK: return "ok";
    case DMPC_ERR_INVALID: return "invalid descriptor or sizes";
    case DMPC_ERR_WORKSPACE: return "workspace too small or misaligned";
    case DMPC_ERR_CUDA: return "CUDA runtime error";
    case DMPC_ERR_UNSUPPORTED: return "unsupported model or option";
  }
  return "unknown error";
}

void dmpc_default_params(dmpc_solver_params* p) {
  memset(p, 0, sizeof(*p));
  p->tol_convergence = 1e-8;
  p->num_scp_iteration_max = 15;
  p->linesearch = 0;
  p->linesearch_eta = 0.4;
  p->n_alphas = 5;
  const double al[5] = {0.01, 0.1, 0.3, 0.7, 1.0};
  for (int i = 0; i < 5; ++i) p->alphas[i] = al[i];
  p->warm_start_backward = 1;
  p->pcg_max_iter = 10000;
  p->pcg_tol_epsilon = 1e-9;
  p->precision = DMPC_PREC_MIXED;
  p->max_refinement = 30;
  p->inner_rel_tol = 1e-3;
  p->threads_per_block = 0;
  p->blocks_in_smem = -1;
}

size_t dmpc_workspace_size(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params) {
  DevArgs* a = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(n_groups, groups, nullptr, params, a, &ws, &sm, &thr);
  delete a;
  return rc == DMPC_OK ? ws : 0;
}

static int launch_common(bool adjoint, int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj,
                         const dmpc_solver_params* params, void* workspace, size_t workspace_bytes, void* stream) {
  DevArgs* args = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(n_groups, groups, adj, params, args, &ws, &sm, &thr);
  if (rc != DMPC_OK) {
    delete args;
    return rc;
  }
  if (ws > workspace_bytes || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0) {
    delete args;
    return DMPC_ERR_WORKSPACE;
  }
  if (args->total_blocks == 0) {
    delete args;
    return DMPC_OK;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (adjoint) {
    e = cudaFuncSetAttribute(k_sqp_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
      k_sqp_adj<<<args->total_blocks, thr, sm, st>>>(*args, workspace);
      e = cudaGetLastError();
    }
  } else {
    e = cudaFuncSetAttribute(k_sqp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
      k_sqp_fwd<<<args->total_blocks, thr, sm, st>>>(*args, workspace);
      e = cudaGetLastError();
    }
  }
  delete args;
  return cuda_rc(e);
}

int dmpc_solve_fwd(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params, void* workspace,
                   size_t workspace_bytes, void* stream) {
  return launch_common(false, n_groups, groups, nullptr, params, workspace, workspace_bytes, stream);
}

int dmpc_solve_adj(int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj, const dmpc_solver_params* params,
                   void* workspace, size_t workspace_bytes, void* stream) {
  if (!adj) return DMPC_ERR_INVALID;
  return launch_common(true, n_groups, groups, adj, params, workspace, workspace_bytes, stream);
}

int dmpc_rollout_adj(const dmpc_group* group, const dmpc_rollout* ro, const dmpc_adjoint* adj,
                     const dmpc_rollout_adjoint* rr, const dmpc_solver_params* params, void* workspace,
                     size_t workspace_bytes, void* stream) {
  if (!group || !ro || !adj || !rr || ro->num_steps < 1) return DMPC_ERR_INVALID;
  if (ro->simulator < DMPC_SIM_LINEAR || ro->simulator > DMPC_SIM_MODEL_SCHEME) return DMPC_ERR_INVALID;
  if (!ro->cost_state_weights || !ro->cost_control_weights) return DMPC_ERR_INVALID;
  if (ro->simulator == DMPC_SIM_LINEAR && (!ro->sim_A || !ro->sim_B)) return DMPC_ERR_INVALID;
  if (!ro->step_initial_state || !ro->step_states || !ro->step_controls ||
      !ro->step_dual || !ro->step_lin_states || !ro->step_lin_controls || !ro->step_status || !ro->step_num_iter ||
      !ro->step_convergence_error || !ro->step_convergence_errors || !ro->step_linesearch_alphas ||
      !ro->step_num_pcg_iters || !rr->cost_cotangent || !rr->scratch_dl_dcontrols || !rr->scratch_dual)
    return DMPC_ERR_INVALID;
  DevArgs* args = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(1, group, adj, params, args, &ws, &sm, &thr);
  if (rc == DMPC_OK && (ws > workspace_bytes || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0))
    rc = DMPC_ERR_WORKSPACE;
  if (rc == DMPC_OK && args->total_blocks > 0) {
    cudaError_t e = cudaFuncSetAttribute(k_rollout_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
      k_rollout_adj<<<args->total_blocks, thr, sm, reinterpret_cast<cudaStream_t>(stream)>>>(*args, *ro, *rr, workspace);
      e = cudaGetLastError();
    }
    rc = cuda_rc(e);
  }
  delete args;
  return rc;
}

int dmpc_rollout_fwd(const dmpc_group* group, const dmpc_rollout* ro, const dmpc_solver_params* params,
                     void* workspace, size_t workspace_bytes, void* stream) {
  if (!group || !ro || ro->num_steps < 1) return DMPC_ERR_INVALID;
  if (ro->simulator < DMPC_SIM_LINEAR || ro->simulator > DMPC_SIM_MODEL_SCHEME) return DMPC_ERR_INVALID;
  if (!ro->cost_state_weights || !ro->cost_control_weights) return DMPC_ERR_INVALID;
  if (ro->simulator == DMPC_SIM_LINEAR && (!ro->sim_A || !ro->sim_B || !ro->sim_b)) return DMPC_ERR_INVALID;
  if (!ro->step_initial_state || !ro->step_states || !ro->step_controls ||
      !ro->step_dual || !ro->step_lin_states || !ro->step_lin_controls || !ro->step_status || !ro->step_num_iter ||
      !ro->step_convergence_error || !ro->step_convergence_errors || !ro->step_linesearch_alphas ||
      !ro->step_num_pcg_iters || !ro->running_cost)
    return DMPC_ERR_INVALID;
  if (!group->initial_state || !group->states || !group->controls || !group->dual || !group->convergence_error ||
      !group->convergence_errors || !group->linesearch_alphas || !group->num_pcg_iters)
    return DMPC_ERR_INVALID;
  DevArgs* args = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(1, group, nullptr, params, args, &ws, &sm, &thr);
  if (rc == DMPC_OK && (ws > workspace_bytes || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0))
    rc = DMPC_ERR_WORKSPACE;
  if (rc == DMPC_OK && args->total_blocks > 0) {
    cudaError_t e = cudaFuncSetAttribute(k_rollout_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
      k_rollout_fwd<<<args->total_blocks, thr, sm, reinterpret_cast<cudaStream_t>(stream)>>>(*args, *ro, workspace);
      e = cudaGetLastError();
    }
    rc = cuda_rc(e);
  }
  delete args;
  return rc;
}

// Forward solve for callers that cannot allocate device memory: it uses the fixed
// library-owned scratch array above instead of a caller workspace.  The first call on
// a device looks up that array's device address (with that device current) and
// caches it; make that first call outside any stream capture.
int dmpc_solve_fwd_noalloc(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params, void* stream) {
  DevArgs* args = new DevArgs;
  size_t need = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(n_groups, groups, nullptr, params, args, &need, &sm, &thr);
  delete args;
  if (rc != DMPC_OK) return rc;
  if (need > (size_t)DMPC_NOALLOC_SCRATCH_BYTES) return DMPC_ERR_WORKSPACE;
  int dev = -1;
  const cudaError_t de = cudaGetDevice(&dev);
  if (de != cudaSuccess) return cuda_rc(de);
  if (dev < 0 || dev >= kNoallocMaxDevices) return DMPC_ERR_UNSUPPORTED;
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_device_ptr[dev] == nullptr) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) return cuda_rc(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
      g_noalloc_device_ptr[dev] = p;
    }
    base = g_noalloc_device_ptr[dev];
  }
  return launch_common(false, n_groups, groups, nullptr, params, base, (size_t)DMPC_NOALLOC_SCRATCH_BYTES, stream);
}

int dmpc_linearize(const dmpc_group* group, const dmpc_solver_params* params, double* As, double* Bs, double* Cs,
                   double* Qinv, double* qvec, double* Rinv, double* rvec, void* workspace, size_t workspace_bytes,
                   void* stream) {
  if (!group || group->horizons) return DMPC_ERR_INVALID;
  DevArgs* args = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(1, group, nullptr, params, args, &ws, &sm, &thr);
  if (rc == DMPC_OK && (ws > workspace_bytes || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0))
    rc = DMPC_ERR_WORKSPACE;
  if (rc == DMPC_OK && args->total_blocks > 0) {
    k_linearize<<<args->total_blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*args, workspace, As, Bs, Cs,
                                                                                        Qinv, qvec, Rinv, rvec);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) rc = cuda_rc(le);
  }
  delete args;
  return rc;
}

int dmpc_compute_gamma(int batch, int N, int nx, int nu, const double* As_x_Qinv, const double* Asnext_x_Qinvnext,
                       const double* Bs_x_Rinv, const double* Cs, const double* Q0inv, const double* qvec,
                       const double* rvec, double* gamma, void* stream) {
  if (batch < 0 || N < 1 || nx < 1 || nx > DMPC_MAX_NX || nu < 1 || nu > DMPC_MAX_NU) return DMPC_ERR_INVALID;
  if (batch == 0) return DMPC_OK;
  k_gamma_dense<<<batch, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(N, nx, nu, As_x_Qinv, Asnext_x_Qinvnext,
                                                                           Bs_x_Rinv, Cs, Q0inv, qvec, rvec, gamma);
  return cuda_rc(cudaGetLastError());
}

int dmpc_kkt_recover(int batch, int N, int nx, int nu, const double* lambda, const double* As_next, const double* As,
                     const double* Bs, const double* Qinv, const double* qvec, const double* Rinv, const double* rvec,
                     double* states, double* controls, void* stream) {
  if (batch < 0 || N < 1 || nx < 1 || nx > DMPC_MAX_NX || nu < 1 || nu > DMPC_MAX_NU) return DMPC_ERR_INVALID;
  if (batch == 0) return DMPC_OK;
  const size_t sm = 2 * (size_t)(N + 1) * nx * sizeof(double);
  if (sm > 227 * 1024) return DMPC_ERR_UNSUPPORTED;
  cudaError_t e = cudaFuncSetAttribute(k_recover_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return cuda_rc(e);
  k_recover_dense<<<batch, 256, sm, reinterpret_cast<cudaStream_t>(stream)>>>(N, nx, nu, lambda, As_next, As, Bs,
                                                                              Qinv, qvec, Rinv, rvec, states, controls);
  return cuda_rc(cudaGetLastError());
}

double dmpc_probe_fp32_fma(int blocks, int iters, float* out, void* stream) {
  if (blocks < 1 || iters < 1 || !out) return -1.0;
  k_fma_probe<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(iters, 1.0f, out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  return (double)blocks * 256.0 * (double)iters * 64.0 * 2.0;  // flops issued
}

size_t dmpc_schur_workspace_size(int batch, int N, int nx) {
  return align_up((size_t)batch * 4 * (N + 1) * nx * nx * sizeof(double), 256);
}

int dmpc_schur_assemble(int batch, int N, int nx, int nu, const double* As_next, const double* As, const double* Bs,
                        const double* Cs, const double* Qinv, const double* qvec, const double* Rinv,
                        const double* rvec, double* S, double* Phiinv, double* gamma, void* workspace,
                        size_t workspace_bytes, void* stream) {
  if (batch < 0 || N < 1 || nx < 1 || nx > DMPC_MAX_NX || nu < 1 || nu > DMPC_MAX_NU) return DMPC_ERR_INVALID;
  if (workspace_bytes < dmpc_schur_workspace_size(batch, N, nx)) return DMPC_ERR_WORKSPACE;
  if (batch == 0) return DMPC_OK;
  k_schur_dense<<<batch, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      N, nx, nu, As_next, As, Bs, Cs, Qinv, qvec, Rinv, rvec, S, Phiinv, gamma, reinterpret_cast<double*>(workspace));
  return cuda_rc(cudaGetLastError());
}

int dmpc_pcg_solve(int batch, int N, int nx, int nu, const double* S, const double* Phiinv, const double* gamma,
                   const double* lambda_guess, const double* As_next, const double* As, const double* Bs,
                   const double* Qinv, const double* qvec, const double* Rinv, const double* rvec, int max_iter,
                   double tol_epsilon, double* lambda, double* states, double* controls, int32_t* num_iterations,
                   double* convergence_eta, void* stream) {
  if (batch < 0 || N < 1 || nx < 1 || nx > DMPC_MAX_NX || nu < 1 || nu > DMPC_MAX_NU) return DMPC_ERR_INVALID;
  if (batch == 0) return DMPC_OK;
  const size_t sm = 128 * sizeof(double) + 5 * (size_t)(N + 1) * nx * sizeof(double);
  if (sm > 227 * 1024) return DMPC_ERR_UNSUPPORTED;
  cudaError_t e = cudaFuncSetAttribute(k_pcg_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return cuda_rc(e);
  k_pcg_dense<<<batch, 256, sm, reinterpret_cast<cudaStream_t>(stream)>>>(
      N, nx, nu, S, Phiinv, gamma, lambda_guess, As_next, As, Bs, Qinv, qvec, Rinv, rvec, max_iter, tol_epsilon,
      lambda, states, controls, num_iterations, convergence_eta);
  return cuda_rc(cudaGetLastError());
}

}  // extern "C"
