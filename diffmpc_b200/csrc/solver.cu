// Host side of the batched SQP + Schur-complement PCG solver for sm_100a, and the dense-layout
// parity kernels of the lower-level entry points.
//
// The SQP kernels (k_sqp.cu, device code in sqp_device.cuh) solve one instance per CTA from
// start to finish: the SQP loop of diffmpc/solvers/sqp.py:436-560 (linearize -> assemble S,
// Phi^-1, gamma -> PCG -> recover (x, u) -> optional line search -> convergence test) runs
// entirely on the device with per-instance early exit, and the adjoint (sqp.py:668-798) reuses
// the same building blocks.  Each launch is a persistent grid of the CTAs that can be resident
// at once; they take instances of every group from a work counter, so one launch solves a
// ragged, mixed-model batch of any size in a workspace that grows with the resident CTAs only.
//
// Precision.  DMPC_PREC_FP64 runs the reference's FP64 PCG recurrence.  DMPC_PREC_MIXED runs the
// PCG iterations in FP32 in the basis scaled by the Cholesky factors of the diagonal blocks,
// where S and the block preconditioner Phi^-1 both reduce to the identity plus or minus one
// off-diagonal block per stage (see pcg_rows_scaled), with FP64 residual replacement: the
// residual gamma - S lambda and the stopping test eta = r^T Phi^-1 r <= eps use the FP64
// blocks, so the reference's absolute stopping rule (pcg.py:397-403) is applied in FP64.
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
#include "layout.cuh"
#include "models.cuh"

namespace dmpc_impl {
namespace {

// ---------------------------------------------------------------- dense-layout parity kernels
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

// ---------------------------------------------------------------- PSD projection (jax_utils.py:75-95)
// project_matrix_onto_positive_semidefinite_cone for a batch of n x n matrices, n <= 32: one warp
// per matrix.  As jnp.linalg.eigh does by default, the input is symmetrized, (M + M^T) / 2; its
// eigen-decomposition comes from the cyclic Jacobi method (Golub and Van Loan, Matrix
// Computations, sections 8.5.2-8.5.3: for each off-diagonal (p, q) the rotation with
// tau = (a_qq - a_pp) / (2 a_pq), t = sign(tau) / (|tau| + sqrt(1 + tau^2)), c = 1 / sqrt(1 + t^2),
// s = t c zeroes a_pq), sweeping until the off-diagonal mass is below (eps_64 ||A||_F)^2 or after
// kPsdMaxSweeps sweeps.  Lane k owns row k of the two rotated columns of A and V.  The result is
// V diag(max(lambda, minimum_eigenvalue)) V^T, symmetrized as the reference does; the projection
// onto the cone does not depend on the order or signs of the eigenvectors.  A matrix with a NaN or
// infinite entry gives all-NaN output (its eigen-decomposition is not a number, and jnp.maximum
// propagates NaN).  Shared memory per warp: A, V (n x n) and the clipped eigenvalues (n).
constexpr int kPsdMaxSweeps = 50;
constexpr int kPsdWarps = 4;
__global__ void __launch_bounds__(32 * kPsdWarps) k_psd_project(int batch, int n, const double* in,
                                                                  double min_eig, double* out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long b = (long long)blockIdx.x * kPsdWarps + warp;
  if (b >= batch) return;  // the whole warp leaves; the kernel has no CTA barrier
  const int nn = n * n;
  double* A = reinterpret_cast<double*>(smem) + (size_t)warp * (2 * nn + n);
  double* V = A + nn;
  double* mu = V + nn;
  const double* M = in + (size_t)b * nn;
  double fro = 0.0;
  for (int i = lane; i < nn; i += 32) {
    const int r = i / n, c = i - r * n;
    const double a = 0.5 * (M[i] + M[c * n + r]);
    A[i] = a;
    V[i] = (r == c) ? 1.0 : 0.0;
    fro += a * a;
  }
  fro = warp_sum(fro);
  double* o = out + (size_t)b * nn;
  if (!(fro <= 1.7976931348623157e308)) {  // a NaN or infinite entry: the eigen-decomposition is NaN
    for (int i = lane; i < nn; i += 32) o[i] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  __syncwarp();
  const double tol = 4.930380657631324e-32 * fro;  // (2^-52)^2 ||A||_F^2
  for (int sweep = 0; sweep < kPsdMaxSweeps; ++sweep) {
    double off = 0.0;
    for (int i = lane; i < nn; i += 32) {
      const int r = i / n;
      if (r != i - r * n) off += A[i] * A[i];
    }
    off = warp_sum(off);
    if (!(off > tol)) break;  // converged, or not a number
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p * n + q];
        if (apq == 0.0) continue;  // the same shared value in every lane
        const double app = A[p * n + p], aqq = A[q * n + q];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), sn = t * c;
        double akp = 0.0, akq = 0.0, vkp = 0.0, vkq = 0.0;
        if (lane < n) {
          akp = A[lane * n + p];
          akq = A[lane * n + q];
          vkp = V[lane * n + p];
          vkq = V[lane * n + q];
        }
        __syncwarp();
        if (lane < n) {
          if (lane != p && lane != q) {
            const double nkp = c * akp - sn * akq, nkq = sn * akp + c * akq;
            A[lane * n + p] = nkp;
            A[p * n + lane] = nkp;
            A[lane * n + q] = nkq;
            A[q * n + lane] = nkq;
          }
          V[lane * n + p] = c * vkp - sn * vkq;
          V[lane * n + q] = sn * vkp + c * vkq;
        }
        if (lane == 0) {
          A[p * n + p] = app - t * apq;
          A[q * n + q] = aqq + t * apq;
          A[p * n + q] = 0.0;
          A[q * n + p] = 0.0;
        }
        __syncwarp();
      }
    }
  }
  if (lane < n) {
    const double l = A[lane * n + lane];
    mu[lane] = (l < min_eig) ? min_eig : l;
  }
  __syncwarp();
  // P = V diag(mu) V^T into A, then out = (P + P^T) / 2
  for (int i = lane; i < nn; i += 32) {
    const int r = i / n, c = i - r * n;
    double a = 0.0;
    for (int k = 0; k < n; ++k) a = fma(V[r * n + k] * mu[k], V[c * n + k], a);
    A[i] = a;
  }
  __syncwarp();
  for (int i = lane; i < nn; i += 32) {
    const int r = i / n, c = i - r * n;
    o[i] = 0.5 * (A[i] + A[c * n + r]);
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

// Static shared memory of the SQP kernels (the per-instance context, the scaled-basis flag,
// the work item and, in the rollout kernels, the step views and the state cotangent; k_sqp.cu
// checks the bound at compile time).  It counts against the same per-CTA and per-SM limits as
// the dynamic request.
constexpr size_t kStaticSmemReserve = 2048;
// shared memory the runtime keeps per resident CTA
constexpr size_t kSmemPerCtaReserved = 1024;

struct DeviceInfo {
  int sms;            // multiprocessors
  size_t smem_optin;  // dynamic + static shared memory one CTA may use
  size_t smem_sm;     // shared memory of one SM
};

// Limits of the current device; B200 values when there is none (sizes computed then are only
// used to report a workspace size or to reach the launch, which fails).
DeviceInfo device_info() {
  DeviceInfo d{148, 227 * 1024, 228 * 1024};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return d;
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0) d.sms = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && v > 0)
    d.smem_optin = (size_t)v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess && v > 0)
    d.smem_sm = (size_t)v;
  return d;
}

// Mixed precision takes the compile-time row PCG (pcg_rows_scaled, 4 rows per thread) when the
// instance's K ceil(nx / 4) threads fit the CTA.
bool rows_path(const dmpc_solver_params* p, int nx, int K, int threads, int cfg = kCfgRows) {
  const int tpk = cfg == kCfgDual ? rows_tpk(nx) : (nx + 3) / 4;
  return p->precision == DMPC_PREC_MIXED && rows_nx(nx) && K * tpk <= threads;
}

// Threads per CTA (256..512): one thread per knot and row quadruple of the row PCG when it
// fits, else one thread per row up to 512 (several rows per thread beyond that).  At least 256:
// the FP64 setup phases (assembly, factorisations) spread over all threads, and short horizons
// leave too few rows to keep them busy (measured: nx=8, 40 knots runs 17 % faster at 256 threads
// than at 160).
// One thread per PCG row (per knot and row quadruple on the row PCG), rounded up to whole warps,
// at most 512.  The floor: 256 threads while the batch leaves SMs idle (fewer instances than
// two per SM: the assembly and linearization phases then use the extra warps), 64 otherwise (small
// instances then share an SM as several resident CTAs).
int choose_threads_wide(const dmpc_solver_params* p, int nx, int K, bool busy) {
  int rows = K * nx;
  if (p->precision == DMPC_PREC_MIXED && rows_nx(nx) && K * ((nx + 3) / 4) <= 512) rows = K * ((nx + 3) / 4);
  int t = ((rows + 31) / 32) * 32;
  const int floor = busy ? 64 : 256;
  if (t < floor) t = floor;
  if (t > 512) t = 512;
  return t;
}

// Shared memory one CTA needs for a group, and where the group's blocks go (G.blocks_smem,
// G.w64_off, G.smem_block_budget), for a CTA of `threads` threads with at most `cap` bytes.
// Returns 0 when even the minimum does not fit.
size_t group_smem(const dmpc_solver_params* p, const dmpc_group& g, DevGroup& G, int threads, size_t cap, int cfg) {
  const size_t base = smem_bytes_for(g.nx, g.horizon, p->precision, false, cfg);
  G.blocks_smem = 0;
  G.smem_block_budget = 0;
  G.w64_off = 0;
  if (base > cap) return 0;
  if (p->precision != DMPC_PREC_MIXED) return base;
  if (rows_path(p, g.nx, G.K, threads, cfg) && p->blocks_in_smem != 1) {
    // The row PCG reads the FP32 W blocks once per FP32 segment into registers (they stay in
    // the workspace); the FP64 W blocks of its residual replacements go to shared memory if they
    // fit, except in the two-CTA configuration: there they would take most of the SM's shared
    // memory from L1, and the replacements are rare (measured: the quadrotor N=60 headline runs
    // 7 % faster with them in the workspace).
    const size_t w64b = (size_t)G.K * g.nx * g.nx * sizeof(double);
    if (p->blocks_in_smem != 0 && cfg != kCfgDual && align_up(base, 16) + w64b <= cap) {
      G.w64_off = (uint32_t)align_up(base, 16);
      return G.w64_off + w64b;
    }
    return base;
  }
  // Generic path: FP32 blocks for every instance in shared memory (1); in a ragged group whose
  // longest instance does not fit, each instance checks its own size at run time (2); else
  // workspace (0).  Per-instance horizons live in device memory, hence mode 2.
  const size_t need_all = smem_bytes_for(g.nx, g.horizon, p->precision, true, cfg);
  if (p->blocks_in_smem != 0) {
    if (need_all <= cap) {
      G.blocks_smem = 1;
      return need_all;
    }
    if (g.horizons && base + (size_t)2 * g.nx * pad_ld(g.nx) * sizeof(float) <= cap) {
      G.blocks_smem = 2;
      G.smem_block_budget = (uint64_t)(cap - base);
      return cap;
    }
  }
  if (p->blocks_in_smem == 1) return 0;
  return base;
}

int blocks_per_sm(int cfg, int threads, size_t smem) {
  if (cfg == kCfgRows) return sqp_blocks_per_sm_cfg1(threads, smem);
  if (cfg == kCfgRows384) return sqp_blocks_per_sm_cfg3(threads, smem);
  if (cfg == kCfgDual) return sqp_blocks_per_sm_cfg2(threads, smem);
  return sqp_blocks_per_sm_cfg0(threads, smem);
}

// Validates the call and fills the launch descriptor: configuration, threads, shared memory,
// work order, slot size and count.  *ws_total: the workspace that holds a slot for every CTA
// that can be resident (counter included).
int fill_args(int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj, const dmpc_solver_params* p,
              DevArgs* args, size_t* ws_total, size_t* smem_max, int* threads) {
  if (n_groups < 1 || n_groups > kMaxGroups || !groups || !p) return DMPC_ERR_INVALID;
  if (p->precision != DMPC_PREC_FP64 && p->precision != DMPC_PREC_MIXED) return DMPC_ERR_INVALID;
  if (p->n_alphas < 1 || p->n_alphas > DMPC_MAX_ALPHAS) return DMPC_ERR_INVALID;
  if (p->threads_per_block != 0 &&
      (p->threads_per_block < 64 || p->threads_per_block > 512 || (p->threads_per_block & 31) != 0))
    return DMPC_ERR_INVALID;
  if (p->num_scp_iteration_max < 1 || p->pcg_max_iter < 1 || p->max_refinement < 1) return DMPC_ERR_INVALID;
  if (p->cta_config < DMPC_CTA_AUTO || p->cta_config > DMPC_CTA_DUAL) return DMPC_ERR_INVALID;
  memset(args, 0, sizeof(DevArgs));
  args->n_groups = n_groups;
  args->p = *p;
  const DeviceInfo dev = device_info();
  const size_t cap_wide = dev.smem_optin - kStaticSmemReserve;
  size_t cap_dual = dev.smem_sm / 2 - kSmemPerCtaReserved - kStaticSmemReserve;
  if (cap_dual > cap_wide) cap_dual = cap_wide;
  int total = 0;
  for (int k = 0; k < n_groups; ++k) {
    const dmpc_group& g = groups[k];
    if (!model_dims_ok(g.model, g.nx, g.nu)) return DMPC_ERR_UNSUPPORTED;
    if (g.horizon < 1 || g.batch < 0 || g.scheme < 0 || g.scheme > 2) return DMPC_ERR_INVALID;
    if (g.n_model_params != model_param_count(g.model, g.nx, g.nu)) return DMPC_ERR_INVALID;
    DevGroup& G = args->grp[k];
    G.g = g;
    if (adj) G.a = adj[k];
    G.K = g.horizon + 1;
    G.ld32 = pad_ld(g.nx);
    if (adj) {
      const int ng = adj[k].n_param_grads;
      if (ng < 0 || ng > g.n_model_params || ng > DMPC_MAX_PARAM_GRADS) return DMPC_ERR_INVALID;
      for (int q = 0; q < ng; ++q) {
        const int idx = adj[k].param_grad_index[q];
        if (idx < 0 || idx >= g.n_model_params) return DMPC_ERR_INVALID;
        G.pg_idx[q] = idx;
      }
    }
    total += g.batch;
  }
  // configuration, unless the caller chose one:
  // - two CTAs per SM (pcg_rows_t) when every group is mixed precision with a compile-time row
  //   layout whose K rows_tpk(nx) threads fit 256, the one-CTA row layout would need more than
  //   three warps, and the batch has more instances than SMs (measured: quadrotor N=60, B=4096,
  //   22 % faster than the one-CTA row layout; attitude N=50, B=1024, 102 threads, 4 %);
  // - else the row configuration when every group has a compile-time row PCG whose K ceil(nx/4)
  //   threads fit 384, or is ragged (instances too long for it take the generic PCG inside the
  //   same launch);
  // - else the wide configuration.
  int cfg = kCfgWide;
  if (p->cta_config == DMPC_CTA_ROWS) cfg = kCfgRows;
  else if (p->cta_config == DMPC_CTA_DUAL) cfg = kCfgDual;
  else if (p->cta_config == DMPC_CTA_AUTO && (p->threads_per_block == 0 || p->threads_per_block <= 384)) {
    bool rows = true, dual = p->threads_per_block == 0 || p->threads_per_block == 256;
    for (int k = 0; k < n_groups; ++k) {
      const int nx = groups[k].nx, K = groups[k].horizon + 1;
      rows = rows && (rows_path(p, nx, K, 384) || (p->precision == DMPC_PREC_MIXED && rows_nx(nx) && groups[k].horizons));
      dual = dual && rows_path(p, nx, K, 256, kCfgDual) && K * ((nx + 3) / 4) > 96;
    }
    if (dual && total > dev.sms) cfg = kCfgDual;
    else if (rows) cfg = kCfgRows;
  }
  const int max_thr = cfg == kCfgWide ? 512 : (cfg == kCfgRows ? 384 : 256);
  if (p->threads_per_block > max_thr || (cfg == kCfgDual && p->threads_per_block != 0 && p->threads_per_block != 256))
    return DMPC_ERR_INVALID;
  args->cfg = cfg;
  int thr = 0;
  if (p->threads_per_block > 0) {
    thr = p->threads_per_block;
  } else if (cfg == kCfgDual) {
    thr = 256;
  } else {
    const bool busy = total >= 2 * dev.sms;
    for (int k = 0; k < n_groups; ++k) {
      const int t = choose_threads_wide(p, groups[k].nx, groups[k].horizon + 1, busy);
      if (t > thr) thr = t;
    }
    if (thr > max_thr) thr = max_thr;
  }
  // more than 256 threads take the 384-thread bound (168 registers a thread)
  if (cfg == kCfgRows && thr > 256) cfg = kCfgRows384;
  args->cfg = cfg;
  const size_t cap = cfg == kCfgDual ? cap_dual : cap_wide;
  size_t smax = 0, stride = 0;
  for (int k = 0; k < n_groups; ++k) {
    const dmpc_group& g = groups[k];
    DevGroup& G = args->grp[k];
    const size_t sm = group_smem(p, g, G, thr, cap, cfg);
    if (sm == 0) return DMPC_ERR_UNSUPPORTED;
    if (sm > smax) smax = sm;
    const int ng = adj ? adj[k].n_param_grads : g.n_model_params;  // size for any later adjoint call
    const Layout L = make_layout(g.nx, g.nu, g.horizon, G.ld32, G.blocks_smem != 1,
                                 ng > g.n_model_params ? ng : g.n_model_params);
    if (L.bytes > stride) stride = L.bytes;
  }
  // work order: the most expensive instances (K nx^2) first, so that the last CTAs to finish
  // carry the short instances
  int order[kMaxGroups];
  for (int k = 0; k < n_groups; ++k) order[k] = k;
  for (int a = 1; a < n_groups; ++a)
    for (int b = a; b > 0; --b) {
      const dmpc_group &x = groups[order[b]], &y = groups[order[b - 1]];
      if ((double)(x.horizon + 1) * x.nx * x.nx > (double)(y.horizon + 1) * y.nx * y.nx) {
        const int t = order[b];
        order[b] = order[b - 1];
        order[b - 1] = t;
      }
    }
  int first = 0;
  for (int k = 0; k < n_groups; ++k) {
    args->grp[order[k]].first_item = first;
    first += groups[order[k]].batch;
  }
  int per_sm = blocks_per_sm(args->cfg, thr, smax);
  if (per_sm <= 0) per_sm = cfg == kCfgDual ? 2 : 1;
  const long long resident = (long long)dev.sms * per_sm;
  args->total_items = total;
  args->slots = (int)(total < resident ? total : resident);
  args->slot_stride = stride;
  *ws_total = kQueueBytes + (size_t)args->slots * stride;
  *smem_max = smax;
  *threads = thr;
  return DMPC_OK;
}

// Zeroes the work counter and launches `kind` with as many slots as the workspace holds.
int launch(int kind, DevArgs* args, const LaunchExtra& ex, void* workspace, size_t workspace_bytes, int threads,
           size_t smem, void* stream) {
  if (args->total_items == 0) return DMPC_OK;
  if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0 || workspace_bytes < kQueueBytes + args->slot_stride)
    return DMPC_ERR_WORKSPACE;
  const size_t fit = (workspace_bytes - kQueueBytes) / args->slot_stride;
  if ((size_t)args->slots > fit) args->slots = (int)fit;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return cuda_rc(e);
  if (args->cfg == kCfgRows) e = sqp_launch_cfg1(kind, *args, ex, workspace, threads, smem, st);
  else if (args->cfg == kCfgRows384) e = sqp_launch_cfg3(kind, *args, ex, workspace, threads, smem, st);
  else if (args->cfg == kCfgDual) e = sqp_launch_cfg2(kind, *args, ex, workspace, threads, smem, st);
  else e = sqp_launch_cfg0(kind, *args, ex, workspace, threads, smem, st);
  return cuda_rc(e);
}

int launch_groups(int kind, int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj,
                  const dmpc_solver_params* params, const LaunchExtra& ex, void* workspace, size_t workspace_bytes,
                  void* stream) {
  DevArgs* args = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(n_groups, groups, adj, params, args, &ws, &sm, &thr);
  if (rc == DMPC_OK) rc = launch(kind, args, ex, workspace, workspace_bytes, thr, sm, stream);
  delete args;
  return rc;
}

}  // namespace
}  // namespace dmpc_impl

using namespace dmpc_impl;

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
  p->cta_config = DMPC_CTA_AUTO;
}

size_t dmpc_workspace_size(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params) {
  DevArgs* a = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(n_groups, groups, nullptr, params, a, &ws, &sm, &thr);
  delete a;
  return rc == DMPC_OK ? ws : 0;
}

int dmpc_solve_fwd(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params, void* workspace,
                   size_t workspace_bytes, void* stream) {
  const LaunchExtra ex{};
  return launch_groups(kLaunchFwd, n_groups, groups, nullptr, params, ex, workspace, workspace_bytes, stream);
}

int dmpc_solve_adj(int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj, const dmpc_solver_params* params,
                   void* workspace, size_t workspace_bytes, void* stream) {
  if (!adj) return DMPC_ERR_INVALID;
  const LaunchExtra ex{};
  return launch_groups(kLaunchAdj, n_groups, groups, adj, params, ex, workspace, workspace_bytes, stream);
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
  LaunchExtra ex{};
  ex.ro = ro;
  ex.rr = rr;
  return launch_groups(kLaunchRolloutAdj, 1, group, adj, params, ex, workspace, workspace_bytes, stream);
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
  LaunchExtra ex{};
  ex.ro = ro;
  return launch_groups(kLaunchRolloutFwd, 1, group, nullptr, params, ex, workspace, workspace_bytes, stream);
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
  if (rc == DMPC_OK && need > (size_t)DMPC_NOALLOC_SCRATCH_BYTES) rc = DMPC_ERR_WORKSPACE;
  int dev = -1;
  if (rc == DMPC_OK) {
    const cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess) rc = cuda_rc(de);
    else if (dev < 0 || dev >= kNoallocMaxDevices) rc = DMPC_ERR_UNSUPPORTED;
  }
  void* base = nullptr;
  if (rc == DMPC_OK) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_device_ptr[dev] == nullptr) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) rc = cuda_rc(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
      else g_noalloc_device_ptr[dev] = p;
    }
    base = g_noalloc_device_ptr[dev];
  }
  if (rc == DMPC_OK) {
    const LaunchExtra ex{};
    rc = launch(kLaunchFwd, args, ex, base, (size_t)DMPC_NOALLOC_SCRATCH_BYTES, thr, sm, stream);
  }
  delete args;
  return rc;
}

int dmpc_linearize(const dmpc_group* group, const dmpc_solver_params* params, double* As, double* Bs, double* Cs,
                   double* Qinv, double* qvec, double* Rinv, double* rvec, void* workspace, size_t workspace_bytes,
                   void* stream) {
  if (!group || group->horizons) return DMPC_ERR_INVALID;
  LaunchExtra ex{};
  ex.As = As;
  ex.Bs = Bs;
  ex.Cs = Cs;
  ex.Qinv = Qinv;
  ex.qv = qvec;
  ex.Rinv = Rinv;
  ex.rv = rvec;
  DevArgs* args = new DevArgs;
  size_t ws = 0, sm = 0;
  int thr = 0;
  int rc = fill_args(1, group, nullptr, params, args, &ws, &sm, &thr);
  if (rc == DMPC_OK) {
    args->cfg = kCfgWide;  // the dense linearization kernel lives in the wide configuration's object
    rc = launch(kLaunchLinearize, args, ex, workspace, workspace_bytes, 256, 0, stream);
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

int dmpc_psd_project(int batch, int n, const double* matrices, double minimum_eigenvalue, double* out,
                     void* stream) {
  if (batch < 0 || n < 1 || n > 32 || (batch > 0 && (!matrices || !out))) return DMPC_ERR_INVALID;
  if (batch == 0) return DMPC_OK;
  const size_t sm = (size_t)kPsdWarps * (2 * (size_t)n * n + n) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_psd_project, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return cuda_rc(e);
  const long long blocks = ((long long)batch + kPsdWarps - 1) / kPsdWarps;
  if (blocks > 0x7fffffffLL) return DMPC_ERR_INVALID;
  k_psd_project<<<(unsigned)blocks, 32 * kPsdWarps, sm, reinterpret_cast<cudaStream_t>(stream)>>>(
      batch, n, matrices, minimum_eigenvalue, out);
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
