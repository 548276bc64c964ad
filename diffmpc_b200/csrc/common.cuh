// Shared device helpers: CTA-wide reductions and a warp-level SPD block inverse.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DMPC_FULL_MASK 0xffffffffu

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(DMPC_FULL_MASK, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(DMPC_FULL_MASK, v, o));
  return v;
}

// CTA-wide sum, deterministic (fixed order).  `red` holds 2 x 64 doubles and is
// used alternately, so back-to-back reductions need a single __syncthreads each:
// a buffer is rewritten only after another reduction's barrier has passed.
__device__ __forceinline__ double block_sum(double v, double* red, int& parity) {
  v = warp_sum(v);
  double* buf = red + (parity << 6);
  if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  const int nw = blockDim.x >> 5;
  for (int i = 0; i < nw; ++i) s += buf[i];
  parity ^= 1;
  return s;
}

// CTA-wide sum of per-thread FP32 partials: an FP32 butterfly inside each warp, then an FP64
// butterfly of width w2 (a power of two >= the warp count) over the warp sums.  Every thread
// gets the same value: a butterfly adds the same two operands in every lane of a pair, and
// addition is commutative.  `red` holds 2 x 64 doubles used alternately, as in block_sum.
__device__ __forceinline__ double block_sum_f32w(float v, double* red, int& parity, int w2) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(DMPC_FULL_MASK, v, o);
  double* buf = red + (parity << 6);
  const int lane = threadIdx.x & 31;
  if (lane == 0) buf[threadIdx.x >> 5] = (double)v;
  __syncthreads();
  const int l = lane & (w2 - 1);
  double s = (l < (int)(blockDim.x >> 5)) ? buf[l] : 0.0;
  for (int o = w2 >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(DMPC_FULL_MASK, s, o);
  parity ^= 1;
  return s;
}

// block_sum_f32w with a broadcast second stage: every thread reads all warp sums (FP64, two per
// 16-byte load) and adds them in one fixed order, instead of a butterfly of FP64 shuffles.  The
// CTA must have an even number of warps, at most 16.
__device__ __forceinline__ double block_sum_f32b(float v, double* red, int& parity) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(DMPC_FULL_MASK, v, o);
  double* buf = red + (parity << 6);
  if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = (double)v;
  __syncthreads();
  const double2* b2 = reinterpret_cast<const double2*>(buf);
  const int np = (int)(blockDim.x >> 6);
  double s = 0.0;
  if (np == 4) {
    const double2 a = b2[0], b = b2[1], c = b2[2], d = b2[3];
    s = ((a.x + a.y) + (b.x + b.y)) + ((c.x + c.y) + (d.x + d.y));
  } else {
    for (int i = 0; i < np; ++i) {
      const double2 a = b2[i];
      s += a.x + a.y;
    }
  }
  parity ^= 1;
  return s;
}

// Smallest power of two >= the CTA's warp count (the width of block_sum_f32w's second stage).
__device__ __forceinline__ int warp_pow2() {
  const int nw = blockDim.x >> 5;
  int w = 1;
  while (w < nw) w <<= 1;
  return w;
}

// a / b rounded to FP32, for the FP32 step lengths of the PCG recursion: an FP32 division of the
// rounded operands while both are normal floats away from the ends of the range (one FP32
// rounding more than (float)(a / b)), else the FP64 quotient rounded.  NaN takes the FP64 path.
__device__ __forceinline__ float quot32(double a, double b) {
  const float fa = (float)a, fb = (float)b;
  const float aa = fabsf(fa), ab = fabsf(fb);
  if (aa >= 1e-30f && ab >= 1e-30f && aa <= 1e30f && ab <= 1e30f) return fa / fb;
  return (float)(a / b);
}

// CTA-wide max.  NaN propagates (a NaN operand makes the result NaN).
__device__ __forceinline__ double block_max(double v, double* red, int& parity) {
  bool nan = v != v;
  v = warp_max(nan ? 0.0 : v);
  unsigned anynan = __ballot_sync(DMPC_FULL_MASK, nan);
  double* buf = red + (parity << 6);
  if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = anynan ? __longlong_as_double(0x7ff8000000000000ll) : v;
  __syncthreads();
  double s = buf[0];
  const int nw = blockDim.x >> 5;
  for (int i = 1; i < nw; ++i) {
    double b = buf[i];
    s = (b != b || s != s) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(s, b);
  }
  parity ^= 1;
  return s;
}

// In-place Gauss-Jordan inverse of an SPD n x n block by ONE warp.
// L (n x n, row-major) holds the matrix on entry and is destroyed; R receives
// the inverse.  Lane c owns augmented columns c and c + 32 of [L | R].
// SPD blocks need no pivoting (every pivot is a positive Schur complement).
__device__ inline void warp_spd_inverse(double* L, double* R, int n) {
  const int lane = threadIdx.x & 31;
  const int ncol = 2 * n;
  for (int c = lane; c < ncol; c += 32) {
    if (c >= n)
      for (int i = 0; i < n; ++i) R[i * n + (c - n)] = (i == c - n) ? 1.0 : 0.0;
  }
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    const double inv_piv = 1.0 / L[k * n + k];
    __syncwarp();
    for (int c = lane; c < ncol; c += 32) {
      if (c < n)
        L[k * n + c] = (c == k) ? 1.0 : L[k * n + c] * inv_piv;
      else
        R[k * n + (c - n)] *= inv_piv;
    }
    __syncwarp();
    for (int c = lane; c < ncol; c += 32) {
      if (c == k) continue;
      double* colp = (c < n) ? (L + c) : (R + (c - n));
      const double rk = colp[k * n];
      for (int i = 0; i < n; ++i) {
        if (i == k) continue;
        colp[i * n] -= L[i * n + k] * rk;
      }
    }
    __syncwarp();
    if (lane == 0)
      for (int i = 0; i < n; ++i)
        if (i != k) L[i * n + k] = 0.0;
    __syncwarp();
  }
}

// Cholesky factor and its inverse for one SPD n x n block (n <= 32) by ONE warp.
// A (row-major) holds the block on entry; its lower triangle is overwritten by L
// with A = L L^T.  X (n x n, row-major) receives L^-1, zeros above the diagonal
// included.  Lane i owns row i of A during the factorisation and column i of X
// during the forward substitution.  Returns false in every lane if a pivot is not
// positive and finite (the block is not numerically SPD).
__device__ inline bool warp_chol_inverse(double* A, double* X, int n) {
  const int lane = threadIdx.x & 31;
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    const double piv = A[k * n + k];
    ok = ok && piv > 0.0 && isfinite(piv);
    const double d = sqrt(piv);
    __syncwarp();
    if (lane == k) A[k * n + k] = d;
    if (lane > k && lane < n) A[lane * n + k] = A[lane * n + k] / d;
    __syncwarp();
    if (lane > k && lane < n) {
      const double lik = A[lane * n + k];
      for (int j = k + 1; j <= lane; ++j) A[lane * n + j] -= lik * A[j * n + k];
    }
    __syncwarp();
  }
  if (lane < n) {
    const int j = lane;
    for (int i = 0; i < j; ++i) X[i * n + j] = 0.0;
    X[j * n + j] = 1.0 / A[j * n + j];
    for (int i = j + 1; i < n; ++i) {
      double acc = 0.0;
      for (int k = j; k < i; ++k) acc = fma(A[i * n + k], X[k * n + j], acc);
      X[i * n + j] = -acc / A[i * n + i];
    }
  }
  __syncwarp();
  return ok;
}

// Register-resident variant for compile-time NX: a group of W lanes (W = 16 for NX <= 16,
// else 32; a warp holds 32 / W groups, each on its own block) factors the SPD block th
// (NX x NX, row-major) as L L^T and writes X = L^-1 to li (row-major, zeros above the
// diagonal).  Lane i of the group holds row i of the block, then of L, in registers; the
// forward substitution gives lane c column c of X.  Operands cross lanes by width-W
// shuffles, so the only memory traffic is one read of th and one coalesced write of X.
// Each pivot's reciprocal is formed once and reused by the substitution.  Lanes >= NX
// mirror row 0, and a group with `active` false (no block left for it) computes on th
// without storing; all lanes of the warp must call this together.  Returns false if a
// pivot of an active group is not positive and finite.
template <int NX, int W>
__device__ __forceinline__ bool group_chol_inverse_regs(const double* __restrict__ th, double* __restrict__ li,
                                                        bool active) {
  static_assert(NX <= W && (W == 16 || W == 32), "one lane per row");
  const int lane = threadIdx.x & (W - 1);
  const int r = lane < NX ? lane : 0;
  double a[NX], rd[NX];
#pragma unroll
  for (int j = 0; j < NX; ++j) a[j] = th[r * NX + j];
  bool ok = true;
#pragma unroll
  for (int k = 0; k < NX; ++k) {
    const double piv = __shfl_sync(DMPC_FULL_MASK, a[k], k, W);
    ok = ok && piv > 0.0 && isfinite(piv);
    const double d = sqrt(piv);
    rd[k] = 1.0 / d;
    a[k] = (lane == k) ? d : a[k] * rd[k];  // lanes > k: L[lane][k]; lanes < k keep a finished row
#pragma unroll
    for (int j = k + 1; j < NX; ++j) {
      const double ljk = __shfl_sync(DMPC_FULL_MASK, a[k], j, W);
      if (lane >= j) a[j] = fma(-a[k], ljk, a[j]);
    }
  }
  // X[i][c] = (delta_ic - sum_{k<i} L[i][k] X[k][c]) / L[i][i]; lane c keeps column c
  double x[NX];
#pragma unroll
  for (int i = 0; i < NX; ++i) {
    double acc = (lane == i) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k) acc = fma(-__shfl_sync(DMPC_FULL_MASK, a[k], i, W), x[k], acc);
    x[i] = acc * rd[i];
  }
  if (active && lane < NX) {
#pragma unroll
    for (int i = 0; i < NX; ++i) li[i * NX + lane] = x[i];
  }
  return ok || !active;
}
