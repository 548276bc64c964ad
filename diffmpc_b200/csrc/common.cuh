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
