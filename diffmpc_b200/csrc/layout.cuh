// Launch descriptors and workspace layout shared by the host code (solver.cu) and the SQP
// kernels (k_sqp.cu, compiled once per launch configuration).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/dmpc.h"

namespace dmpc_impl {

constexpr int kMaxGroups = 8;

// Launch configurations of the SQP kernels (dmpc_solver_params.cta_config).  kCfgWide: up to 512
// threads, one CTA per SM, 128 registers per thread.  kCfgRows: up to 256 threads, one CTA per
// SM, up to 255 registers per thread, which the compile-time row PCG needs to keep its W
// coefficients in registers without spilling; kCfgRows384 the same up to 384 threads (168
// registers).  kCfgDual: 256 threads, two CTAs per SM, 128 registers.
constexpr int kCfgWide = 0;
constexpr int kCfgRows = 1;
constexpr int kCfgDual = 2;
constexpr int kCfgRows384 = 3;

// Bytes at the start of every workspace that hold the persistent kernels' work counter.
constexpr size_t kQueueBytes = 256;

struct DevGroup {
  dmpc_group g;
  dmpc_adjoint a;
  int32_t first_item;   // index of this group's first instance in the launch's work order
  int32_t K;            // horizon + 1
  int32_t ld32;         // row stride of FP32 blocks and padded vectors (pad_ld)
  int32_t blocks_smem;  // FP32 blocks: 0 workspace, 1 shared memory, 2 per instance (shared if they fit)
  uint64_t smem_block_budget;  // mode 2: shared-memory bytes available for one instance's blocks
  uint32_t w64_off;     // mixed row path: shared-memory byte offset of the FP64 W blocks (0: workspace)
  int32_t pg_idx[DMPC_MAX_PARAM_GRADS];
};

// One launch.  The grid is `slots` persistent CTAs; each takes instances from the work counter
// at the start of the workspace (zeroed before the launch) until `total_items` are handed out,
// and solves each in its own slot of `slot_stride` bytes after the counter, so the workspace
// grows with the number of resident CTAs, not with the batch.
struct DevArgs {
  int32_t n_groups;
  int32_t total_items;
  int32_t slots;
  int32_t cfg;
  size_t slot_stride;
  dmpc_solver_params p;
  DevGroup grp[kMaxGroups];
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------- workspace layout (one slot)
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

// nx with a compile-time row PCG (pcg_rows_scaled, 4 rows per thread, ceil(nx / 4) threads per
// knot; pcg_rows_t in the two-CTA configuration, rows_tpk(nx) threads per knot)
__host__ __device__ inline bool rows_nx(int nx) {
  return nx == 3 || nx == 4 || nx == 6 || nx == 7 || nx == 8 || nx == 12 || nx == 13;
}

// Threads per knot of the two-CTA row PCG (pcg_rows_t): 4 rows each, a power of two.
__host__ __device__ constexpr int rows_tpk(int nx) { return nx <= 4 ? 1 : (nx <= 8 ? 2 : 4); }

// Bytes of the PCG vectors in shared memory (16-byte multiple).  FP64: five K nx vectors.
// Mixed: five padded FP32 vectors of K + 2 segments (the generic PCG; the row PCG uses two and
// keeps its FP64 exchange vector in the rest); in the two-CTA configuration with a row PCG, the
// larger of that and pcg_rows_t's four FP32 vectors of K + 2 segments of 4 rows_tpk(nx) floats
// plus its FP64 exchange vector (K + 2 segments of nx) and 12 constants.
__host__ __device__ inline size_t pcg_vec_bytes(int nx, int K, int precision, int cfg) {
  if (precision == DMPC_PREC_FP64) return 5 * (size_t)K * nx * sizeof(double);
  size_t b = align_up(5 * (size_t)(K + 2) * pad_ld(nx) * sizeof(float), 16);
  if (cfg == kCfgDual && rows_nx(nx)) {
    const size_t t = 4 * (size_t)(K + 2) * 4 * rows_tpk(nx) * sizeof(float) +
                     ((size_t)(K + 2) * nx + 12) * sizeof(double);
    if (align_up(t, 16) > b) b = align_up(t, 16);
  }
  return b;
}

// shared memory bytes of one CTA: 2x64 reduction doubles + 8 line-search values + PCG vectors
// (+ FP32 blocks)
__host__ __device__ inline size_t smem_bytes_for(int nx, int N, int precision, bool blocks_smem, int cfg) {
  const size_t K = N + 1;
  size_t b = 136 * sizeof(double) + pcg_vec_bytes(nx, (int)K, precision, cfg);
  if (precision != DMPC_PREC_FP64 && blocks_smem) b += (size_t)K * nx * pad_ld(nx) * sizeof(float);
  return align_up(b, 16);
}

// What each kernel launch does.
enum LaunchKind { kLaunchFwd = 0, kLaunchAdj = 1, kLaunchRolloutFwd = 2, kLaunchRolloutAdj = 3, kLaunchLinearize = 4 };

// Extra operands of the rollout and dense-linearization launches.
struct LaunchExtra {
  const dmpc_rollout* ro;
  const dmpc_rollout_adjoint* rr;
  double *As, *Bs, *Cs, *Qinv, *qv, *Rinv, *rv;
};

// Implemented in k_sqp.cu, one set per configuration.  `ws` is the whole workspace (work
// counter first); the caller zeroes the counter on `st` before the launch.
cudaError_t sqp_launch_cfg0(int kind, const DevArgs& args, const LaunchExtra& ex, void* ws, int threads,
                            size_t smem, cudaStream_t st);
cudaError_t sqp_launch_cfg1(int kind, const DevArgs& args, const LaunchExtra& ex, void* ws, int threads,
                            size_t smem, cudaStream_t st);
cudaError_t sqp_launch_cfg2(int kind, const DevArgs& args, const LaunchExtra& ex, void* ws, int threads,
                            size_t smem, cudaStream_t st);
cudaError_t sqp_launch_cfg3(int kind, const DevArgs& args, const LaunchExtra& ex, void* ws, int threads,
                            size_t smem, cudaStream_t st);
// resident CTAs per SM of the solver kernels (the smallest over the forward, adjoint and rollout kernels)
int sqp_blocks_per_sm_cfg0(int threads, size_t smem);
int sqp_blocks_per_sm_cfg1(int threads, size_t smem);
int sqp_blocks_per_sm_cfg2(int threads, size_t smem);
int sqp_blocks_per_sm_cfg3(int threads, size_t smem);

}  // namespace dmpc_impl
