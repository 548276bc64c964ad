// The SQP kernels of one launch configuration and their host launch wrappers.  Compiled once
// per configuration: -DDMPC_CFG=0 (up to 512 threads, one CTA per SM), 1 (up to 256 threads,
// one CTA per SM, up to 255 registers a thread), 2 (256 threads, two CTAs per SM) and 3 (up to
// 384 threads, one CTA per SM, up to 168 registers a thread); solver.cu picks the configuration
// per launch.
#ifndef DMPC_CFG
#error "compile with -DDMPC_CFG=0, 1, 2 or 3"
#endif
#include "sqp_device.cuh"

// Static shared memory of the SQP kernels (the per-instance context, the scaled-basis flag, the
// work item and, in the rollout kernels, the per-step group and adjoint views and the state
// cotangent) must stay within the reserve the host's shared-memory budget sets aside.
static_assert(sizeof(dmpc_impl::Inst) + sizeof(dmpc_group) + sizeof(dmpc_adjoint) +
                      (2 * DMPC_MAX_NX + DMPC_MAX_NU) * sizeof(double) + 2 * sizeof(double) + 64 <= 2048,
              "static shared memory reserve too small");

#define DMPC_CAT2(a, b) a##b
#define DMPC_CAT(a, b) DMPC_CAT2(a, b)

namespace dmpc_impl {

cudaError_t DMPC_CAT(sqp_launch_cfg, DMPC_CFG)(int kind, const DevArgs& args, const LaunchExtra& ex, void* ws,
                                               int threads, size_t smem, cudaStream_t st) {
  const int grid = args.slots;
  cudaError_t e = cudaSuccess;
  switch (kind) {
    case kLaunchFwd:
      e = cudaFuncSetAttribute(k_sqp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) {
        k_sqp_fwd<<<grid, threads, smem, st>>>(args, ws);
        e = cudaGetLastError();
      }
      break;
    case kLaunchAdj:
      e = cudaFuncSetAttribute(k_sqp_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) {
        k_sqp_adj<<<grid, threads, smem, st>>>(args, ws);
        e = cudaGetLastError();
      }
      break;
    case kLaunchRolloutFwd:
      e = cudaFuncSetAttribute(k_rollout_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) {
        k_rollout_fwd<<<grid, threads, smem, st>>>(args, *ex.ro, ws);
        e = cudaGetLastError();
      }
      break;
    case kLaunchRolloutAdj:
      e = cudaFuncSetAttribute(k_rollout_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) {
        k_rollout_adj<<<grid, threads, smem, st>>>(args, *ex.ro, *ex.rr, ws);
        e = cudaGetLastError();
      }
      break;
#if DMPC_CFG == 0
    case kLaunchLinearize:
      k_linearize<<<grid, 256, 0, st>>>(args, ws, ex.As, ex.Bs, ex.Cs, ex.Qinv, ex.qv, ex.Rinv, ex.rv);
      e = cudaGetLastError();
      break;
#endif
    default:
      e = cudaErrorInvalidValue;
  }
  return e;
}

// Resident CTAs per SM of the solver kernels for this block size and dynamic shared memory
// (the smallest over the forward, adjoint and rollout kernels), or 0 if the runtime cannot say.
int DMPC_CAT(sqp_blocks_per_sm_cfg, DMPC_CFG)(int threads, size_t smem) {
  const void* kernels[4] = {reinterpret_cast<const void*>(k_sqp_fwd), reinterpret_cast<const void*>(k_sqp_adj),
                            reinterpret_cast<const void*>(k_rollout_fwd),
                            reinterpret_cast<const void*>(k_rollout_adj)};
  int best = 1 << 30;
  for (const void* k : kernels) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem) != cudaSuccess) return 0;
    if (n < best) best = n;
  }
  return best;
}

}  // namespace dmpc_impl
