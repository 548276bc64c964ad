/*
 * dmpc_xla.h -- XLA custom-call (FFI) handler core of the B200 differentiable-MPC solve.
 *
 * The reference exposes its solve to JAX programs as a jax.custom_vjp
 * (diffmpc/solvers/sqp.py:572-801): the forward is SQPSolver._solve (sqp.py:436-560), the
 * backward SQPSolver.solve_bwd (sqp.py:668-798).  A JAX binding of this library registers two
 * XLA FFI targets and pairs them in the same custom_vjp.  Each target receives XLA's device
 * buffers in the fixed operand orders below; the functions in this header map them onto
 * dmpc_solve_fwd / dmpc_solve_adj (dmpc.h) and check every buffer's size first.  They need no
 * XLA headers.  csrc/xla_ffi.cc also defines the XLA handler symbols dmpc_xla_fwd_handler and
 * dmpc_xla_adj_handler when compiled with -DDMPC_WITH_XLA_FFI and jaxlib's include directory;
 * jaxlib is not part of the image this library is built in, so that part is unvalidated.
 *
 * Buffers: device pointer + byte size (XLA's untyped_data() and size_bytes()).  Every array is
 * float64 unless marked int32, row-major, batch first; K = horizon + 1, mi =
 * params->num_scp_iteration_max, P = problem->n_model_params.  An optional buffer is given with
 * 0 bytes (its data pointer is then ignored).
 *
 * Forward arguments (DMPC_XLA_FWD_ARGS):
 *   0 dt (B)            1 initial_state (B,nx)   2 final_state (B,nx)
 *   3 reference_state (B,K,nx)   4 reference_control (B,K,nu)
 *   5 w_x (B,nx)        6 w_u (B,nu)             7 w_f (B,nx)      8 model_params (B,P)
 *   9 horizons (B) int32, optional (ragged batch)
 *   10 guess states (B,K,nx)   11 guess controls (B,K,nu)   12 guess dual (B,K,nx)
 * Forward results (DMPC_XLA_FWD_RETS):
 *   0 states (B,K,nx)   1 controls (B,K,nu)   2 dual (B,K,nx)   3 convergence_error (B)
 *   4 status (B) int32  5 num_iter (B) int32   6 convergence_errors (B,mi)
 *   7 linesearch_alphas (B,mi)   8 num_pcg_iters (B,mi) int32
 *   9 lin_states (B,K,nx)   10 lin_controls (B,K,nu)
 *   11 workspace (uint8, at least dmpc_xla_workspace_size bytes)
 * The guess is copied into results 0-2 unless XLA aliases them (same pointer); the
 * histories start from zero.
 *
 * Adjoint arguments (DMPC_XLA_ADJ_ARGS): 0-9 as the forward's, then
 *   10 states   11 controls   12 dual   13 lin_states   14 lin_controls  (forward results)
 *   15 dl_dstates (B,K,nx)   16 dl_dcontrols (B,K,nu)
 *   17 dual_backward_guess (B,K,nx), optional (zeros)
 * Adjoint results (DMPC_XLA_ADJ_RETS):
 *   0 dual_backward (B,K,nx)   1 g_initial_state (B,nx)   2 g_final_state (B,nx)
 *   3 g_w_x (B,nx)   4 g_w_u (B,nu)   5 g_w_f (B,nx)   6 g_reference_state (B,K,nx)
 *   7 g_reference_control (B,K,nu)   8 g_model_params (B,n_param_grads)
 *   9 num_pcg_iter (B) int32   10 workspace
 * Gradient results 1-8 and 9 are optional: a 0-byte result is not computed.
 *
 * Return codes are dmpc.h's: DMPC_ERR_INVALID for a wrong operand count, size or problem
 * description (nothing is launched), DMPC_ERR_WORKSPACE for a workspace below
 * dmpc_xla_workspace_size.
 */
#ifndef DMPC_XLA_H
#define DMPC_XLA_H

#include <stddef.h>
#include <stdint.h>

#include "dmpc.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The static part of the problem (the reference's ocp static parameters: model, horizon,
 * discretization scheme, penalize_control_reference) and the batch size.  XLA passes these as
 * the custom call's attributes. */
typedef struct dmpc_xla_problem {
  int32_t model, nx, nu, horizon, batch, scheme, penalize_control_reference, n_model_params;
} dmpc_xla_problem;

typedef struct dmpc_xla_buffer {
  void* data;
  uint64_t bytes;
} dmpc_xla_buffer;

#define DMPC_XLA_FWD_ARGS 13
#define DMPC_XLA_FWD_RETS 12
#define DMPC_XLA_ADJ_ARGS 18
#define DMPC_XLA_ADJ_RETS 11

/* Operand names in order, "args: a,b,...; rets: c,d,..." (for the binding's own checks). */
const char* dmpc_xla_fwd_operands(void);
const char* dmpc_xla_adj_operands(void);

/* Bytes of the workspace result: dmpc_workspace_size for this problem plus 256 bytes, so that the
 * handler can align the 256-byte boundary dmpc_solve_fwd asks for inside any XLA buffer.  0 for
 * an invalid problem. */
size_t dmpc_xla_workspace_size(const dmpc_xla_problem* problem, const dmpc_solver_params* params);

int dmpc_xla_solve_fwd(const dmpc_xla_problem* problem, const dmpc_solver_params* params,
                       const dmpc_xla_buffer* args, int n_args, const dmpc_xla_buffer* rets, int n_rets,
                       void* stream);

/* param_grad_index: HOST array of n_param_grads model-parameter indices (the custom call's
 * attribute), whose gradients go to result 8. */
int dmpc_xla_solve_adj(const dmpc_xla_problem* problem, const dmpc_solver_params* params,
                       const int32_t* param_grad_index, int n_param_grads, const dmpc_xla_buffer* args,
                       int n_args, const dmpc_xla_buffer* rets, int n_rets, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DMPC_XLA_H */
