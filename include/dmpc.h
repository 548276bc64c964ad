/*
 * dmpc.h -- C ABI of the B200 (sm_100a) batched differentiable-MPC inner solve.
 *
 * The library solves many independent optimal-control problems of the form
 *
 *   min  sum_{t<N} w_x.(x_t - xref_t)^2 + w_u.(u_t - uref_t)^2
 *        + (w_x + w_f).(x_N - x_final)^2
 *   s.t. x_0 = x_init,  x_{t+1} = F(x_t, u_t)   (one Euler / midpoint / RK4 step)
 *
 * by SQP whose QPs are solved with the Schur-complement block-tridiagonal
 * preconditioned conjugate gradient method, and differentiates the solution
 * with the implicit-function adjoint that reuses the same Schur/PCG machinery.
 * It replaces, call for call, the reference's JAX solver:
 *
 *   dmpc_solve_fwd      <- SQPSolver._solve                 diffmpc/solvers/sqp.py:436-560
 *   dmpc_solve_adj      <- SQPSolver _solve_bwd/_solve_bwd_pcg/_compute_mixed_derivatives
 *                                                            diffmpc/solvers/sqp.py:605-798
 *   dmpc_schur_assemble <- PCGOptimalControl.compute_S_Phiinv + compute_gamma
 *                                                            diffmpc/solvers/pcg.py:160-288
 *   dmpc_pcg_solve      <- PCGOptimalControl.solve_KKT_Schur diffmpc/solvers/pcg.py:350-445
 *                          (+ get_states_controls_from_kkt_multipliers pcg.py:290-348)
 *   dmpc_compute_gamma  <- PCGOptimalControl.compute_gamma   diffmpc/solvers/pcg.py:245-288
 *   dmpc_kkt_recover    <- PCGOptimalControl.get_states_controls_from_kkt_multipliers
 *                                                            diffmpc/solvers/pcg.py:290-348
 *   dmpc_linearize      <- OptimalControlProblem.get_dynamics_linearized_matrices_with_states_controls
 *                          + get_cost_linearized_matrices + SQPSolver.get_cost_terms
 *                                                            diffmpc/problems/optimal_control_problem.py:249-398,
 *                                                            diffmpc/solvers/sqp.py:160-260
 *
 * Conventions.  Every pointer is a DEVICE pointer unless stated otherwise;
 * floating-point data is float64, row-major, instance-major (SoA over the
 * batch).  N is the reference's `horizon`; K = N + 1 knots.  All calls are
 * stream-ordered, never synchronise the host, and never allocate: scratch
 * memory is the caller's `workspace` (size from dmpc_workspace_size).
 *
 * Launches are persistent: a grid of the CTAs that can be resident at once takes the
 * instances from a work counter kept in the first 256 bytes of the workspace (zeroed by a
 * stream-ordered memset before each launch), and each CTA solves its instances one after
 * another in its own slot of the rest of the workspace.  The workspace therefore grows with
 * the number of resident CTAs, not with the batch; a workspace smaller than
 * dmpc_workspace_size but holding the counter and at least one slot also works, with fewer
 * CTAs.  Calls that share a workspace must not overlap on the GPU.
 * Return value: DMPC_OK or a DMPC_ERR_* code; per-instance solver status is
 * written to device memory with the reference's values (0 success, -100 error).
 */
#ifndef DMPC_H_
#define DMPC_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMPC_ABI_VERSION 3

/* return codes */
#define DMPC_OK 0
#define DMPC_ERR_INVALID 1      /* bad descriptor / sizes (the reference raises ValueError/KeyError) */
#define DMPC_ERR_WORKSPACE 2    /* workspace too small or misaligned */
#define DMPC_ERR_CUDA 3         /* a CUDA runtime call failed */
#define DMPC_ERR_UNSUPPORTED 4  /* model or option not supported (reference: NotImplementedError) */

/* per-instance solver status, SolverReturnStatus (diffmpc/solvers/sqp.py:31-35) */
#define DMPC_STATUS_SUCCESS 0
#define DMPC_STATUS_ERROR (-100)

/* dynamics models (diffmpc/dynamics/, one file per model).  Model parameter vectors:
 *   LINEAR      nx, nu free;  [A (nx*nx), B (nx*nu), b (nx)]     linear_dynamics.py:46-70
 *   QUADROTOR   nx=13, nu=4;  [mass, inertia (3x3 row-major, 9)] quadrotor_dynamics.py:84-133
 *   SPACECRAFT  nx=3,  nu=3;  [inertia_vector (3)]                spacecraft_dynamics.py:31-66
 *   ATTITUDE    nx=7,  nu=3;  [inertia_vector (3)]  quaternion + rate (no reference counterpart)
 *   CARTPOLE    nx=4,  nu=1;  [masscart, masspole, length, gravity] cartpole_dynamics.py:36-80 */
#define DMPC_MODEL_LINEAR 0
#define DMPC_MODEL_QUADROTOR 1
#define DMPC_MODEL_SPACECRAFT 2
#define DMPC_MODEL_ATTITUDE 3
#define DMPC_MODEL_CARTPOLE 4

/* DiscretizationScheme (diffmpc/dynamics/integrators.py:12-17) */
#define DMPC_EULER 0
#define DMPC_MIDPOINT 1
#define DMPC_RK4 2

/* PCG arithmetic */
#define DMPC_PREC_FP64 0   /* all-FP64 PCG, the reference's arithmetic */
#define DMPC_PREC_MIXED 1  /* FP32 PCG iterations with FP64 residual replacement */

#define DMPC_MAX_NX 32
#define DMPC_MAX_NU 16
#define DMPC_MAX_ALPHAS 8
#define DMPC_MAX_PARAM_GRADS 64
#define DMPC_MAX_GROUPS 8

/* Solver options: diffmpc/solvers/params/sqp.yaml plus the precision controls. */
typedef struct dmpc_solver_params {
  double tol_convergence;         /* sqp.yaml tol_convergence */
  int32_t num_scp_iteration_max;  /* sqp.yaml num_scp_iteration_max */
  int32_t linesearch;             /* sqp.yaml linesearch (0/1) */
  double linesearch_eta;          /* sqp.yaml linesearch_eta */
  int32_t n_alphas;               /* len(linesearch_alphas) <= DMPC_MAX_ALPHAS */
  double alphas[DMPC_MAX_ALPHAS]; /* sqp.yaml linesearch_alphas */
  int32_t warm_start_backward;    /* sqp.yaml warm_start_backward */
  int32_t pcg_max_iter;           /* sqp.yaml pcg.max_iter.  MIXED: FP32 iterations use at most half of it;
                                     an FP64 fallback recurrence then gets a full budget of its own */
  double pcg_tol_epsilon;         /* sqp.yaml pcg.tol_epsilon (absolute, on eta = r^T Phi^-1 r) */
  int32_t precision;              /* DMPC_PREC_* */
  int32_t max_refinement;         /* MIXED: FP64 residual replacements per QP solve before the FP64
                                     fallback */
  double inner_rel_tol;           /* MIXED: the FP32 recursion's eta falls by this factor between FP64
                                     residual replacements */
  int32_t threads_per_block;      /* 0 = automatic: one thread per knot and row quadruple of the FP32 PCG
                                     (else per row), 256..512; or 64..512, a multiple of 32, within the
                                     cta_config's limit (diffmpc_b200.autotune) */
  int32_t blocks_in_smem;         /* MIXED, the FP32 scaled off-diagonal blocks: -1 shared memory when they
                                     fit (per instance in a ragged group), 0 workspace, 1 require shared */
  int32_t cta_config;             /* DMPC_CTA_*: CTA shape of the solver kernels (diffmpc_b200.autotune) */
} dmpc_solver_params;

/* dmpc_solver_params.cta_config.  AUTO: DUAL when every group is mixed precision with a
 * compile-time row layout (nx in {3,4,6,7,8,12,13}) whose K rows_tpk(nx) threads fit 256
 * (rows_tpk = 1, 2, 4 for nx <= 4, 8, 16), its one-CTA row layout would need more than three warps
 * and the batch has more instances than SMs; else ROWS when every group has a row layout whose
 * K ceil(nx/4) threads fit 384 (or is ragged: its longer instances take the generic PCG); else
 * WIDE. */
#define DMPC_CTA_AUTO 0
#define DMPC_CTA_WIDE 1 /* up to 512 threads (threads_per_block or automatic), one CTA per SM */
#define DMPC_CTA_ROWS 2 /* 256..384 threads (threads_per_block or automatic), one CTA per SM; up to 255
                           registers per thread at 256 threads, 168 above, for the row PCG */
#define DMPC_CTA_DUAL 3 /* 256 threads, two CTAs per SM, 128 registers per thread; mixed precision
                           takes the row PCG with one register copy of each scaled block */

/* One group = instances sharing model, nx, nu and max horizon (a batch).
 * Per-instance horizons may differ (ragged batch): arrays are padded to K = horizon + 1
 * rows and instance i uses its first horizons[i] + 1 rows. */
typedef struct dmpc_group {
  int32_t model, nx, nu;
  int32_t horizon;                 /* N (maximum over the group when `horizons` is given) */
  int32_t batch;                   /* number of instances */
  int32_t scheme;                  /* DMPC_EULER / DMPC_MIDPOINT / DMPC_RK4 */
  int32_t penalize_control_reference;
  int32_t n_model_params;          /* length of each instance's model parameter vector */
  const int32_t* horizons;         /* (batch) per-instance N_i in [1, horizon], or NULL */
  /* problem parameters (optimal_control_problem.py:153-206 key names) */
  const double* dt;                /* (batch) discretization_resolution */
  const double* initial_state;     /* (batch, nx) */
  const double* final_state;       /* (batch, nx) */
  const double* reference_state;   /* (batch, K, nx) reference_state_trajectory */
  const double* reference_control; /* (batch, K, nu) reference_control_trajectory */
  const double* w_x;               /* (batch, nx) weights_penalization_reference_state_trajectory */
  const double* w_u;               /* (batch, nu) weights_penalization_control_squared */
  const double* w_f;               /* (batch, nx) weights_penalization_final_state */
  const double* model_params;      /* (batch, n_model_params) */
  /* initial guess on entry, solution on exit (SQPSolution fields, sqp.py:38-57) */
  double* states;                  /* (batch, K, nx) */
  double* controls;                /* (batch, K, nu); row N is zero on exit (pcg.py:346) */
  double* dual;                    /* (batch, K, nx) KKT multipliers */
  double* convergence_error;       /* (batch) in: guess value, out: final */
  int32_t* status;                 /* (batch) out */
  int32_t* num_iter;               /* (batch) out */
  double* convergence_errors;      /* (batch, num_scp_iteration_max) in/out */
  double* linesearch_alphas;       /* (batch, num_scp_iteration_max) in/out */
  int32_t* num_pcg_iters;          /* (batch, num_scp_iteration_max) in/out */
  double* lin_states;              /* (batch, K, nx) out: iterate of the last linearization */
  double* lin_controls;            /* (batch, K, nu) out */
  /* precision record of each QP solve, optional (NULL: not written); (batch, num_scp_iteration_max) out */
  int32_t* num_pcg_corrections;    /* FP64 residual replacements of the FP32 PCG (0 in FP64) */
  int32_t* num_pcg_fp64_iters;     /* of num_pcg_iters, the iterations run by the FP64 recurrence */
} dmpc_group;

/* Adjoint inputs/outputs for one group (sqp.py:668-798).  Gradient outputs
 * that are NULL are not computed. */
typedef struct dmpc_adjoint {
  const double* dl_dstates;          /* (batch, K, nx) cotangent of states */
  const double* dl_dcontrols;        /* (batch, K, nu) cotangent of controls (row N unused) */
  const double* dual_backward_guess; /* (batch, K, nx) warm start, or NULL for zeros */
  double* dual_backward;             /* (batch, K, nx) out: adjoint multipliers */
  int32_t* num_pcg_iter;             /* (batch) out, may be NULL */
  double* g_initial_state;           /* (batch, nx) */
  double* g_final_state;             /* (batch, nx) */
  double* g_w_x;                     /* (batch, nx) */
  double* g_w_u;                     /* (batch, nu) */
  double* g_w_f;                     /* (batch, nx) */
  double* g_reference_state;         /* (batch, K, nx) */
  double* g_reference_control;       /* (batch, K, nu) */
  int32_t n_param_grads;             /* number of model-parameter gradients (<= DMPC_MAX_PARAM_GRADS) */
  const int32_t* param_grad_index;   /* (n_param_grads) HOST array of model-parameter indices */
  double* g_model_params;            /* (batch, n_param_grads) */
  /* adjoint solution (x~, u~), optional (batch, K, nx) / (batch, K, nu) */
  double* adj_states;
  double* adj_controls;
  /* precision record of the adjoint QP solve, optional: (batch) out, as in dmpc_group */
  int32_t* num_pcg_corrections;
  int32_t* num_pcg_fp64_iter;
} dmpc_adjoint;

/* Closed-loop rollout (benchmarking/reinforcement-learning/benchmark_diffmpc.py:140-175, the
 * rollout_step scanned with lax.scan and vmapped over instances).  For k = 0..num_steps-1:
 * solve the MPC with initial state x_k starting from step k-1's solution (warm_start) or from
 * the group's initial guess, apply u_k = controls[0], simulate x_{k+1} (see `simulator`) and add
 * the weighted squared deviations of x_{k+1} and u_k to the running cost (the reference scripts'
 * negated reward: |x|^2 + |u|^2 for the linear benchmark, 10 |x|^2 + |u|^2 for the spacecraft
 * one, |p - p_ref|^2 + 0.1 |u - u_ref|^2 for the RL_quadrotor notebook).  All pointers are device memory; K = horizon+1,
 * T = num_steps. */
#define DMPC_SIM_LINEAR 0 /* x+ = A x + B u + b (benchmark_diffmpc.py:148-150) */
#define DMPC_SIM_MODEL 1  /* x+ = x + dt f(x, u): one Euler step of the group's model with each instance's
                             dt and model parameters (spacecraft/benchmark_diffmpc.py:87-89) */
#define DMPC_SIM_MODEL_SCHEME 2 /* one step of the group's own integrator (its discretization scheme),
                                   as the RL_quadrotor notebook simulates (cell 12) */
typedef struct {
  int32_t num_steps;                /* T >= 1 */
  int32_t warm_start;               /* 1: step k starts from step k-1's solution */
  int32_t simulator;                /* DMPC_SIM_LINEAR, DMPC_SIM_MODEL or DMPC_SIM_MODEL_SCHEME */
  int32_t reserved;                 /* 0 */
  /* running cost += sum_i ws_i (x_{k+1,i} - xr_i)^2 + sum_j wc_j (u_{k,j} - ur_j)^2; all four
   * arrays are shared by the batch, and a null reference is zero */
  const double* cost_state_weights;   /* (nx) */
  const double* cost_control_weights; /* (nu) */
  const double* cost_state_ref;       /* (nx) or null */
  const double* cost_control_ref;     /* (nu) or null */
  const double* sim_A;              /* (batch, nx, nx) DMPC_SIM_LINEAR only */
  const double* sim_B;              /* (batch, nx, nu) DMPC_SIM_LINEAR only */
  const double* sim_b;              /* (batch, nx)     DMPC_SIM_LINEAR only */
  double* step_initial_state;       /* (T+1, batch, nx): x_0 (copied from the group) .. x_T */
  double* step_states;              /* (T, batch, K, nx) solutions */
  double* step_controls;            /* (T, batch, K, nu) */
  double* step_dual;                /* (T, batch, K, nx) */
  double* step_lin_states;          /* (T, batch, K, nx) last linearization points (adjoint) */
  double* step_lin_controls;        /* (T, batch, K, nu) */
  int32_t* step_status;             /* (T, batch) */
  int32_t* step_num_iter;           /* (T, batch) */
  double* step_convergence_error;   /* (T, batch) */
  double* step_convergence_errors;  /* (T, batch, num_scp_iteration_max) */
  double* step_linesearch_alphas;   /* (T, batch, num_scp_iteration_max) */
  int32_t* step_num_pcg_iters;      /* (T, batch, num_scp_iteration_max) */
  double* running_cost;             /* (batch) */
} dmpc_rollout;

/* Reverse sweep of a rollout's gradient.  All pointers are device memory. */
typedef struct {
  const double* cost_cotangent;     /* (batch) dL/d running_cost */
  int32_t through_state;            /* 1: add each solve's dL/dx_k (the reference's custom VJP does not) */
  double* scratch_dl_dcontrols;     /* (batch, K, nu) working array */
  double* scratch_dual;             /* (batch, K, nx) working array */
  double* g_initial_state;          /* (batch, nx) dL/dx_0, optional */
} dmpc_rollout_adjoint;

int dmpc_abi_version(void);
const char* dmpc_error_string(int code);
/* Name of the last CUDA runtime error an entry point returned DMPC_ERR_CUDA for on the
 * calling thread ("cudaSuccess" if none).  No reference counterpart: the reference
 * surfaces XLA runtime errors as Python exceptions. */
const char* dmpc_last_cuda_error(void);

/* Bytes of workspace the forward/adjoint calls need for these groups: the work counter plus one
 * slot (the largest instance's scratch) per CTA that can be resident on the current device. */
size_t dmpc_workspace_size(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params);

/* Fills `params` with the reference defaults (sqp.yaml:1-11) and MIXED precision. */
void dmpc_default_params(dmpc_solver_params* params);

/* Forward SQP solve of every instance of every group (n_groups <= DMPC_MAX_GROUPS) in ONE kernel launch
 * (SQPSolver._solve, sqp.py:436-560).  Workspace must be 256-byte aligned. */
int dmpc_solve_fwd(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free forward solve.  No reference counterpart: the reference (JAX)
 * never hands out raw device memory.  It exists for callers that cannot call
 * cudaMalloc at solve time -- a real-time MPC control loop where an allocation may
 * stall the device for an unbounded time, or a host framework that owns the device
 * allocator and only lends a stream (e.g. a plugin or custom-call handler).
 * Same semantics and outputs as dmpc_solve_fwd, but the scratch memory is a fixed
 * array of DMPC_NOALLOC_SCRATCH_BYTES (32 MiB) inside this library, held on every GPU
 * that loads the library until the process exits.  Problems that need more scratch
 * than that (dmpc_workspace_size) are rejected with DMPC_ERR_WORKSPACE and nothing is
 * launched.  The first call on a device looks up the array's device address with that
 * device current; make that call before any stream capture.  The address is cached per device
 * for the life of the process: after cudaDeviceReset the cached address is stale, so a process
 * that resets a device must not call this entry point on that device again.  All calls share the one
 * array and it keeps the previous call's contents (the solver initialises everything it
 * reads), so calls that may overlap on the GPU -- on different streams, or from several
 * host threads -- race and must be serialised by the caller. */
#define DMPC_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int dmpc_solve_fwd_noalloc(int n_groups, const dmpc_group* groups, const dmpc_solver_params* params,
                           void* stream);

/* Adjoint solve + gradients at the forward solution held in `groups`
 * (states/controls/dual = z*, lambda*; lin_states/lin_controls = last linearization).
 * One launch for all groups (sqp.py:668-798). */
int dmpc_solve_adj(int n_groups, const dmpc_group* groups, const dmpc_adjoint* adj,
                   const dmpc_solver_params* params, void* workspace, size_t workspace_bytes,
                   void* stream);

/* ---- lower-level entry points, reference dense layouts (pcg.py:13-67) ---- */

/* Linearize at (states, controls) of `group` (no solve): writes As (batch,N,nx,nx),
 * Bs (batch,N,nx,nu), Cs (batch,K,nx), Qinv (batch,K,nx,nx), qvec (batch,K,nx),
 * Rinv (batch,N,nu,nu), rvec (batch,N,nu).  As_next is -I (optimal_control_problem.py:393-397).
 * Uniform horizon only; workspace from dmpc_workspace_size(1, group, params). */
int dmpc_linearize(const dmpc_group* group, const dmpc_solver_params* params, double* As, double* Bs,
                   double* Cs, double* Qinv, double* qvec, double* Rinv, double* rvec, void* workspace,
                   size_t workspace_bytes, void* stream);

/* compute_S_Phiinv + compute_gamma for general QP data (pcg.py:160-288), batch of
 * `batch` uniform problems: As_next, As (batch,N,nx,nx), Bs (batch,N,nx,nu), Cs (batch,K,nx),
 * Qinv (batch,K,nx,nx), qvec (batch,K,nx), Rinv (batch,N,nu,nu), rvec (batch,N,nu)
 *  -> S, Phiinv (batch,K,nx,3nx), gamma (batch,K,nx). */
int dmpc_schur_assemble(int batch, int N, int nx, int nu, const double* As_next, const double* As,
                        const double* Bs, const double* Cs, const double* Qinv, const double* qvec,
                        const double* Rinv, const double* rvec, double* S, double* Phiinv,
                        double* gamma, void* workspace, size_t workspace_bytes, void* stream);
size_t dmpc_schur_workspace_size(int batch, int N, int nx);

/* project_matrix_onto_positive_semidefinite_cone (jax_utils.py:75-95), as SQPSolver.get_cost_terms
 * applies it to every cost Hessian with minimum_eigenvalue 1e-9 (sqp.py:191-196): for each of the
 * `batch` row-major n x n matrices (1 <= n <= 32) in device memory, out = V diag(max(lambda,
 * minimum_eigenvalue)) V^T of the symmetrized input (M + M^T) / 2 (jnp.linalg.eigh symmetrizes by
 * default), itself symmetrized.  FP64 Jacobi eigen-decomposition, one warp per matrix.  `out` may
 * equal `matrices`.  A matrix with a NaN or infinite entry gives all-NaN output.  The fused solver does not call it: its cost Hessians are diagonal, where the
 * projection is max(h_ii, 1e-9) exactly. */
int dmpc_psd_project(int batch, int n, const double* matrices, double minimum_eigenvalue, double* out,
                     void* stream);

/* solve_KKT_Schur on the dense S / Phiinv layout (pcg.py:350-445), FP64, with the
 * reference's stopping rule; then (x, u) from lambda (pcg.py:290-348).
 * lambda_guess (batch,K,nx) -> lambda, states (batch,K,nx), controls (batch,K,nu),
 * num_iterations (batch), convergence_eta (batch). */
int dmpc_pcg_solve(int batch, int N, int nx, int nu, const double* S, const double* Phiinv,
                   const double* gamma, const double* lambda_guess, const double* As_next,
                   const double* As, const double* Bs, const double* Qinv, const double* qvec,
                   const double* Rinv, const double* rvec, int max_iter, double tol_epsilon,
                   double* lambda, double* states, double* controls, int32_t* num_iterations,
                   double* convergence_eta, void* stream);

/* compute_gamma from premultiplied matrices (pcg.py:245-288): As_x_Qinv, Asnext_x_Qinvnext
 * (batch,N,nx,nx), Bs_x_Rinv (batch,N,nx,nu), Cs (batch,K,nx), Q0inv (batch,nx,nx),
 * qvec (batch,K,nx), rvec (batch,N,nu) -> gamma (batch,K,nx). */
int dmpc_compute_gamma(int batch, int N, int nx, int nu, const double* As_x_Qinv,
                       const double* Asnext_x_Qinvnext, const double* Bs_x_Rinv, const double* Cs,
                       const double* Q0inv, const double* qvec, const double* rvec, double* gamma,
                       void* stream);

/* The whole closed-loop rollout of every instance in ONE kernel launch (one CTA per
 * instance runs all T steps); see dmpc_rollout.  `group` is a single group: its
 * initial_state is x_0, and its states/controls/dual, convergence_error and histories hold
 * the initial guess (read, not written).  Per-step solutions and linearization points go to
 * the rollout's step arrays, so that the adjoint of step k is dmpc_solve_adj on a group
 * view pointing at them.  Same workspace as dmpc_solve_fwd for `group`. */
int dmpc_rollout_fwd(const dmpc_group* group, const dmpc_rollout* rollout, const dmpc_solver_params* params,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Gradient of the rollout of dmpc_rollout_fwd (jax.grad of the reference's scan), every step
 * of every instance in ONE launch: a reverse sweep over the steps that runs the adjoint of
 * each step's solve (dmpc_solve_adj, at the solution and linearization point the forward kept
 * in `rollout`) for the control cotangent that the simulator chain gives it.  `adj` selects
 * the parameter gradients as for dmpc_solve_adj; they are ACCUMULATED over the steps into
 * adj's g_* outputs, which the caller zeroes first.  adj's dl_dstates, dl_dcontrols,
 * dual_backward_guess, dual_backward, g_initial_state, adj_states, adj_controls and
 * num_pcg_iter are not used.  Same workspace as dmpc_solve_adj for `group`. */
int dmpc_rollout_adj(const dmpc_group* group, const dmpc_rollout* rollout, const dmpc_adjoint* adj,
                     const dmpc_rollout_adjoint* rollout_adjoint, const dmpc_solver_params* params,
                     void* workspace, size_t workspace_bytes, void* stream);

/* get_states_controls_from_kkt_multipliers (pcg.py:290-348), general dense matrices:
 * lambda (batch,K,nx) -> states (batch,K,nx), controls (batch,K,nu) with row N zero. */
int dmpc_kkt_recover(int batch, int N, int nx, int nu, const double* lambda, const double* As_next,
                     const double* As, const double* Bs, const double* Qinv, const double* qvec,
                     const double* Rinv, const double* rvec, double* states, double* controls,
                     void* stream);

/* Diagnostic: launches an FP32 FMA throughput probe (`blocks` x 256 threads, `iters`
 * rounds of 64 FMAs per thread) on `stream` and returns the FLOPs it issues, or -1.
 * Timing it with events gives the measured FP32 CUDA-core peak used as the roofline
 * denominator of the shared-memory-resident PCG.  `out` (device, >= blocks floats) is
 * written only to keep the computation live.  No reference counterpart. */
double dmpc_probe_fp32_fma(int blocks, int iters, float* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DMPC_H_ */
