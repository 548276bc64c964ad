"""GPU parity at the benchmark configurations' exact shapes, against the CPU oracle.

- linear LTI, nx=6, nu=3, N=20, batch 1, FP64, PCG tolerance 1e-10: the first QP solve reaches the
  solution and the second measures a step at the PCG truncation level (about 5e-6, above the 1e-8
  convergence tolerance, so the status is the same ERROR the oracle reports after its 2 iterations);
- spacecraft attitude, nx=7, nu=3, N=50, 10 SQP iterations, mixed precision;
- quadrotor, nx=13, nu=4, N=60, RK4, forward + adjoint of sum u_0^2 w.r.t. x0, log-weights and
  mass, mixed precision at the headline's PCG tolerance 1e-20 (row PCG, 256-thread CTA);
- the l1-merit line search with the FP32 PCG;
- ill-conditioned QPs (state weights over 1e-6..1e6) on both FP32 PCGs: stall detection and hand-over.

Bars: FP64 1e-8 relative on controls and states; mixed precision 1e-6 on controls and 1e-5 on
gradients (the headline's parity bars).
"""

import pytest
import torch

from diffmpc_b200 import workloads
from tests.oracle_util import oracle_forward, oracle_gradients, rel_err
from tests.test_gpu_sqp import DEV, gpu_solve

pytestmark = pytest.mark.gpu


def test_linear_n20_batch1_converges_in_one_sqp_iteration():
    dyn, st, bt, sp = workloads.linear_lti(B=1, N=20, seed=1000)
    sp["precision"] = "fp64"
    assert sp["pcg"]["tol_epsilon"] == 1e-10 and sp["num_scp_iteration_max"] == 2
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-8
    assert rel_err(sol.states, osol.states) < 1e-8
    assert int(sol.status[0]) == int(osol.status[0])
    assert int(sol.num_iter[0]) == int(osol.num_iter[0]) == 2
    ce, oce = sol.convergence_errors.cpu()[0], osol.convergence_errors[0]
    assert abs(float(ce[0] - oce[0])) <= 1e-8 * float(oce[0])
    # the second step is PCG truncation: both far below the first
    assert float(ce[1]) < 1e-4 and float(oce[1]) < 1e-4


def test_attitude_n50_mixed_matches_oracle():
    dyn, st, bt, sp = workloads.attitude(B=2, N=50, seed=1001)
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = 1e-18
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-6
    assert rel_err(sol.states, osol.states) < 1e-6


def test_quadrotor_n60_forward_and_adjoint_mixed_matches_oracle():
    dyn, st, bt, sp = workloads.quadrotor(B=2, N=60, seed=1002)
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = 1e-20
    keys = ["initial_state", "weights_penalization_reference_state_trajectory",
            "weights_penalization_control_squared", "mass"]
    w = {k: bt[k].clone().to(DEV).requires_grad_(True) for k in keys}
    solver, sol = gpu_solve(dyn, st, bt, sp, weights=w)
    (sol.controls[:, 0] ** 2).sum().backward()
    osolver, osol = oracle_forward(dyn, st, bt, sp, weights={k: bt[k] for k in keys})
    assert rel_err(sol.controls, osol.controls) < 1e-6
    dlu = torch.zeros_like(osol.controls)
    dlu[:, 0] = 2 * osol.controls[:, 0]
    og, _, _ = oracle_gradients(osolver, osol, bt, {k: bt[k] for k in keys}, torch.zeros_like(osol.states), dlu)
    for k in keys:
        assert rel_err(w[k].grad, og[k]) < 1e-5, k


def test_linesearch_mixed_matches_oracle():
    dyn, st, bt, sp = workloads.quadrotor(B=2, N=10, seed=13)
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = 1e-20
    sp["linesearch"] = True
    sp["num_scp_iteration_max"] = 6
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    # the alphas are discrete choices: equal when the candidates' merit values are resolved
    assert torch.allclose(sol.linesearch_alphas.cpu(), osol.linesearch_alphas)
    assert rel_err(sol.controls, osol.controls) < 1e-6


@pytest.mark.parametrize("nx", [5, 6])
def test_ill_conditioned_qps_hand_over_to_fp64_and_match_oracle(nx):
    """State weights over 1e-6..1e6 (cond(S) 1e7..1e9): the FP32 recursion stalls on most of these
    QPs.  The stall detection (a segment cut after max(2 x the previous one, 200) iterations, then
    the stagnation rule) hands them to the FP64 recurrence after a few hundred FP32 iterations;
    without it a stalled QP runs half the 10000-iteration budget in FP32 before the FP64 finish, so
    a count below 5000 shows the hand-over.  nx=6 takes the compile-time row PCG, nx=5 the generic
    one.  PCG tolerance 1e-20: at 1e-16 the stopping test on these systems admits control errors
    of about 1e-5 (two solves that both pass it differ by that much), at 1e-20 about 1e-7."""
    dyn, st, bt, sp = workloads.linear_lti(B=3, N=40, nx=nx, nu=3, seed=1003, log10_wx=6.0)
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = 1e-20
    solver, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-6
    assert rel_err(sol.states, osol.states) < 1e-6
    its = sol.num_pcg_iters.cpu()
    assert int(its.max()) < sp["pcg"]["max_iter"] // 2, its
    # the precision record shows the hand-over: FP64 iterations in the first QP of most instances,
    # after at least one FP64 residual replacement
    rec = solver.last_forward_pcg_record.cpu()
    assert int((rec[1, :, 0] > 0).sum()) >= 2, rec
    assert bool((rec[0, :, 0] >= 1).all()), rec
    assert bool((rec[1] <= its).all())
    # the FP64 path records every iteration as FP64 and no replacement
    sp["precision"] = "fp64"
    solver64, sol64 = gpu_solve(dyn, st, bt, sp)
    rec64 = solver64.last_forward_pcg_record.cpu()
    assert torch.equal(rec64[1], sol64.num_pcg_iters.cpu()) and int(rec64[0].abs().sum()) == 0
