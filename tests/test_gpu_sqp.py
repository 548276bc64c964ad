"""GPU parity of the fused SQP forward and adjoint kernels against the CPU oracle.

Tolerances: the all-FP64 path follows the reference's arithmetic and is held
to 1e-8 relative on states/controls/duals; the FP32-PCG + FP64-refinement path
is held to 1e-6 relative on controls and 1e-5 on gradients.  The mixed path is
compared at a tight PCG tolerance (1e-13): at the reference default 1e-9 the
FP64 solution itself moves by up to ~1e-5 relative when the tolerance is
tightened, so two correct solvers can only agree to that level there.
"""

import numpy as np
import pytest
import torch

from diffmpc_b200 import OptimalControlProblem, SQPSolver, workloads
from tests.oracle_util import oracle_forward, oracle_gradients, rel_err

pytestmark = pytest.mark.gpu

DEV = "cuda"


def gpu_solve(dyn, st, bt, sp, weights=None, guess=None):
    prog = OptimalControlProblem(dyn, st)
    solver = SQPSolver(prog, params=sp)
    p = workloads.to_device(bt, DEV)
    if guess is None:
        guess = solver.initial_guess(p)
    sol = solver.solve(guess, p, weights or {})
    torch.cuda.synchronize()
    return solver, sol


CASES = {
    "spacecraft_euler": lambda: _spacecraft(B=3, N=12),
    "quadrotor_rk4": lambda: workloads.quadrotor(B=3, N=12, seed=7),
    "attitude_euler": lambda: workloads.attitude(B=3, N=15, seed=8),
    "linear_lti": lambda: workloads.linear_lti(B=2, N=10, seed=9),
}


def _spacecraft(B, N, seed=3, scheme=0):
    from diffmpc_b200 import SpacecraftDynamics
    from diffmpc_b200.problem import load_problem_params

    rng = np.random.default_rng(seed)
    st = load_problem_params("spacecraft.yaml")
    st["horizon"] = N
    st["discretization_scheme"] = scheme
    K = N + 1
    st["reference_state_trajectory"] = torch.zeros(K, 3, dtype=torch.float64)
    st["reference_control_trajectory"] = torch.zeros(K, 3, dtype=torch.float64)
    st["inertia_vector"] = torch.tensor(1.0 + 9.0 * rng.random(3), dtype=torch.float64)
    bt = {}
    for k, v in st.items():
        bt[k] = v[None].expand(B, *v.shape).clone() if isinstance(v, torch.Tensor) else v
    bt["initial_state"] = torch.tensor(-0.1 + 0.2 * rng.random((B, 3)), dtype=torch.float64)
    from diffmpc_b200.problem import load_solver_params

    sp = load_solver_params("sqp.yaml")
    sp["pcg"]["tol_epsilon"] = 1e-14
    return SpacecraftDynamics(), st, bt, sp


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_forward_matches_oracle(case, precision):
    dyn, st, bt, sp = CASES[case]()
    sp["precision"] = precision
    if precision == "mixed":
        sp["pcg"]["tol_epsilon"] = min(sp["pcg"]["tol_epsilon"], 1e-13)
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    tol = 1e-8 if precision == "fp64" else 1e-6
    assert rel_err(sol.controls, osol.controls) < tol
    assert rel_err(sol.states, osol.states) < tol
    if precision == "fp64":
        # status / SQP iteration counts are decided by QP solutions whose differences sit at
        # the PCG truncation level; only the reference arithmetic reproduces them exactly
        assert torch.equal(sol.status.cpu().long(), osol.status)
        assert rel_err(sol.dual, osol.dual) < 1e-7
        assert torch.equal(sol.num_iter.cpu().long(), osol.num_iter)


@pytest.mark.parametrize("scheme", [0, 1, 2])
def test_integrators_spacecraft(scheme):
    dyn, st, bt, sp = _spacecraft(B=2, N=8, scheme=scheme)
    sp["precision"] = "fp64"
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_adjoint_quadrotor_matches_oracle(precision):
    """Gradients of sum(u_0^2) w.r.t. x0, w_x, w_u and mass (the headline workload's loss)."""
    dyn, st, bt, sp = workloads.quadrotor(B=2, N=10, seed=11)
    sp["precision"] = precision
    sp["pcg"]["tol_epsilon"] = 1e-14
    keys = ["initial_state", "weights_penalization_reference_state_trajectory",
            "weights_penalization_control_squared", "mass"]
    w = {k: bt[k].clone().to(DEV).requires_grad_(True) for k in keys}
    solver, sol = gpu_solve(dyn, st, bt, sp, weights=w)
    loss = (sol.controls[:, 0] ** 2).sum()
    loss.backward()
    osolver, osol = oracle_forward(dyn, st, bt, sp, weights={k: bt[k] for k in keys})
    dlu = torch.zeros_like(osol.controls)
    dlu[:, 0] = 2 * osol.controls[:, 0]
    og, _, _ = oracle_gradients(osolver, osol, bt, {k: bt[k] for k in keys}, torch.zeros_like(osol.states), dlu)
    tol = 1e-7 if precision == "fp64" else 1e-5
    for k in keys:
        assert rel_err(w[k].grad, og[k]) < tol, k


def test_adjoint_cost_keys_spacecraft():
    """w_f, final_state and reference trajectories gradients (closed-form mixed partials)."""
    dyn, st, bt, sp = _spacecraft(B=2, N=9)
    bt["weights_penalization_final_state"] = torch.full((2, 3), 0.5, dtype=torch.float64)
    bt["final_state"] = torch.tensor([[0.01, -0.02, 0.03]] * 2, dtype=torch.float64)
    sp["precision"] = "fp64"
    keys = ["weights_penalization_final_state", "final_state", "reference_state_trajectory", "inertia_vector"]
    w = {k: bt[k].clone().to(DEV).requires_grad_(True) for k in keys}
    _, sol = gpu_solve(dyn, st, bt, sp, weights=w)
    loss = sol.states.square().sum() + sol.controls.square().sum()
    loss.backward()
    osolver, osol = oracle_forward(dyn, st, bt, sp, weights={k: bt[k] for k in keys})
    og, _, _ = oracle_gradients(
        osolver, osol, bt, {k: bt[k] for k in keys}, 2 * osol.states, 2 * osol.controls
    )
    for k in keys:
        assert rel_err(w[k].grad, og[k]) < 1e-7, k


def test_ragged_horizons_match_per_instance_oracle():
    dyn, st, bt, sp = workloads.quadrotor(B=3, N=12, seed=5)
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = 1e-13
    hz = torch.tensor([12, 7, 10], dtype=torch.int32)
    p = dict(bt)
    p["horizons"] = hz
    _, sol = gpu_solve(dyn, st, p, sp)
    for i, n in enumerate(hz.tolist()):
        sti = dict(st)
        sti["horizon"] = n
        bti = workloads.subset(bt, slice(i, i + 1))
        bti["reference_state_trajectory"] = bti["reference_state_trajectory"][:, : n + 1]
        bti["reference_control_trajectory"] = bti["reference_control_trajectory"][:, : n + 1]
        _, osol = oracle_forward(dyn, sti, bti, sp)
        assert rel_err(sol.controls[i, : n + 1], osol.controls[0]) < 1e-6
        assert rel_err(sol.states[i, : n + 1], osol.states[0]) < 1e-6


def test_linesearch_matches_oracle():
    dyn, st, bt, sp = workloads.quadrotor(B=2, N=10, seed=13)
    sp["precision"] = "fp64"
    sp["linesearch"] = True
    sp["num_scp_iteration_max"] = 6
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert torch.allclose(sol.linesearch_alphas.cpu(), osol.linesearch_alphas)
    assert rel_err(sol.controls, osol.controls) < 1e-8


def test_warm_start_resolve_is_stable():
    """Re-solving from the converged solution keeps it (test_solver_pcg.py:179-227 on SQP level)."""
    dyn, st, bt, sp = _spacecraft(B=2, N=9)
    sp["precision"] = "mixed"
    solver, sol = gpu_solve(dyn, st, bt, sp)
    sol2 = solver.solve(sol, workloads.to_device(bt, DEV))
    assert rel_err(sol2.controls, sol.controls) < 1e-7
    assert int(sol2.num_iter.max()) <= int(sol.num_iter.max())


@pytest.mark.parametrize("case", ["quadrotor_rk4", "linear_lti"])
def test_solution_qp_matrices_match_oracle(case):
    """With return_qp_matrices the solution carries the last SQP iteration's QP data, as the
    reference's SQPSolution does (sqp.py:44-46): dmpc_linearize (A, B, C, Q^-1, q, R^-1, r at the
    saved linearization point), the premultiplied products and S, Phi^-1 (dmpc_schur_assemble).
    They match the oracle's compute_qp_parameters at the same point to FP64 rounding."""
    from tests.oracle_util import oracle_solver, tensor_params

    dyn, st, bt, sp = CASES[case]()
    sp["return_qp_matrices"] = True
    solver, sol = gpu_solve(dyn, st, bt, sp)
    assert sol.qp_parameters is not None and sol.schur_complement_matrices is not None
    os_ = oracle_solver(dyn, st, sp)
    x, u = sol.linearization_states.cpu(), sol.linearization_controls.cpu()
    qp, premult, schur = os_.compute_qp_parameters(x, u, tensor_params(bt))
    pairs = [
        (sol.qp_parameters.dynamics.As, qp.dynamics.As), (sol.qp_parameters.dynamics.Bs, qp.dynamics.Bs),
        (sol.qp_parameters.dynamics.Cs, qp.dynamics.Cs), (sol.qp_parameters.dynamics.As_next, qp.dynamics.As_next),
        (sol.qp_parameters.cost.Qinv, qp.cost.Qinv), (sol.qp_parameters.cost.qvec, qp.cost.qvec),
        (sol.qp_parameters.cost.Rinv, qp.cost.Rinv), (sol.qp_parameters.cost.rvec, qp.cost.rvec),
        (sol.dynamics_cost_premultiplied_matrices.As_x_Qinv, premult.As_x_Qinv),
        (sol.dynamics_cost_premultiplied_matrices.Asnext_x_Qinvnext, premult.Asnext_x_Qinvnext),
        (sol.dynamics_cost_premultiplied_matrices.Bs_x_Rinv, premult.Bs_x_Rinv),
        (sol.schur_complement_matrices.S, schur.S),
        (sol.schur_complement_matrices.preconditioner_Phiinv, schur.preconditioner_Phiinv),
    ]
    for i, (a, b) in enumerate(pairs):
        assert a.shape == b.shape, i
        # q = J - x^T H cancels to exact zeros in the oracle where the reference trajectory is
        # zero; relative to max(|b|, 1) the FP64 rounding left there is measured like elsewhere
        b = b.to(torch.float64)
        err = float((a.cpu() - b).abs().max() / max(float(b.abs().max()), 1.0))
        assert err < 1e-10, (i, err)
    # without the option the fields stay empty (no extra kernels on the solve path)
    sp["return_qp_matrices"] = False
    _, sol2 = gpu_solve(dyn, st, bt, sp)
    assert sol2.qp_parameters is None and sol2.schur_complement_matrices is None
