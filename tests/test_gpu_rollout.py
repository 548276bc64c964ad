"""Fused closed-loop rollout (dmpc_rollout_fwd forward, dmpc_rollout_adj reverse sweep).

* Every step of the one-launch rollout equals the same step run as a separate
  SQPSolver.solve call from the host (same kernels, same guess chain), and the
  one-launch backward sweep equals the sweep run as one adjoint launch per step.
* Running cost, per-step controls and gradients w.r.t. cost weights and the simulator's
  model matrix match the oracle's rollout (oracle/rollout.py), whose gradient is pinned
  to finite differences on the CPU: FP64 to 1e-9 / 1e-7, mixed precision at PCG tolerance
  1e-13 to 1e-6 / 1e-5.
"""

import pytest
import torch

from diffmpc_b200 import OptimalControlProblem, SQPSolver, workloads
from diffmpc_b200.rollout import ClosedLoopRollout
from oracle.rollout import rollout as oracle_rollout
from tests.oracle_util import oracle_solver, rel_err, tensor_params

pytestmark = pytest.mark.gpu
DEV = "cuda"
KW = "weights_penalization_reference_state_trajectory"
KU = "weights_penalization_control_squared"


def _setup(precision, warm, B=3, N=12, seed=11):
    dyn, st, bt, sp, (A, Bm, b) = workloads.rl_linear(B=B, seed=seed, nx=8, nu=4, N=N, warm_start=warm)
    sp["precision"] = precision
    sp["pcg"]["tol_epsilon"] = 1e-13
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    return dyn, st, bt, sp, (A, Bm, b), solver, workloads.to_device(bt, DEV)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("warm", [True, False])
def test_fused_rollout_steps_equal_host_loop_of_solves(precision, warm):
    dyn, st, bt, sp, (A, Bm, b), solver, p = _setup(precision, warm)
    T = 4
    roll = ClosedLoopRollout(solver, A.to(DEV), Bm.to(DEV), b.to(DEV), T, warm_start=warm)
    cost = roll(p["initial_state"], p)
    torch.cuda.synchronize()
    guess0 = solver.initial_guess(p)
    guess, x = guess0, p["initial_state"]
    c = torch.zeros_like(cost)
    Ad, Bd, bd = A.to(DEV), Bm.to(DEV), b.to(DEV)
    tol = 1e-10 if precision == "fp64" else 1e-5
    for k in range(T):
        q = dict(p)
        q["initial_state"] = x
        sol = solver.solve(guess, q)
        assert rel_err(roll.last.controls[k], sol.controls) < tol, k
        assert rel_err(roll.last.x[k], x) < tol, k
        u = sol.controls[:, 0]
        x = x @ Ad.T + u @ Bd.T + bd
        c = c + (x ** 2).sum(-1) + (u ** 2).sum(-1)
        guess = sol if warm else guess0
    assert rel_err(cost, c) < tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("warm,through_state", [(True, False), (False, False), (True, True)])
def test_rollout_cost_and_gradients_match_oracle(precision, warm, through_state):
    dyn, st, bt, sp, (A, Bm, b), solver, p = _setup(precision, warm)
    T = 3
    wkeys = [KW, KU] + (["A"] if precision == "fp64" else [])
    w = {k: p[k].clone().requires_grad_(True) for k in wkeys}
    roll = ClosedLoopRollout(solver, A.to(DEV), Bm.to(DEV), b.to(DEV), T, warm_start=warm,
                             through_state=through_state)
    cost = roll(p["initial_state"], p, w)
    cost.sum().backward()
    torch.cuda.synchronize()

    osolver = oracle_solver(dyn, st, sp)
    op = tensor_params(bt)
    ow = {k: op[k].clone().requires_grad_(True) for k in wkeys}
    B = op["initial_state"].shape[0]
    ocost, ous, _ = oracle_rollout(osolver, op, op["initial_state"], ow, A.expand(B, 8, 8), Bm.expand(B, 8, 4),
                                   b.expand(B, 8), T, warm_start=warm, through_state=through_state)
    ocost.sum().backward()
    ctol, gtol = (1e-9, 1e-7) if precision == "fp64" else (1e-6, 1e-5)
    assert rel_err(cost, ocost) < ctol
    for k in range(T):
        assert rel_err(roll.last.controls[k][:, 0], ous[k]) < ctol, k
    for k in wkeys:
        assert rel_err(w[k].grad, ow[k].grad) < gtol, k


@pytest.mark.parametrize("through_state", [False, True])
def test_fused_backward_equals_per_step_adjoint_sweep(through_state):
    """dmpc_rollout_adj (one launch) against the same sweep as one dmpc_solve_adj per step."""
    dyn, st, bt, sp, (A, Bm, b), solver, p = _setup("fp64", True, B=4)
    grads = []
    for fused in (True, False):
        w = {KW: p[KW].clone().requires_grad_(True), "A": p["A"].clone().requires_grad_(True)}
        x0 = p["initial_state"].clone().requires_grad_(True)
        roll = ClosedLoopRollout(solver, A.to(DEV), Bm.to(DEV), b.to(DEV), 4, through_state=through_state,
                                 fused_backward=fused)
        (roll(x0, p, w) * torch.arange(1, 5, device=DEV)).sum().backward()
        grads.append((w[KW].grad, w["A"].grad, x0.grad))
    for a, c in zip(*grads):
        assert rel_err(a, c) < 1e-12


def test_reference_benchmark_configuration_matches_oracle():
    """The reference's closed-loop benchmark configuration (nx=8, nu=4, 40 knots, one SQP
    iteration with the line search at alpha = 1, PCG 1e-12, warm start), five steps."""
    dyn, st, bt, sp, (A, Bm, b) = workloads.rl_linear(B=2, seed=5, N=39, warm_start=True)
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    p = workloads.to_device(bt, DEV)
    w = {KW: p[KW].clone().requires_grad_(True)}
    roll = ClosedLoopRollout(solver, A.to(DEV), Bm.to(DEV), b.to(DEV), 5, warm_start=True)
    cost = roll(p["initial_state"], p, w)
    cost.sum().backward()
    osolver = oracle_solver(dyn, st, sp)
    op = tensor_params(bt)
    ow = {KW: op[KW].clone().requires_grad_(True)}
    ocost, _, _ = oracle_rollout(osolver, op, op["initial_state"], ow, A.expand(2, 8, 8), Bm.expand(2, 8, 4),
                                 b.expand(2, 8), 5, warm_start=True)
    ocost.sum().backward()
    # mixed precision (the solver default) at the benchmark's PCG tolerance 1e-12
    assert rel_err(cost, ocost) < 1e-6
    assert rel_err(w[KW].grad, ow[KW].grad) < 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("through_state", [False, True])
def test_model_simulator_rollout_matches_oracle(precision, through_state):
    """Spacecraft with its own Euler step as the simulator and cost 10 |x|^2 + |u|^2
    (spacecraft/benchmark_diffmpc.py:68-96)."""
    dyn, st, bt, sp = workloads.rl_spacecraft(B=3, seed=13, N=20)
    sp["precision"] = precision
    # the spacecraft's states and controls are ~1e-2 and its weight gradients ~1e-4, so the
    # absolute PCG tolerance must be tighter for the same relative accuracy: against eps = 1e-24
    # the oracle's own controls move by 1.6e-6 at eps = 1e-13, and its w_x gradient by 9e-4 at
    # 1e-13, 1.8e-5 at 1e-16 and 3e-7 at 1e-20
    sp["pcg"]["tol_epsilon"] = 1e-20
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    p = workloads.to_device(bt, DEV)
    T = 4
    wkeys = [KW, KU]
    w = {k: p[k].clone().requires_grad_(True) for k in wkeys}
    roll = ClosedLoopRollout(solver, num_sim_steps=T, simulator="euler", state_weight=10.0,
                             through_state=through_state)
    cost = roll(p["initial_state"], p, w)
    cost.sum().backward()
    osolver = oracle_solver(dyn, st, sp)
    op = tensor_params(bt)
    ow = {k: op[k].clone().requires_grad_(True) for k in wkeys}
    ocost, ous, _ = oracle_rollout(osolver, op, op["initial_state"], ow, None, None, None, T, warm_start=True,
                                   through_state=through_state, simulator="euler", state_weight=10.0)
    ocost.sum().backward()
    ctol, gtol = (1e-9, 1e-7) if precision == "fp64" else (1e-6, 1e-5)
    assert rel_err(cost, ocost) < ctol
    for k in range(T):
        assert rel_err(roll.last.controls[k][:, 0], ous[k]) < ctol, k
    for k in wkeys:
        assert rel_err(w[k].grad, ow[k].grad) < gtol, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rl_spacecraft_notebook_rollout_on_gpu(precision):
    """notebooks/RL_spacecraft.ipynb cells 5-14 as one fused rollout: 2 spacecraft, 40 knots, 20
    steps of the model's Euler step, reward -(10 |x|^2 + |u|^2), the shared weights updated once
    with learning rate 1.  The recorded loss is -2.8196995973193135; the printed weights agree to
    the adjoint's stopping tolerance (the oracle pin gives the same bound)."""
    import numpy as np

    from diffmpc_b200 import SpacecraftDynamics
    from tests.test_oracle_pins import STATIC, _batched, _spacecraft_params

    np.random.seed(0)
    inertia = 1.0 + np.random.rand(3) * 9.0
    x0s = -0.1 + np.random.rand(2, 3) * 0.2
    p = _spacecraft_params(39)
    p["inertia_vector"] = inertia
    st = {k: (torch.as_tensor(np.asarray(v), dtype=torch.float64) if k not in STATIC else v) for k, v in p.items()}
    from diffmpc_b200 import load_solver_params

    sp = load_solver_params("sqp.yaml")
    sp.update(num_scp_iteration_max=1, linesearch=True, linesearch_alphas=[1.0], precision=precision)
    sp["pcg"]["tol_epsilon"] = 1e-12
    solver = SQPSolver(OptimalControlProblem(SpacecraftDynamics(), st), params=sp)
    bp = {k: v.to(DEV) for k, v in _batched(p, 2).items()}
    keys = [KW, KU]
    w = {k: torch.tensor(p[k], dtype=torch.float64, device=DEV, requires_grad=True) for k in keys}
    roll = ClosedLoopRollout(solver, num_sim_steps=20, simulator="euler", state_weight=10.0)
    cost = roll(torch.tensor(x0s, device=DEV), bp, w)
    loss = -cost.sum()
    loss.backward()
    want = -2.8196995973193135
    assert abs(float(loss) - want) < (1e-10 if precision == "fp64" else 1e-6) * abs(want)
    new_u = torch.clamp(w[KU] + w[KU].grad, min=1e-10).detach().cpu().numpy()
    new_x = torch.clamp(w[KW] + w[KW].grad, min=1e-10).detach().cpu().numpy()
    assert np.allclose(new_u, [0.9955808, 0.9085766, 0.8319815], atol=5e-5)
    assert np.allclose(new_x, [1.0033015, 1.09093417, 1.16958629], atol=5e-5)


def test_rl_quadrotor_notebook_rollout_on_gpu():
    """notebooks/RL_quadrotor.ipynb cell 12 as one fused rollout (FP64): one quadrotor, 20 knots,
    RK4, 10 steps of the model's own integrator, <= 50 SQP iterations with the line search,
    reward -(|p - p_ref|^2 + 0.1 |u - u_ref|^2).  The recorded loss is -241.93737859418738.
    Every solve stops at the SQP cap unconverged and a 1e-14 relative change of x0 moves the
    loss by ~8e-4 relative, so the loss is held to 2e-3 (the oracle pin's bound)."""
    import numpy as np

    from diffmpc_b200 import QuadrotorDynamics, load_solver_params
    from tests.test_oracle_pins import STATIC, _batched

    np.random.seed(0)
    x0 = np.array([0.0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0])[None].repeat(1, 0)
    x0[:, :3] = -4 + np.random.rand(1, 3) * 8
    x0[:, 3:6] = -0.1 + np.random.rand(1, 3) * 0.2
    delta = 0.5 * np.random.randn(4)
    q = np.array([1, 0, 0, 0]) + delta / np.linalg.norm(delta)
    x0[:, 6:10] = q / np.linalg.norm(q)
    N = 19
    xref = np.array([0.0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0])
    uref = np.array([0.981, 0, 0, 0])
    p = dict(
        horizon=N, discretization_resolution=0.03, discretization_scheme=2, initial_state=x0[0],
        final_state=xref, reference_state_trajectory=np.repeat(xref[None], N + 1, 0),
        reference_control_trajectory=np.repeat(uref[None], N + 1, 0), penalize_control_reference=True,
        weights_penalization_reference_state_trajectory=[1e-4] * 3 + [1e-1] * 3 + [1e-4] * 4 + [1e-1] * 3,
        weights_penalization_final_state=[1e5] * 3 + [1e3] * 10,
        weights_penalization_control_squared=[10, 0.1, 0.1, 0.1],
        mass=np.array([0.1]), inertia=np.array([0.1, 0.01, 0.01, 0.01, 0.1, 0.01, 0.01, 0.01, 0.1]),
    )
    st = {k: (torch.as_tensor(np.asarray(v), dtype=torch.float64) if k not in STATIC else v) for k, v in p.items()}
    sp = load_solver_params("sqp.yaml")
    sp.update(num_scp_iteration_max=50, linesearch=True, precision="fp64")
    sp["pcg"]["tol_epsilon"] = 1e-12
    solver = SQPSolver(OptimalControlProblem(QuadrotorDynamics(), st), params=sp)
    bp = {k: v.to(DEV) for k, v in _batched(p, 1).items()}
    g = solver.initial_guess(bp)
    sts = g.states.clone()
    sts[:, :, 6:10] = sts[:, :, 6:10] / torch.linalg.norm(sts[:, :, 6:10], dim=-1, keepdim=True)
    ctl = torch.tensor([[1.0, 0, 0, 0]], dtype=torch.float64, device=DEV).expand(1, N + 1, 4).clone()
    g = g._replace(states=sts, controls=ctl)
    roll = ClosedLoopRollout(solver, num_sim_steps=10, simulator="integrator",
                             state_weight=[1.0] * 3 + [0.0] * 10, control_weight=0.1,
                             state_ref=xref, control_ref=uref)
    loss = -float(roll(torch.tensor(x0, device=DEV), bp, {}, initial_guess=g).sum())
    want = -241.93737859418738
    assert abs(loss - want) < 2e-3 * abs(want), loss


def test_rollout_in_the_two_cta_configuration_matches_oracle():
    """The fused rollout's forward and reverse sweeps in the two-CTA configuration (the row PCG
    with one register copy of each scaled block, nx=8: two threads per knot), against the oracle's
    rollout at the mixed-precision bars."""
    dyn, st, bt, sp, (A, Bm, b), _, p = _setup("mixed", True)
    sp["cta_config"] = 3  # DMPC_CTA_DUAL
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    T = 3
    w = {k: p[k].clone().requires_grad_(True) for k in (KW, KU)}
    roll = ClosedLoopRollout(solver, A.to(DEV), Bm.to(DEV), b.to(DEV), T, warm_start=True)
    cost = roll(p["initial_state"], p, w)
    cost.sum().backward()
    torch.cuda.synchronize()
    osolver = oracle_solver(dyn, st, sp)
    op = tensor_params(bt)
    ow = {k: op[k].clone().requires_grad_(True) for k in (KW, KU)}
    B = op["initial_state"].shape[0]
    ocost, ous, _ = oracle_rollout(osolver, op, op["initial_state"], ow, A.expand(B, 8, 8), Bm.expand(B, 8, 4),
                                   b.expand(B, 8), T, warm_start=True)
    ocost.sum().backward()
    assert rel_err(cost, ocost) < 1e-6
    for k in range(T):
        assert rel_err(roll.last.controls[k][:, 0], ous[k]) < 1e-6, k
    for k in (KW, KU):
        assert rel_err(w[k].grad, ow[k].grad) < 1e-5, k
