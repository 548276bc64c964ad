"""The oracle's closed-loop rollout (oracle/rollout.py) and its gradient, on the CPU.

* through_state=True: the gradient of the running cost w.r.t. the cost weights equals
  central finite differences of the rollout.
* through_state=False (the reference's semantics: a solve's problem parameters, its
  initial state among them, carry no cotangent): the gradient equals central finite
  differences of the rollout in which every solve keeps the initial state of the
  unperturbed trajectory while the simulator and the cost see the perturbed one.
"""


import pytest
import torch

from diffmpc_b200 import workloads
from oracle.rollout import _model_step, rollout
from tests.oracle_util import oracle_solver, tensor_params

KEY = "weights_penalization_reference_state_trajectory"


def _setup(warm):
    dyn, st, bt, sp, (A, Bm, b) = workloads.rl_linear(B=2, seed=7, nx=4, nu=2, N=6, warm_start=warm)
    solver = oracle_solver(dyn, st, sp)
    p = tensor_params(bt)
    B = p["initial_state"].shape[0]
    sim = (A.expand(B, 4, 4), Bm.expand(B, 4, 2), b.expand(B, 4))
    return solver, p, sim


def _frozen_rollout(solver, p, x0, w, sim, T, warm, xs_nominal, model_sim=False, ws=1.0):
    """Rollout whose k-th solve starts from xs_nominal[k] (no state feedback into the MPC)."""
    A, Bm, b = sim if sim is not None else (None, None, None)
    guess0 = solver.initial_guess({**p, "initial_state": x0})
    guess, x, cost = guess0, x0, torch.zeros(x0.shape[0], dtype=torch.float64)
    for k in range(T):
        sol = solver._solve(guess, {**p, "initial_state": xs_nominal[k]}, w)
        u = sol.controls[:, 0]
        if model_sim:
            x = _model_step(solver, p, x, u)
        else:
            x = torch.einsum("bij,bj->bi", A, x) + torch.einsum("bij,bj->bi", Bm, u) + b
        cost = cost + ws * (x ** 2).sum(-1) + (u ** 2).sum(-1)
        guess = sol if warm else guess0
    return cost


@pytest.mark.parametrize("warm", [True, False])
@pytest.mark.parametrize("through_state", [True, False])
def test_oracle_rollout_gradient_matches_finite_differences(warm, through_state):
    solver, p, sim = _setup(warm)
    T = 3
    w = p[KEY].clone().requires_grad_(True)
    x0 = p["initial_state"]
    cost, us, xs = rollout(solver, p, x0, {KEY: w}, *sim, T, warm_start=warm, through_state=through_state)
    (g,) = torch.autograd.grad(cost.sum(), w)
    xs_nominal = [x.detach() for x in xs]
    h = 1e-6
    for (bi, j) in [(0, 0), (1, 2), (0, 3)]:
        wp, wm = p[KEY].clone(), p[KEY].clone()
        wp[bi, j] += h
        wm[bi, j] -= h
        if through_state:
            fp = rollout(solver, p, x0, {KEY: wp}, *sim, T, warm_start=warm)[0].sum()
            fm = rollout(solver, p, x0, {KEY: wm}, *sim, T, warm_start=warm)[0].sum()
        else:
            fp = _frozen_rollout(solver, p, x0, {KEY: wp}, sim, T, warm, xs_nominal).sum()
            fm = _frozen_rollout(solver, p, x0, {KEY: wm}, sim, T, warm, xs_nominal).sum()
        fd = float((fp - fm) / (2 * h))
        assert abs(float(g[bi, j]) - fd) <= 1e-5 * max(1.0, abs(fd)), (bi, j, float(g[bi, j]), fd)


@pytest.mark.parametrize("through_state", [True, False])
def test_oracle_model_simulator_rollout_gradient_matches_finite_differences(through_state):
    """Spacecraft, the model's own Euler step as the simulator and cost 10 |x|^2 + |u|^2."""
    dyn, st, bt, sp = workloads.rl_spacecraft(B=2, seed=9, N=8)
    solver = oracle_solver(dyn, st, sp)
    p = tensor_params(bt)
    T = 3
    keys = ["weights_penalization_control_squared", KEY]
    w = {k: p[k].clone().requires_grad_(True) for k in keys}
    x0 = p["initial_state"]
    kw = dict(warm_start=True, simulator="euler", state_weight=10.0)
    cost, _, xs = rollout(solver, p, x0, w, None, None, None, T, through_state=through_state, **kw)
    grads = torch.autograd.grad(cost.sum(), [w[k] for k in keys])
    xs_nominal = [x.detach() for x in xs]
    h = 1e-6
    for ki, key in enumerate(keys):
        for (bi, j) in [(0, 0), (1, 2)]:
            vals = []
            for sgn in (1.0, -1.0):
                wq = {k: p[k].clone() for k in keys}
                wq[key][bi, j] += sgn * h
                if through_state:
                    vals.append(rollout(solver, p, x0, wq, None, None, None, T, **kw)[0].sum())
                else:
                    vals.append(_frozen_rollout(solver, p, x0, wq, None, T, True, xs_nominal, model_sim=True,
                                                ws=10.0).sum())
            fd = float((vals[0] - vals[1]) / (2 * h))
            g = float(grads[ki][bi, j])
            assert abs(g - fd) <= 1e-5 * max(1.0, abs(fd)), (key, bi, j, g, fd)
