"""Closed-loop rollout restatement (oracle: test infrastructure only, float64 CPU).

Follows benchmarking/reinforcement-learning/benchmark_diffmpc.py:140-175: ``rollout_step``
scanned over ``num_steps`` steps for a batch of initial states (the reference vmaps the
scan; here the oracle solver is batched).  Step k solves the MPC with initial state x_k,
starting from step k-1's solution (``warm_start``, the carry is ``stop_gradient``-ed) or
from the initial guess, applies u_k = controls[0], simulates
``x_{k+1} = A x_k + B u_k + b`` (:148-150) and adds ``|x_{k+1}|^2 + |u_k|^2`` (the negated
``reward``, :35-37).  The gradient is torch autograd through the oracle's custom-VJP solve,
as ``jax.grad`` runs through the reference's: the solve's problem parameters, x_k among
them, carry no cotangent (sqp.py:781-795).  ``through_state=True`` passes x_k as a weight
instead, which differentiates through the solve's dependence on it.
"""

import torch


def _stop(sol):
    return sol._replace(
        states=sol.states.detach(), controls=sol.controls.detach(), dual=sol.dual.detach(),
        dual_backward_guess=None if sol.dual_backward_guess is None else sol.dual_backward_guess.detach(),
    )


def rollout(solver, problem_params, initial_states, weights, A, Bm, b, num_steps, warm_start=True,
            through_state=False):
    """Returns (running cost (B,), [u_k], [x_k]); differentiable w.r.t. ``weights``."""
    x = initial_states
    guess0 = solver.initial_guess({**problem_params, "initial_state": x.detach()})
    guess = guess0
    cost = torch.zeros(x.shape[0], dtype=torch.float64)
    us, xs = [], [x]
    for _ in range(num_steps):
        if through_state:
            sol = solver.solve(guess, problem_params, {**weights, "initial_state": x})
        else:
            sol = solver.solve(guess, {**problem_params, "initial_state": x.detach()}, weights)
        u = sol.controls[:, 0]
        x_new = torch.einsum("bij,bj->bi", A, x) + torch.einsum("bij,bj->bi", Bm, u) + b
        cost = cost + (x_new ** 2).sum(-1) + (u ** 2).sum(-1)
        guess = _stop(sol) if warm_start else guess0
        x = x_new
        us.append(u)
        xs.append(x)
    return cost, us, xs
