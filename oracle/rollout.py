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
from torch.func import vmap

from oracle.ocp import EULER, predict_next_state


def _stop(sol):
    return sol._replace(
        states=sol.states.detach(), controls=sol.controls.detach(), dual=sol.dual.detach(),
        dual_backward_guess=None if sol.dual_backward_guess is None else sol.dual_backward_guess.detach(),
    )


def _model_step(solver, problem_params, x, u, scheme=EULER):
    """One step of the solver's model with each instance's dt and parameters: Euler as in
    spacecraft/benchmark_diffmpc.py:87-89, or the program's own scheme (RL_quadrotor)."""
    model = solver.program.model
    p = {k: problem_params[k] for k in model.param_keys}
    dt = torch.as_tensor(problem_params["discretization_resolution"], dtype=torch.float64).reshape(-1)
    return vmap(lambda xx, uu, pp, h: predict_next_state(model, h, scheme, pp, xx, uu))(x, u, p, dt)


def rollout(solver, problem_params, initial_states, weights, A, Bm, b, num_steps, warm_start=True,
            through_state=False, simulator="linear", state_weight=1.0, control_weight=1.0, state_ref=0.0,
            control_ref=0.0, initial_guess=None):
    """Returns (running cost (B,), [u_k], [x_k]); differentiable w.r.t. ``weights``.
    ``simulator="euler"`` / ``"integrator"`` replace ``A x + B u + b`` by an Euler step / a step
    of the program's own integrator (A, Bm, b unused).  The cost is
    sum state_weight (x_{k+1} - state_ref)^2 + control_weight (u_k - control_ref)^2 (scalars or
    vectors); the spacecraft script's reward is -(10 |x|^2 + |u|^2), spacecraft/utils.py."""
    x = initial_states
    guess0 = initial_guess if initial_guess is not None else \
        solver.initial_guess({**problem_params, "initial_state": x.detach()})
    guess = guess0
    cost = torch.zeros(x.shape[0], dtype=torch.float64)
    us, xs = [], [x]
    for _ in range(num_steps):
        if through_state:
            sol = solver.solve(guess, problem_params, {**weights, "initial_state": x})
        else:
            sol = solver.solve(guess, {**problem_params, "initial_state": x.detach()}, weights)
        u = sol.controls[:, 0]
        if simulator in ("euler", "integrator"):
            # the model parameters as the solve sees them, not differentiated through the simulator
            scheme = EULER if simulator == "euler" else solver.program.scheme
            x_new = _model_step(solver, {**problem_params, **{k: v.detach() for k, v in weights.items()}}, x, u, scheme)
        else:
            x_new = torch.einsum("bij,bj->bi", A, x) + torch.einsum("bij,bj->bi", Bm, u) + b
        ws, wc = torch.as_tensor(state_weight, dtype=torch.float64), torch.as_tensor(control_weight, dtype=torch.float64)
        xr, ur = torch.as_tensor(state_ref, dtype=torch.float64), torch.as_tensor(control_ref, dtype=torch.float64)
        cost = cost + (ws * (x_new - xr) ** 2).sum(-1) + (wc * (u - ur) ** 2).sum(-1)
        guess = _stop(sol) if warm_start else guess0
        x = x_new
        us.append(u)
        xs.append(x)
    return cost, us, xs
