"""Test helpers: run the CPU oracle on the same seeded inputs as the GPU path."""

import torch

from oracle.models import make_model
from oracle.ocp import STATIC_KEYS, OptimalControlProblem
from oracle.sqp import SQPSolver


def oracle_solver(dyn, static_params, solver_params):
    model = make_model(dyn.model_name, dyn.num_states, dyn.num_controls)
    prog = OptimalControlProblem(model, static_params)
    return SQPSolver(prog, params=solver_params)


def tensor_params(batched):
    return {k: v for k, v in batched.items() if k not in STATIC_KEYS}


def oracle_forward(dyn, static_params, batched, solver_params, weights=None, guess=None):
    s = oracle_solver(dyn, static_params, solver_params)
    tp = tensor_params(batched)
    if guess is None:
        guess = s.initial_guess(tp)
    sol = s._solve(guess, batched, weights or {})
    return s, sol


def oracle_gradients(solver, sol, batched, weights, dl_dstates, dl_dcontrols, dual_backward_guess=None):
    if dual_backward_guess is None:
        dual_backward_guess = torch.zeros_like(sol.dual)
    return solver.solve_bwd(sol, weights, batched, dl_dstates, dl_dcontrols, dual_backward_guess)


def rel_err(a, b):
    a = torch.as_tensor(a, dtype=torch.float64).cpu()
    b = torch.as_tensor(b, dtype=torch.float64).cpu()
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))
