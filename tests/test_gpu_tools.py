"""CUDA-graph replay of the forward solve and the launch-shape autotuner."""

import pytest
import torch

from diffmpc_b200 import OptimalControlProblem, SQPSolver, workloads
from diffmpc_b200.autotune import tune
from diffmpc_b200.graph import GraphedForward
from tests.oracle_util import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _setup(B=4, N=12, seed=51):
    dyn, st, bt, sp = workloads.quadrotor(B=B, N=N, seed=seed)
    sp["pcg"]["tol_epsilon"] = 1e-12
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    return solver, workloads.to_device(bt, DEV)


def test_graph_replay_equals_eager_for_new_initial_states():
    solver, p = _setup()
    g = GraphedForward(solver, solver.initial_guess(p), p)
    for shift in (0.0, 0.05):
        x0 = p["initial_state"] + shift
        q = dict(p)
        q["initial_state"] = x0
        eager = solver.solve(solver.initial_guess(p), q)
        out = g(initial_state=x0)
        torch.cuda.synchronize()
        assert torch.equal(out.controls, eager.controls)
        assert torch.equal(out.states, eager.states)
        assert torch.equal(out.num_iter, eager.num_iter)


def test_autotune_picks_a_valid_cta_size_and_keeps_results():
    solver, p = _setup(B=16, N=10, seed=52)
    ref = solver.solve(solver.initial_guess(p), p)
    best = tune(solver, p, sample=16, repeats=1, use_cache=False, cands=[0, 128, 256])
    assert best in (0, 128, 256)
    assert solver.params["threads_per_block"] == best
    out = solver.solve(solver.initial_guess(p), p)
    torch.cuda.synchronize()
    assert rel_err(out.controls, ref.controls) < 1e-9
