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


def _ragged_groups(B=6, N=24, seed=61):
    import numpy as np

    rng = np.random.default_rng(seed)
    groups = []
    for which in ("linear", "quadrotor"):
        if which == "linear":
            dyn, st, bt, sp = workloads.linear_lti(B=B, nx=12, nu=4, N=N, seed=seed)
        else:
            dyn, st, bt, sp = workloads.quadrotor(B=B, N=N, seed=seed + 1)
        sp["pcg"]["tol_epsilon"] = 1e-13
        sp["num_scp_iteration_max"] = 6
        solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
        p = workloads.to_device(bt, DEV)
        p["horizons"] = torch.tensor(rng.integers(N // 2, N + 1, size=B), dtype=torch.int32, device=DEV)
        groups.append((solver, p))
    return groups


def test_captured_groups_step_replays_bit_equal():
    """Forward + adjoint of two ragged groups (one launch per direction) captured as one graph:
    replays equal the eager step bit for bit, also after the inputs change in place."""
    from diffmpc_b200.batch import solve_groups
    from diffmpc_b200.graph import CapturedStep

    groups = _ragged_groups()

    def step():
        probs, ws = [], []
        for solver, p in groups:
            w = p["initial_state"].clone().requires_grad_(True)
            ws.append(w)
            probs.append((solver, solver.initial_guess(p), p, {"initial_state": w}))
        sols = solve_groups(probs)
        loss = sum((s.controls[:, 0] ** 2).sum() for s in sols)
        grads = torch.autograd.grad(loss, ws)
        return [s.controls for s in sols] + list(grads)

    cap = CapturedStep(step)
    first = None
    for shift in (0.0, 0.02):
        for _, p in groups:
            p["initial_state"].add_(shift)
        out = [t.clone() for t in cap.replay()]
        ref = step()
        torch.cuda.synchronize()
        for a, b in zip(out, ref):
            assert torch.equal(a, b)
        if first is None:
            first = out
    assert not torch.equal(first[0], out[0]) and not torch.equal(first[-1], out[-1])


def test_captured_rollout_step_replays_bit_equal():
    """A 10-step closed-loop rollout, forward and backward (two fused launches), as one graph."""
    from diffmpc_b200.graph import CapturedStep
    from diffmpc_b200.rollout import ClosedLoopRollout

    dyn, st, bt, sp, (A, Bm, b) = workloads.rl_linear(B=8)
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    p = workloads.to_device(bt, DEV)
    roll = ClosedLoopRollout(solver, A.to(DEV), Bm.to(DEV), b.to(DEV), 10, warm_start=True)
    key = "weights_penalization_reference_state_trajectory"

    def step():
        w = p[key].clone().requires_grad_(True)
        c = roll(p["initial_state"], p, {key: w})
        (g,) = torch.autograd.grad(c.sum(), [w])
        return c, g

    cap = CapturedStep(step)
    first = None
    for shift in (0.0, 0.05):
        p["initial_state"].add_(shift)
        c, g = (t.clone() for t in cap.replay())
        rc, rg = step()
        torch.cuda.synchronize()
        assert torch.equal(c, rc) and torch.equal(g, rg)
        if first is None:
            first = c
    assert not torch.equal(first, c)


def test_autotune_over_cta_configurations_for_a_groups_step():
    """tune_step times a forward solve of two ragged groups over the CTA configurations and
    keeps a valid one; the tuned launch gives the same solution (to the PCG truncation level:
    the CTA shape changes the FP32 reduction order)."""
    from diffmpc_b200.autotune import candidates, tune_step
    from diffmpc_b200.batch import solve_groups

    groups = _ragged_groups(B=8, seed=71)
    lead = groups[0][0]

    def step():
        return solve_groups([(s, s.initial_guess(p), p, None) for s, p in groups])

    ref = [s.controls.clone() for s in step()]
    best = tune_step(lead, step, tag="test", repeats=1, use_cache=False)
    assert best in candidates(lead)
    assert (lead.params["cta_config"], lead.params["threads_per_block"]) == best
    out = step()
    torch.cuda.synchronize()
    for a, b in zip(out, ref):
        assert rel_err(a.controls, b) < 1e-6
