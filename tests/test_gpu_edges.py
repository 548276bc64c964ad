"""Edge cases of the fused solver against the CPU oracle: the shortest horizons (one and two
stages, where most threads of a CTA have no knot), and a non-finite initial state, on which the
reference reports ERROR after its single forced SQP iteration and returns nan_to_num'd arrays
(sqp.py:535-559) while the other instances of the batch are unaffected."""

import pytest
import torch

from diffmpc_b200 import workloads
from tests.oracle_util import oracle_forward, rel_err
from tests.test_gpu_sqp import gpu_solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("N", [1, 2])
def test_shortest_horizons_match_oracle(N, precision):
    dyn, st, bt, sp = workloads.quadrotor(B=3, N=N, seed=40 + N)
    sp["precision"] = precision
    sp["pcg"]["tol_epsilon"] = 1e-20
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    tol = 1e-8 if precision == "fp64" else 1e-6
    assert rel_err(sol.controls, osol.controls) < tol
    assert rel_err(sol.states, osol.states) < tol
    if precision == "fp64":
        assert torch.equal(sol.num_iter.cpu().long(), osol.num_iter.long())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_non_finite_initial_state_reports_error_like_the_oracle(precision):
    dyn, st, bt, sp = workloads.linear_lti(B=3, N=12, seed=77)
    sp["precision"] = precision
    sp["pcg"]["tol_epsilon"] = 1e-20
    bt["initial_state"] = bt["initial_state"].clone()
    bt["initial_state"][1, 2] = float("nan")
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    status, ostatus = sol.status.cpu().long(), osol.status.long()
    assert int(status[1]) == int(ostatus[1]) == -100
    assert torch.equal(status, ostatus)
    assert int(sol.num_iter[1]) == int(osol.num_iter[1])
    for name in ("states", "controls", "dual"):
        v = getattr(sol, name).detach().cpu()
        assert bool(torch.isfinite(v).all()), name  # nan_to_num
    keep = [0, 2]
    tol = 1e-8 if precision == "fp64" else 1e-6
    assert rel_err(sol.controls[keep], osol.controls[keep]) < tol
    assert rel_err(sol.states[keep], osol.states[keep]) < tol
