"""GPU parity of the two-CTA configuration (cta_config DUAL: 256 threads, two instances per SM),
whose mixed-precision PCG keeps one register copy of each scaled off-diagonal block and forms the
transposed products with warp-shuffle reduce-scatters (pcg_rows_t), against the CPU oracle.

Every nx with a compiled row layout is covered: 1 thread per knot (nx=3 spacecraft, nx=4
linear), 2 (nx=6, 7, 8) and 4 (nx=12 linear, nx=13 quadrotor), with short horizons (most threads
of the CTA idle) and the headline's N=60 (244 of 256 threads busy).  Bars as elsewhere: controls
1e-6 and gradients 1e-5 relative in mixed precision, at PCG tolerances tight enough for the
oracle's own answer to sit inside them.
"""

import pytest
import torch

from diffmpc_b200 import workloads
from tests.oracle_util import oracle_forward, oracle_gradients, rel_err
from tests.test_gpu_sqp import DEV, _spacecraft, gpu_solve

pytestmark = pytest.mark.gpu

DUAL = 3  # DMPC_CTA_DUAL


def _mixed_dual(sp, eps):
    sp["precision"] = "mixed"
    sp["cta_config"] = DUAL
    sp["pcg"]["tol_epsilon"] = eps
    return sp


@pytest.mark.parametrize("nx,N", [(4, 30), (6, 40), (7, 25), (8, 40), (12, 60)])
def test_linear_dual_matches_oracle(nx, N):
    dyn, st, bt, sp = workloads.linear_lti(B=3, N=N, nx=nx, nu=3, seed=1100 + nx)
    _mixed_dual(sp, 1e-20)
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-6
    assert rel_err(sol.states, osol.states) < 1e-6
    assert torch.equal(sol.num_iter.cpu().long(), osol.num_iter.long())


def test_spacecraft_dual_matches_oracle():
    dyn, st, bt, sp = _spacecraft(B=3, N=12)
    _mixed_dual(sp, 1e-20)
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-6


def test_attitude_n50_dual_matches_oracle():
    dyn, st, bt, sp = workloads.attitude(B=2, N=50, seed=1001)
    _mixed_dual(sp, 1e-18)
    _, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-6
    assert rel_err(sol.states, osol.states) < 1e-6


@pytest.mark.parametrize("N", [10, 60])
def test_quadrotor_dual_forward_and_adjoint_match_oracle(N):
    dyn, st, bt, sp = workloads.quadrotor(B=2, N=N, seed=1002)
    _mixed_dual(sp, 1e-20)
    keys = ["initial_state", "weights_penalization_reference_state_trajectory",
            "weights_penalization_control_squared", "mass"]
    w = {k: bt[k].clone().to(DEV).requires_grad_(True) for k in keys}
    _, sol = gpu_solve(dyn, st, bt, sp, weights=w)
    (sol.controls[:, 0] ** 2).sum().backward()
    osolver, osol = oracle_forward(dyn, st, bt, sp, weights={k: bt[k] for k in keys})
    assert rel_err(sol.controls, osol.controls) < 1e-6
    dlu = torch.zeros_like(osol.controls)
    dlu[:, 0] = 2 * osol.controls[:, 0]
    og, _, _ = oracle_gradients(osolver, osol, bt, {k: bt[k] for k in keys}, torch.zeros_like(osol.states), dlu)
    for k in keys:
        assert rel_err(w[k].grad.detach(), og[k]) < 1e-5, k


def test_ill_conditioned_dual_hands_over_and_matches_oracle():
    """cond(S) 1e7..1e9 (state weights over 1e-6..1e6), nx=6: the two-CTA row PCG applies the
    same stall detection and hand-over as the one-CTA row PCG."""
    dyn, st, bt, sp = workloads.linear_lti(B=3, N=40, nx=6, nu=3, seed=1003, log10_wx=6.0)
    _mixed_dual(sp, 1e-20)
    solver, sol = gpu_solve(dyn, st, bt, sp)
    _, osol = oracle_forward(dyn, st, bt, sp)
    assert rel_err(sol.controls, osol.controls) < 1e-6
    its = sol.num_pcg_iters.cpu()
    assert int(its.max()) < sp["pcg"]["max_iter"] // 2, its
    rec = solver.last_forward_pcg_record.cpu()
    assert int((rec[1, :, 0] > 0).sum()) >= 2, rec


def test_dual_and_row_configurations_agree_on_a_headline_batch():
    """64 quadrotor instances (N=60) at the headline's tolerance: the two-CTA and the one-CTA
    row PCG both land within 1e-6 of the all-FP64 path on every instance's controls."""
    dyn, st, bt, sp = workloads.quadrotor(B=64, N=60, seed=1002)
    sp["pcg"]["tol_epsilon"] = 1e-20
    sp["num_scp_iteration_max"] = 3
    sp["precision"] = "fp64"
    _, s64 = gpu_solve(dyn, st, bt, sp)
    ref = s64.controls.detach()
    for cfg in (DUAL, 2):
        sp["precision"] = "mixed"
        sp["cta_config"] = cfg
        _, sol = gpu_solve(dyn, st, bt, sp)
        c = sol.controls.detach()
        err = ((c - ref).abs().amax(dim=(1, 2)) / ref.abs().amax(dim=(1, 2))).max()
        assert float(err) < 1e-6, (cfg, float(err))
        assert torch.equal(sol.status.cpu(), s64.status.cpu())


def test_dual_solves_are_deterministic():
    """Fixed-order reductions and shuffles: two solves of the same batch (forward and adjoint)
    give bit-equal controls, duals, iteration counts and gradients."""
    dyn, st, bt, sp = workloads.quadrotor(B=300, N=60, seed=1002)  # more instances than SMs: AUTO takes DUAL
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = 1e-20
    sp["num_scp_iteration_max"] = 3
    outs = []
    for _ in range(2):
        w = {"initial_state": bt["initial_state"].clone().to(DEV).requires_grad_(True)}
        _, sol = gpu_solve(dyn, st, bt, sp, weights=w)
        (sol.controls[:, 0] ** 2).sum().backward()
        outs.append((sol.controls.detach().cpu(), sol.dual.detach().cpu(), sol.num_pcg_iters.cpu(), w["initial_state"].grad.cpu()))
    for a, b in zip(*outs):
        assert torch.equal(a, b)
