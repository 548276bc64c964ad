"""Mixed-model ragged batches in one launch, and the large-block (global-memory) path.

* `solve_groups`: linear nx=12 instances and quadrotor instances with per-instance
  horizons in ONE forward launch (and one adjoint launch).  Each instance is
  checked against the oracle solving it alone with its own horizon.
* nx=24, N=128 linear with diagonal Q spanning 1e-3..1e3: its FP32 blocks
  (322 KB) do not fit in shared memory and stay in the workspace; in a ragged group
  each instance places its blocks by its own horizon.
"""

import pytest
import torch

from diffmpc_b200 import OptimalControlProblem, SQPSolver, workloads
from diffmpc_b200.batch import solve_groups
from tests.oracle_util import oracle_forward, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _instance_oracle(dyn, st, bt, sp, i, n):
    sti = dict(st)
    sti["horizon"] = n
    bti = workloads.subset(bt, slice(i, i + 1))
    bti["reference_state_trajectory"] = bti["reference_state_trajectory"][:, : n + 1]
    bti["reference_control_trajectory"] = bti["reference_control_trajectory"][:, : n + 1]
    return oracle_forward(dyn, sti, bti, sp)[1]


def _group(make, hz, tol):
    dyn, st, bt, sp = make()
    sp["precision"] = "mixed"
    sp["pcg"]["tol_epsilon"] = tol
    sp["num_scp_iteration_max"] = 6
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    p = workloads.to_device(bt, DEV)
    p["horizons"] = torch.tensor(hz, dtype=torch.int32)
    return dyn, st, bt, sp, solver, p


def test_mixed_models_ragged_one_launch_match_oracle():
    tol = 1e-13
    la = _group(lambda: workloads.linear_lti(B=3, nx=12, nu=4, N=12, seed=41), [12, 6, 9], tol)
    qa = _group(lambda: workloads.quadrotor(B=3, N=10, seed=42), [10, 5, 8], tol)
    probs = []
    for dyn, st, bt, sp, solver, p in (la, qa):
        probs.append((solver, solver.initial_guess(p), p, {}))
    sols = solve_groups(probs)
    torch.cuda.synchronize()
    for (dyn, st, bt, sp, solver, p), sol in zip((la, qa), sols):
        for i, n in enumerate(p["horizons"].tolist()):
            o = _instance_oracle(dyn, st, bt, sp, i, n)
            # 6 SQP iterations leave these instances unconverged, which amplifies the
            # PCG truncation noise in the states; controls are held to the 1e-6 bar
            assert rel_err(sol.controls[i, : n + 1], o.controls[0]) < 1e-6
            assert rel_err(sol.states[i, : n + 1], o.states[0]) < 1e-5


def test_groups_gradients_equal_single_group_solves():
    tol = 1e-13
    la = _group(lambda: workloads.linear_lti(B=2, nx=12, nu=4, N=10, seed=43), [10, 7], tol)
    qa = _group(lambda: workloads.quadrotor(B=2, N=9, seed=44), [9, 6], tol)
    wa = {"weights_penalization_reference_state_trajectory": la[5]["weights_penalization_reference_state_trajectory"].clone().requires_grad_(True)}
    wq = {"mass": qa[5]["mass"].clone().requires_grad_(True),
          "initial_state": qa[5]["initial_state"].clone().requires_grad_(True)}
    sols = solve_groups([(la[4], la[4].initial_guess(la[5]), la[5], wa), (qa[4], qa[4].initial_guess(qa[5]), qa[5], wq)])
    loss = sum((s.controls[:, 0] ** 2).sum() for s in sols)
    loss.backward()
    # the same problems one group at a time
    wa2 = {k: v.detach().clone().requires_grad_(True) for k, v in wa.items()}
    wq2 = {k: v.detach().clone().requires_grad_(True) for k, v in wq.items()}
    s1 = la[4].solve(la[4].initial_guess(la[5]), la[5], wa2)
    s2 = qa[4].solve(qa[4].initial_guess(qa[5]), qa[5], wq2)
    ((s1.controls[:, 0] ** 2).sum() + (s2.controls[:, 0] ** 2).sum()).backward()
    for a, b in ((wa, wa2), (wq, wq2)):
        for k in a:
            assert rel_err(a[k].grad, b[k].grad) < 1e-10, k


def test_ragged_group_places_blocks_per_instance():
    """nx=24 with horizons 128 and 40: the group's longest instance does not fit in shared
    memory, so each instance decides at run time (the short one keeps its FP32 blocks on
    chip, the long one in the workspace)."""
    dyn, st, bt, sp, solver, p = _group(lambda: workloads.linear_stress(B=2, seed=46), [128, 40], 1e-13)
    sol = solver.solve(solver.initial_guess(p), p)
    torch.cuda.synchronize()
    for i, n in enumerate(p["horizons"].tolist()):
        o = _instance_oracle(dyn, st, bt, sp, i, n)
        assert rel_err(sol.controls[i, : n + 1], o.controls[0]) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_blocks_global_memory_path(precision):
    dyn, st, bt, sp = workloads.linear_stress(B=2, seed=45)
    sp["precision"] = precision
    sp["pcg"]["tol_epsilon"] = 1e-13
    sp["num_scp_iteration_max"] = 2
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    p = workloads.to_device(bt, DEV)
    sol = solver.solve(solver.initial_guess(p), p)
    torch.cuda.synchronize()
    _, o = oracle_forward(dyn, st, bt, sp)
    # ~3500 PCG iterations on a system with diag(Q) spanning 1e-3..1e3: FP64 roundoff alone
    # separates two FP64 implementations by ~1e-8; the mixed path falls back to FP64 when
    # FP32 refinement stagnates
    assert rel_err(sol.controls, o.controls) < (1e-7 if precision == "fp64" else 1e-6)
