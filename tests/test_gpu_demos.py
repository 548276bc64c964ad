"""GPU solver against outputs of the reference solver itself: the 32 cart-pole
expert demonstrations of benchmarking/imitation-learning/demonstrations.pkl
(collect_expert_data.py: N=100, line search, SQP <= 501 iterations, PCG 1e-24),
all 32 re-solved in one launch."""

import numpy as np
import pytest
import torch

from diffmpc_b200 import CartpoleDynamics, OptimalControlProblem, SQPSolver
from tests.test_oracle_pins import DEMOS, cartpole_demo_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cartpole_demonstrations_on_gpu(precision):
    d = np.load(DEMOS)
    p, sp = cartpole_demo_problem()
    sp["precision"] = precision
    st = {k: (torch.as_tensor(np.asarray(v), dtype=torch.float64) if not isinstance(v, (int, bool)) or isinstance(v, float) else v)
          for k, v in p.items()}
    st["horizon"], st["discretization_scheme"], st["penalize_control_reference"] = 100, 0, False
    solver = SQPSolver(OptimalControlProblem(CartpoleDynamics(), st), params=sp)
    B = d["x0"].shape[0]
    bp = {k: (v.to("cuda") if isinstance(v, torch.Tensor) else v) for k, v in st.items()}
    bp["initial_state"] = torch.tensor(d["x0"], device="cuda")
    sol = solver.solve(solver.initial_guess(bp), bp)
    torch.cuda.synchronize()
    ref = torch.tensor(d["ctrl_traj"])
    u = sol.controls.cpu()
    rel = ((u - ref).abs().amax(dim=(1, 2)) / ref.abs().amax(dim=(1, 2)))
    # Every demonstration converged in the reference.  Two of them converge only by line-search
    # creep near the SQP tolerance: on a B200 the FP64 path reaches 1e-8 on demonstration 29 at
    # SQP iteration 501 of 501 and leaves demonstration 30 at ~7e-6, so whether the 1e-8 test is
    # met within the iteration cap there is decided at rounding level.  The mixed path may leave
    # both just short of it; the control trajectories below are held to the recorded ones.
    assert int((sol.status.cpu() == 0).sum()) >= (B - 1 if precision == "fp64" else B - 2)
    assert float(rel.median()) < 1e-6
    assert int((rel < 1e-5).sum()) >= B - 1
