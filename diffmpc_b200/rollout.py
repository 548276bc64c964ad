"""Closed-loop MPC rollout fused on the device, differentiable w.r.t. the solver weights.

The reference's reinforcement-learning benchmarks and notebooks run this loop
(benchmarking/reinforcement-learning/benchmark_diffmpc.py:140-175): a ``lax.scan``
over simulation steps whose body solves the MPC from the current state (warm-started
from the previous solution), applies the first control, steps a discrete linear
simulator ``x+ = A x + B u + b`` and accumulates ``|x+|^2 + |u|^2``; ``vmap`` runs it
for a batch of initial states and ``jax.grad`` differentiates the summed cost w.r.t.
the solver weights.

Here one kernel launch (``dmpc_rollout_fwd``) runs every step of every instance: one
CTA per instance keeps its workspace across the steps, so the loop pays no per-step
launch or host round trip.  The backward pass (``dmpc_rollout_adj``, also one launch)
sweeps the steps in reverse and runs the adjoint of each step's solve at its saved
solution:

    lam_T = 2 x_T
    g_u,k = 2 u_k + B^T lam_{k+1}           (cotangent of controls[0] of step k)
    grad_w += adjoint_k(dl/du_0 = g_u,k)
    lam_k  = A^T lam_{k+1} + 2 x_k  (k >= 1)

As in the reference, a solve's problem parameters (its initial state among them) are
not differentiated (the custom VJP returns no cotangent for them, sqp.py:781-795), so
the state reaches the gradient only through the simulator.  ``through_state=True``
adds each solve's dL/dx_0 to lam_k, i.e. differentiates through the MPC's dependence on
the state as well.
"""

from types import SimpleNamespace
from typing import Dict, Optional

import torch

from . import _lib
from .sqp import AdjointSpec, SQPSolution, SQPSolver, _Call, _ptr


def _per_instance(m, B, shape, device):
    t = torch.as_tensor(m, dtype=torch.float64, device=device)
    if t.dim() == len(shape):
        t = t.expand(B, *shape)
    return t.reshape(B, *shape).contiguous()


class _RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, roll, x0, problem_params, guess, keys, *vals):
        solver = roll.solver
        dev = x0.device
        B = x0.shape[0]
        params = dict(problem_params)
        params.update({k: v.detach() for k, v in zip(keys, vals)})
        params["initial_state"] = x0.detach()
        if guess is None:
            guess = solver.initial_guess(params)
        call = _Call(solver, guess, params, B, dev)
        nx, nu, K, T = call.nx, call.nu, call.K, roll.num_sim_steps
        mi = solver.maxiter
        f64 = lambda *s: torch.zeros(*s, dtype=torch.float64, device=dev)  # noqa: E731
        i32 = lambda *s: torch.zeros(*s, dtype=torch.int32, device=dev)  # noqa: E731
        linear = roll.simulator == "linear"
        # Python numbers are filled on the device: no host-to-device copy (CUDA-graph capture)
        vec = lambda v, n: (torch.full((n,), float(v), dtype=torch.float64, device=dev)  # noqa: E731
                            if isinstance(v, (int, float)) else
                            torch.as_tensor(v, dtype=torch.float64, device=dev).expand(n).contiguous())
        cw = SimpleNamespace(ws=vec(roll.state_weight, nx), wc=vec(roll.control_weight, nu),
                             xr=None if roll.state_ref is None else vec(roll.state_ref, nx),
                             ur=None if roll.control_ref is None else vec(roll.control_ref, nu))
        st = SimpleNamespace(
            A=_per_instance(roll.sim_A, B, (nx, nx), dev) if linear else None,
            Bm=_per_instance(roll.sim_B, B, (nx, nu), dev) if linear else None,
            b=_per_instance(roll.sim_b, B, (nx,), dev) if linear else None,
            x=f64(T + 1, B, nx), states=f64(T, B, K, nx), controls=f64(T, B, K, nu), dual=f64(T, B, K, nx),
            lin_states=f64(T, B, K, nx), lin_controls=f64(T, B, K, nu), status=i32(T, B), num_iter=i32(T, B),
            conv=f64(T, B), conv_hist=f64(T, B, mi), alpha_hist=f64(T, B, mi), pcg_hist=i32(T, B, mi), cost=f64(B),
        )
        r = _lib.Rollout()
        r.num_steps, r.warm_start = T, 1 if roll.warm_start else 0
        r.simulator = {"linear": _lib.SIM_LINEAR, "euler": _lib.SIM_MODEL, "integrator": _lib.SIM_MODEL_SCHEME}[
            roll.simulator]
        r.cost_state_weights, r.cost_control_weights = _ptr(cw.ws), _ptr(cw.wc)
        r.cost_state_ref, r.cost_control_ref = _ptr(cw.xr), _ptr(cw.ur)
        r.sim_A, r.sim_B, r.sim_b = _ptr(st.A), _ptr(st.Bm), _ptr(st.b)
        r.step_initial_state, r.step_states, r.step_controls = _ptr(st.x), _ptr(st.states), _ptr(st.controls)
        r.step_dual, r.step_lin_states, r.step_lin_controls = _ptr(st.dual), _ptr(st.lin_states), _ptr(st.lin_controls)
        r.step_status, r.step_num_iter, r.step_convergence_error = _ptr(st.status), _ptr(st.num_iter), _ptr(st.conv)
        r.step_convergence_errors, r.step_linesearch_alphas = _ptr(st.conv_hist), _ptr(st.alpha_hist)
        r.step_num_pcg_iters, r.running_cost = _ptr(st.pcg_hist), _ptr(st.cost)
        lib = _lib.load()
        n = lib.dmpc_workspace_size(1, call.group, solver._c_params)
        if n == 0 and B > 0:
            raise ValueError("invalid problem description for the B200 solver")
        ws = solver._workspace(n, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        ev = solver._event_pair()
        _lib.check(lib.dmpc_rollout_fwd(call.group, r, solver._c_params, ws.data_ptr(), ws.numel(), stream),
                   "dmpc_rollout_fwd")
        solver._event_end(ev, "k_rollout_fwd")
        roll.last = st
        ctx.roll, ctx.call, ctx.st, ctx.keys, ctx.r, ctx.cw = roll, call, st, keys, r, cw
        ctx.shapes = [v.shape for v in vals]
        return st.cost.clone()

    @staticmethod
    def backward(ctx, g_cost):
        roll, call, st, keys = ctx.roll, ctx.call, ctx.st, ctx.keys
        if roll.fused_backward or roll.simulator != "linear":
            acc, gx0 = _fused_sweep(ctx, g_cost)
        else:
            acc, gx0 = _per_step_sweep(ctx, g_cost)
        B = call.B
        out = []
        for key, shape in zip(keys, ctx.shapes):
            gk = acc[key].reshape(B, -1)
            n = 1
            for s in shape:
                n *= s
            out.append(gk.sum(0).reshape(shape) if gk.shape[1] == n else gk.reshape(shape))
        return (None, gx0, None, None, None) + tuple(out)


def _fused_sweep(ctx, g_cost):
    """dmpc_rollout_adj: the whole reverse sweep in one launch per parameter chunk."""
    roll, call, st, keys = ctx.roll, ctx.call, ctx.st, ctx.keys
    solver = roll.solver
    B, K, nx, nu = call.B, call.K, call.nx, call.nu
    dev = st.x.device
    go = g_cost.to(torch.float64).reshape(B).contiguous()
    view = SimpleNamespace(group=call.group, states=st.states[0], B=B, K=K, nx=nx, nu=nu)
    spec = AdjointSpec(solver.program.dynamics, view, None, None, None, keys)
    scratch_u = torch.zeros(B, K, nu, dtype=torch.float64, device=dev)
    scratch_l = torch.zeros(B, K, nx, dtype=torch.float64, device=dev)
    gx0 = torch.zeros(B, nx, dtype=torch.float64, device=dev)
    rr = _lib.RolloutAdjoint()
    rr.cost_cotangent, rr.through_state = _ptr(go), 1 if roll.through_state else 0
    rr.scratch_dl_dcontrols, rr.scratch_dual, rr.g_initial_state = _ptr(scratch_u), _ptr(scratch_l), _ptr(gx0)
    lib = _lib.load()
    ws = solver._workspace(lib.dmpc_workspace_size(1, call.group, solver._c_params), dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for ci in range(spec.n_chunks):
        spec.select_chunk(ci)
        ev = solver._event_pair()
        _lib.check(lib.dmpc_rollout_adj(call.group, ctx.r, spec.adj, rr, solver._c_params, ws.data_ptr(), ws.numel(),
                                        stream), "dmpc_rollout_adj")
        solver._event_end(ev, "k_rollout_adj")
    grads = spec.gradients()
    return {k: grads[k] for k in keys}, gx0


def _per_step_sweep(ctx, g_cost):
    """The same sweep with one batched dmpc_solve_adj launch per step (host loop)."""
    roll, call, st, keys = ctx.roll, ctx.call, ctx.st, ctx.keys
    solver = roll.solver
    B, K, nx, nu, T = call.B, call.K, call.nx, call.nu, roll.num_sim_steps
    go = g_cost.to(torch.float64).reshape(B, 1)
    cw = ctx.cw
    dcx = lambda x: 2.0 * go * cw.ws * (x - (0.0 if cw.xr is None else cw.xr))  # noqa: E731
    dcu = lambda u: 2.0 * go * cw.wc * (u - (0.0 if cw.ur is None else cw.ur))  # noqa: E731
    akeys = list(keys) + (["initial_state"] if roll.through_state and "initial_state" not in keys else [])
    acc = {}
    lam = dcx(st.x[T])
    for k in reversed(range(T)):
        u = st.controls[k, :, 0]
        g_u = dcu(u) + torch.einsum("bij,bi->bj", st.Bm, lam)
        dlu = torch.zeros(B, K, nu, dtype=torch.float64, device=u.device)
        dlu[:, 0] = g_u
        g = _lib.Group.from_buffer_copy(call.group)
        g.initial_state = _ptr(st.x[k])
        g.states, g.controls, g.dual = _ptr(st.states[k]), _ptr(st.controls[k]), _ptr(st.dual[k])
        g.lin_states, g.lin_controls = _ptr(st.lin_states[k]), _ptr(st.lin_controls[k])
        g.status, g.num_iter, g.convergence_error = _ptr(st.status[k]), _ptr(st.num_iter[k]), _ptr(st.conv[k])
        g.convergence_errors, g.linesearch_alphas = _ptr(st.conv_hist[k]), _ptr(st.alpha_hist[k])
        g.num_pcg_iters = _ptr(st.pcg_hist[k])
        view = SimpleNamespace(group=g, states=st.states[k], B=B, K=K, nx=nx, nu=nu)
        dbg = torch.zeros(B, K, nx, dtype=torch.float64, device=u.device)
        grads = solver._run_adj(view, None, dlu, dbg, akeys) if akeys else {}
        for key in keys:
            acc[key] = grads[key] if key not in acc else acc[key] + grads[key]
        lam = torch.einsum("bij,bi->bj", st.A, lam)
        if roll.through_state:
            lam = lam + grads["initial_state"]
        if k >= 1:
            lam = lam + dcx(st.x[k])
    return acc, lam


class ClosedLoopRollout:
    """MPC-in-the-loop rollout of ``num_sim_steps`` steps.

    ``simulator="linear"``: ``x+ = sim_A x + sim_B u + sim_b`` (each shared by the batch or
    given per instance), as in benchmark_diffmpc.py:148-150.  ``simulator="euler"``: one Euler
    step ``x+ = x + dt f(x, u)`` of the solver's own model with each instance's ``dt`` and
    model parameters, as in spacecraft/benchmark_diffmpc.py:87-89.  ``simulator="integrator"``:
    one step of the solver's own integrator (its discretization scheme), as the RL_quadrotor
    notebook simulates.  The model simulators use the model parameters the solves see (a
    weight that overrides one applies to both) and are not differentiated with respect to them.

    ``rollout(initial_states, problem_params, weights)`` returns the running cost
    ``sum_k sum_i state_weight_i (x_{k+1,i} - state_ref_i)^2 + sum_j control_weight_j
    (u_{k,j} - control_ref_j)^2`` per instance (shape ``(B,)``; weights are scalars or
    vectors shared by the batch, references default to zero).  The reference scripts' reward
    is its negative: weights 1, 1 for the linear benchmark, 10, 1 for the spacecraft one.  It
    is differentiable with respect to ``weights`` (any key ``SQPSolver.solve`` accepts) and
    ``initial_states``.
    ``warm_start`` starts each solve from the previous step's solution, as the
    reference's ``warm_start`` flag does.  The backward pass is one launch per parameter
    chunk (``dmpc_rollout_adj``); for the linear simulator ``fused_backward=False`` runs
    the same sweep as one ``dmpc_solve_adj`` launch per step instead.  After a call, ``last`` holds every step's
    solution (``states``, ``controls``, ``x`` ...) and iteration counts.
    """

    def __init__(self, solver: SQPSolver, sim_A=None, sim_B=None, sim_b=None, num_sim_steps: int = 1,
                 warm_start: bool = True, through_state: bool = False, fused_backward: bool = True,
                 simulator: str = "linear", state_weight=1.0, control_weight=1.0, state_ref=None, control_ref=None):
        if num_sim_steps < 1:
            raise ValueError("num_sim_steps must be >= 1")
        if simulator not in ("linear", "euler", "integrator"):
            raise ValueError("simulator must be 'linear', 'euler' or 'integrator'")
        if simulator == "linear" and (sim_A is None or sim_B is None or sim_b is None):
            raise ValueError("the linear simulator needs sim_A, sim_B and sim_b")
        self.simulator = simulator
        self.state_weight, self.control_weight = state_weight, control_weight
        self.state_ref, self.control_ref = state_ref, control_ref
        self.solver = solver
        self.sim_A, self.sim_B, self.sim_b = sim_A, sim_B, sim_b
        self.num_sim_steps = int(num_sim_steps)
        self.warm_start = bool(warm_start)
        self.through_state = bool(through_state)
        self.fused_backward = bool(fused_backward)
        self.last = None

    def __call__(self, initial_states: torch.Tensor, problem_params: Dict, weights: Optional[Dict] = None,
                 initial_guess: Optional[SQPSolution] = None) -> torch.Tensor:
        weights = weights or {}
        if "initial_state" in weights:
            raise ValueError("the rollout's initial states are `initial_states`, not a weight")
        x0 = torch.as_tensor(initial_states, dtype=torch.float64)
        keys = sorted(weights.keys())
        vals = [torch.as_tensor(weights[k], dtype=torch.float64, device=x0.device) for k in keys]
        return _RolloutFunction.apply(self, x0, problem_params, initial_guess, keys, *vals)

    def solutions(self, k: int) -> SQPSolution:
        """Step k's solution (no gradient)."""
        st = self.last
        return SQPSolution(st.states[k], st.controls[k], st.dual[k], None, None, None, st.status[k], st.num_iter[k],
                           st.conv[k], st.conv_hist[k], st.alpha_hist[k], st.pcg_hist[k], None,
                           st.lin_states[k], st.lin_controls[k])
