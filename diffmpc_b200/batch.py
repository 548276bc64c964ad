"""Several problem groups in one launch.

``solve_groups`` solves groups that differ in model, state size or horizon (for
example linear nx=12 instances next to quadrotor instances, each group with ragged
per-instance horizons) with ONE forward kernel launch and, on backward, ONE adjoint
launch.  Each group is described as in ``SQPSolver.solve``; the solver options must
be the same for all groups (they go into one parameter block).  The outputs are the
per-group ``SQPSolution``s, differentiable with respect to each group's ``weights``
exactly like ``SQPSolver.solve``.
"""

from typing import Dict, List, Sequence, Tuple

import torch

from . import _lib
from .sqp import AdjointSpec, SQPSolution, SQPSolver, _Call

Problem = Tuple[SQPSolver, SQPSolution, Dict, Dict]


class _GroupsFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, problems, key_lists, holder, *flat):
        calls, shapes, pos = [], [], 0
        for (solver, guess, params, _), keys in zip(problems, key_lists):
            dbg = flat[pos]
            vals = flat[pos + 1 : pos + 1 + len(keys)]
            pos += 1 + len(keys)
            merged = dict(params)
            merged.update({k: v.detach() for k, v in zip(keys, vals)})
            calls.append(_Call(solver, guess, merged, guess.states.shape[0], guess.states.device))
            shapes.append([v.shape for v in vals])
        lead = problems[0][0]
        lib = _lib.load()
        groups = (_lib.Group * len(calls))(*[c.group for c in calls])
        n = lib.dmpc_workspace_size(len(calls), groups, lead._c_params)
        if n == 0 and sum(c.B for c in calls) > 0:
            raise ValueError("invalid group description for the B200 solver")
        dev = calls[0].states.device
        ws = lead._workspace(n, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        ev = lead._event_pair()
        _lib.check(lib.dmpc_solve_fwd(len(calls), groups, lead._c_params, ws.data_ptr(), ws.numel(), stream),
                   "dmpc_solve_fwd")
        lead._event_end(ev, "k_sqp_fwd")
        for (solver, _, _, _), c in zip(problems, calls):
            solver.last_forward_pcg_record = c.pcg_record
        holder["calls"] = calls
        ctx.problems, ctx.key_lists, ctx.calls, ctx.shapes, ctx.groups = problems, key_lists, calls, shapes, groups
        outs = []
        pos = 0
        for c, keys in zip(calls, key_lists):
            outs += [c.states.clone(), c.controls.clone(), c.dual.clone(), flat[pos].detach().clone()]
            pos += 1 + len(keys)
        return tuple(outs)

    @staticmethod
    def backward(ctx, *grads):
        lib = _lib.load()
        specs = []
        for gi, (c, keys) in enumerate(zip(ctx.calls, ctx.key_lists)):
            g_states, g_controls, _, g_dbg = grads[4 * gi : 4 * gi + 4]
            spec = AdjointSpec(ctx.problems[gi][0].program.dynamics, c, g_states, g_controls, g_dbg, keys)
            if spec.n_chunks > 1:
                raise NotImplementedError("more than DMPC_MAX_PARAM_GRADS model-parameter gradients in one group")
            spec.select_chunk(0)
            specs.append(spec)
        lead = ctx.problems[0][0]
        adjs = (_lib.Adjoint * len(specs))(*[sp.adj for sp in specs])
        dev = ctx.calls[0].states.device
        n = lib.dmpc_workspace_size(len(specs), ctx.groups, lead._c_params)
        ws = lead._workspace(n, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        ev = lead._event_pair()
        _lib.check(lib.dmpc_solve_adj(len(specs), ctx.groups, adjs, lead._c_params, ws.data_ptr(), ws.numel(), stream),
                   "dmpc_solve_adj")
        lead._event_end(ev, "k_sqp_adj")
        lead.last_adjoint_pcg_iters = [sp.adj_iters for sp in specs]
        lead.last_adjoint_pcg_record = [sp.adj_record for sp in specs]
        out = [None, None, None]
        for spec, c, keys, shapes in zip(specs, ctx.calls, ctx.key_lists, ctx.shapes):
            g = spec.gradients()
            out.append(g["__dual_backward__"])
            for k, shape in zip(keys, shapes):
                n_el = 1
                for sdim in shape:
                    n_el *= sdim
                gk = g[k].reshape(c.B, -1)
                out.append(gk.sum(0).reshape(shape) if gk.shape[1] == n_el else gk.reshape(shape))
        return tuple(out)


def solve_groups(problems: Sequence[Problem]) -> List[SQPSolution]:
    """Solve every group of ``problems`` = [(solver, initial_guess, problem_params, weights), ...]
    in one forward launch (batched guesses with a leading batch dimension)."""
    if not 1 <= len(problems) <= _lib.DMPC_MAX_GROUPS:
        raise ValueError(f"1..{_lib.DMPC_MAX_GROUPS} groups per launch")
    key_lists, flat = [], []
    for solver, guess, params, weights in problems:
        weights = weights or {}
        keys = sorted(weights)
        key_lists.append(keys)
        dev = guess.states.device
        dbg = guess.dual_backward_guess
        flat.append(torch.zeros_like(guess.dual, dtype=torch.float64) if dbg is None else dbg)
        flat += [torch.as_tensor(weights[k], dtype=torch.float64, device=dev) for k in keys]
    holder = {}
    outs = _GroupsFunction.apply(list(problems), key_lists, holder, *flat)
    sols = []
    for gi, c in enumerate(holder["calls"]):
        states, controls, dual, dbg = outs[4 * gi : 4 * gi + 4]
        sols.append(SQPSolution(states, controls, dual, None, None, None, c.status, c.num_iter, c.conv,
                                c.conv_hist, c.alpha_hist, c.pcg_hist, dbg, c.lin_states, c.lin_controls))
    return sols
