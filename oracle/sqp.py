"""SQP solver restatement (oracle, float64, batched).

Follows diffmpc/solvers/sqp.py: QP assembly (:160-260), one SQP iteration
(:262-299), the l1-merit line search (:301-411), the SQP ``while_loop`` with
status and ``nan_to_num`` (:436-560), and the implicit-function backward with
mixed partial derivatives (:589-798).

Batching: every tensor carries a leading batch dimension ``B``.  Problem
parameters are a dict whose tensor values are batched ``(B, ...)``; the
three static keys (horizon, discretization_scheme, penalize_control_reference)
live on the problem object.

One documented difference: the reference evaluates the mixed derivatives of
the backward pass with the program's construction-time parameters overridden
by ``weights`` (sqp.py:629 ``self.make_params_with_weights(w)``); this
restatement uses the call's parameters overridden by ``weights``.  The two
agree whenever the call's parameters that are not in ``weights`` equal the
program's, which holds for every recorded reference output.
"""

import copy
from typing import Any, NamedTuple

import torch
from torch.func import grad, jacfwd, jacrev, vmap

from . import pcg as P
from .ocp import STATIC_KEYS

SUCCESS, ERROR = 0, -100  # sqp.py:31-35

DEFAULT_SOLVER_PARAMS = {  # solvers/params/sqp.yaml:1-11
    "verbose": False,
    "tol_convergence": 1e-8,
    "num_scp_iteration_max": 15,
    "linesearch": False,
    "linesearch_eta": 0.4,
    "linesearch_alphas": [0.01, 0.1, 0.3, 0.7, 1.0],
    "warm_start_backward": True,
    "pcg": {"verbose": False, "max_iter": 10000, "tol_epsilon": 1e-9},
}


def default_solver_params():
    return copy.deepcopy(DEFAULT_SOLVER_PARAMS)


class SQPSolution(NamedTuple):  # sqp.py:38-57
    states: torch.Tensor
    controls: torch.Tensor
    dual: torch.Tensor
    qp_parameters: Any
    dynamics_cost_premultiplied_matrices: Any
    schur_complement_matrices: Any
    status: torch.Tensor
    num_iter: torch.Tensor
    convergence_error: torch.Tensor
    convergence_errors: torch.Tensor
    linesearch_alphas: torch.Tensor
    num_pcg_iters: torch.Tensor
    dual_backward_guess: torch.Tensor = None


def project_psd(M, minimum_eigenvalue):
    """PSD projection by eigen-decomposition (jax_utils.py:75-95).  The input is symmetrized first,
    (M + M^T) / 2, as jnp.linalg.eigh does by default (symmetrize_input=True); torch's eigh would
    otherwise read only the lower triangle."""
    S, V = torch.linalg.eigh(0.5 * (M + M.mT))
    S = torch.clamp(S, min=minimum_eigenvalue)
    proj = V @ (torch.diag_embed(S) @ V.mT)
    return 0.5 * (proj + proj.mT)


def _sel(mask, new, old):
    m = mask.reshape(mask.shape + (1,) * (new.dim() - mask.dim()))
    return torch.where(m, new, old)


def _sel_tree(mask, new, old):
    if isinstance(new, torch.Tensor):
        return _sel(mask, new, old)
    return type(new)(*[_sel_tree(mask, a, b) for a, b in zip(new, old)])


class SQPSolver:
    """Restatement of SQPSolver (sqp.py:60-802) on batched inputs."""

    def __init__(self, program, name="SQPSolver", params=None):
        if params is None:
            params = default_solver_params()
        self.program = program
        self.name = name
        self.params = params
        self.maxiter = int(params["num_scp_iteration_max"])
        self.pcg = P.PCGOptimalControl(
            program.horizon,
            program.num_state_variables,
            program.num_control_variables,
            params["pcg"],
        )

    # -- helpers --------------------------------------------------------------
    def _tensor_params(self, params):
        return {k: v for k, v in params.items() if k not in STATIC_KEYS}

    def make_params_with_weights(self, weights, problem_params):
        new = dict(problem_params)
        for k, v in weights.items():
            new[k] = v
        return new

    def initial_guess(self, params):
        """Batched straight-line guess (sqp.py:143-158)."""
        tp = self._tensor_params(params)
        x, u = vmap(self.program.initial_guess)(tp)
        B = x.shape[0]
        K, nx = x.shape[1], x.shape[2]
        z = torch.zeros(B, K, nx, dtype=torch.float64)
        mi = self.maxiter
        return SQPSolution(
            x,
            u,
            z.clone(),
            self.pcg.zero_qp_parameters((B,)),
            self.pcg.zero_dynamics_cost_premultiplied_matrices((B,)),
            self.pcg.zero_schur_complement_matrices((B,)),
            torch.zeros(B, dtype=torch.int64),
            torch.zeros(B, dtype=torch.int64),
            torch.zeros(B, dtype=torch.float64),
            torch.zeros(B, mi, dtype=torch.float64),
            torch.zeros(B, mi, dtype=torch.float64),
            torch.zeros(B, mi, dtype=torch.int64),
            z.clone(),
        )

    # -- QP assembly ------------------------------------------------------------
    def get_cost_terms(self, states, controls, tp):
        QN, qN, Q, q, R, r = vmap(self.program.get_cost_linearized_matrices)(states, controls, tp)
        Qs = torch.cat([Q, QN[:, None]], dim=1)
        qs = torch.cat([q, qN[:, None]], dim=1)
        Qs = project_psd(Qs, 1e-9)
        Rs = project_psd(R, 1e-9)
        return Qs, qs, Rs, r

    def compute_qp_parameters(self, states, controls, tp):
        Qs, qs, Rs, rs = self.get_cost_terms(states, controls, tp)
        dyn = P.QPDynamicsParameters(
            *vmap(self.program.get_dynamics_linearized_matrices)(states, controls, tp)
        )
        Qinv = torch.linalg.inv(Qs)
        Rinv = torch.linalg.inv(Rs)
        qp = P.QPParameters(dyn, P.QPCostParameters(Qinv, qs, Rinv, rs))
        premult = P.premultiplied_matrices(qp)
        schur = P.compute_S_Phiinv(qp)
        return qp, premult, schur

    def solve_one_scp_iteration(self, states, controls, dual, tp):
        qp, premult, schur = self.compute_qp_parameters(states, controls, tp)
        gammas = P.compute_gamma(
            premult, qp.dynamics.Cs, qp.cost.Qinv[:, 0], qp.cost.qvec, qp.cost.rvec
        )
        sol, dbg = self.pcg.solve_KKT_Schur(qp, schur, gammas, dual)
        return sol, qp, premult, schur, dbg.num_iterations

    # -- line search (sqp.py:301-411) -------------------------------------------
    def linesearch(self, states, controls, new_states, new_controls, tp):
        eta = self.params["linesearch_eta"]
        alphas = torch.tensor(self.params["linesearch_alphas"], dtype=torch.float64)
        n_alpha = alphas.numel()
        prog = self.program
        nx = prog.num_state_variables
        K = prog.horizon + 1

        def one(x, u, xn, un, p):
            dx, du = xn - x, un - u
            z = torch.cat([x, u], dim=-1).reshape(-1)
            dz = torch.cat([dx, du], dim=-1).reshape(-1)

            def cost_fn(zz):
                zz = zz.reshape(K, -1)
                return prog.cost(zz[:, :nx], zz[:, nx:], p)

            cost = cost_fn(z)
            cost_dz = jacrev(cost_fn)(z)
            cdz = torch.dot(cost_dz, dz)
            l1 = torch.sum(torch.abs(prog.equality_constraints(x, u, p)))
            mu_min = cdz / (0.5 * l1)
            mu = torch.maximum(torch.tensor(0.1, dtype=torch.float64), mu_min)
            merit = cost + mu * l1
            merit_d = cdz + -mu * l1

            def decrease(alpha):
                cx, cu = x + alpha * dx, u + alpha * du
                c = prog.cost(cx, cu, p)
                eq = prog.equality_constraints(cx, cu, p)
                return c + mu * torch.sum(torch.abs(eq)) - (merit + eta * alpha * merit_d)

            return torch.stack([decrease(alphas[i]) for i in range(n_alpha)])

        dv = vmap(one)(states, controls, new_states, new_controls, tp)  # (B, n_alpha)
        B = dv.shape[0]
        # while_loop from index n+1 down; gathers clamp their index (JAX semantics)
        out = torch.empty(B, dtype=torch.float64)
        clamp = lambda i: min(max(i, 0), n_alpha - 1)  # noqa: E731
        for b in range(B):
            i, alpha = n_alpha + 1, float(alphas.max())
            while not (bool(dv[b, clamp(i)] < 0) or i == 0):
                i, alpha = i - 1, float(alphas[clamp(i - 1)])
            out[b] = alpha
        a = out[:, None, None]
        return states + a * (new_states - states), controls + a * (new_controls - controls), out

    # -- forward solve (sqp.py:436-560) -------------------------------------------
    def _solve(self, guess, problem_params, weights=None):
        weights = weights or {}
        tp = self._tensor_params(self.make_params_with_weights(weights, problem_params))
        tp = {k: v.detach() if isinstance(v, torch.Tensor) else v for k, v in tp.items()}
        tol = self.params["tol_convergence"]
        B = guess.states.shape[0]
        states = guess.states.detach()
        controls = guess.controls.detach()
        dual = guess.dual.detach()
        qp = guess.qp_parameters
        premult = guess.dynamics_cost_premultiplied_matrices
        schur = guess.schur_complement_matrices
        num_iter = torch.zeros(B, dtype=torch.int64)
        conv_err = torch.as_tensor(guess.convergence_error, dtype=torch.float64).expand(B).clone()
        conv_errs = guess.convergence_errors.clone()
        alphas_rec = guess.linesearch_alphas.clone()
        pcg_iters = guess.num_pcg_iters.clone()
        ar = torch.arange(B)
        while True:
            cont = ((num_iter < self.maxiter) & (conv_err > tol)) | (num_iter < 1)
            if not bool(cont.any()):
                break
            sol, qp_n, pm_n, sc_n, npcg = self.solve_one_scp_iteration(states, controls, dual, tp)
            xs_n, us_n = sol.states, sol.controls
            if self.params["linesearch"]:
                xs_n, us_n, alpha = self.linesearch(states, controls, xs_n, us_n, tp)
                idx = num_iter.clamp(max=self.maxiter - 1)
                upd = alphas_rec.clone()
                upd[ar, idx] = alpha
                alphas_rec = _sel(cont & (num_iter < self.maxiter), upd, alphas_rec)
            err = torch.maximum(
                (xs_n - states).abs().amax(dim=(-2, -1)), (us_n - controls).abs().amax(dim=(-2, -1))
            )
            idx = num_iter.clamp(max=self.maxiter - 1)
            ok = cont & (num_iter < self.maxiter)
            ce = conv_errs.clone()
            ce[ar, idx] = err
            pi = pcg_iters.clone()
            pi[ar, idx] = npcg
            conv_errs = _sel(ok, ce, conv_errs)
            pcg_iters = _sel(ok, pi, pcg_iters)
            states = _sel(cont, xs_n, states)
            controls = _sel(cont, us_n, controls)
            dual = _sel(cont, sol.kkt_multipliers, dual)
            qp = _sel_tree(cont, qp_n, qp)
            premult = _sel_tree(cont, pm_n, premult)
            schur = _sel_tree(cont, sc_n, schur)
            num_iter = torch.where(cont, num_iter + 1, num_iter)
            conv_err = torch.where(cont, err, conv_err)
        nan = torch.isnan(states).any(dim=(-2, -1)) | torch.isnan(controls).any(dim=(-2, -1))
        status = torch.where(nan | (conv_err > tol), ERROR, SUCCESS).to(torch.int64)
        return SQPSolution(
            torch.nan_to_num(states),
            torch.nan_to_num(controls),
            torch.nan_to_num(dual),
            qp,
            premult,
            schur,
            status,
            num_iter,
            conv_err,
            conv_errs,
            alphas_rec,
            pcg_iters,
            guess.dual_backward_guess,
        )

    # -- backward (sqp.py:605-798) ---------------------------------------------------
    def mixed_derivatives(self, weights, states, controls, lambdas, tp):
        """Per weight key: f_dx_theta, f_du_theta, g_dx_theta^lambda, g_du_theta^lambda, g_theta."""
        prog = self.program

        def one(w, x, u, lam, p):
            def params_of(ww):
                q = dict(p)
                q.update(ww)
                return q

            def cost_grad(ww):
                return grad(lambda xx, uu: prog.cost(xx, uu, params_of(ww)), argnums=(0, 1))(x, u)

            def constraints(ww):
                return prog.equality_constraints(x, u, params_of(ww))

            def weighted_dz(ww):
                return jacfwd(
                    lambda xx, uu: lam.reshape(-1) @ prog.equality_constraints(xx, uu, params_of(ww)),
                    argnums=(0, 1),
                )(x, u)

            f_dx, f_du = jacfwd(cost_grad)(w)
            g = jacfwd(constraints)(w)
            gw_dx, gw_du = jacfwd(weighted_dz)(w)
            return f_dx, f_du, gw_dx, gw_du, g

        return vmap(one)(weights, states, controls, lambdas, tp)

    def solve_bwd(self, solution, weights, problem_params, dl_dstates, dl_dcontrols, dual_backward_guess):
        """Returns ``(dL/dtheta dict, dual_backward)`` (sqp.py:668-765)."""
        if not self.params["warm_start_backward"]:
            dual_backward_guess = torch.zeros_like(solution.dual)
        qp = solution.qp_parameters
        qs = -dl_dstates
        rs = -dl_dcontrols[:, :-1]
        cost_qp = P.QPCostParameters(qp.cost.Qinv, qs, qp.cost.Rinv, rs)
        qp2 = P.QPParameters(qp.dynamics, cost_qp)
        gam = P.compute_gamma(
            solution.dynamics_cost_premultiplied_matrices,
            torch.zeros_like(qp.dynamics.Cs),
            cost_qp.Qinv[:, 0],
            qs,
            rs,
        )
        lin, dbg = self.pcg.solve_KKT_Schur(
            qp2, solution.schur_complement_matrices, gam, dual_backward_guess
        )
        tp = self._tensor_params(self.make_params_with_weights(weights, problem_params))
        tp = {k: v.detach() for k, v in tp.items()}
        w = {k: torch.as_tensor(v, dtype=torch.float64).detach() for k, v in weights.items()}
        f_dx, f_du, gw_dx, gw_du, g = self.mixed_derivatives(
            w, solution.states, solution.controls, solution.dual, tp
        )
        xt, ut, lt = lin.states, lin.controls, lin.kkt_multipliers.reshape(lin.kkt_multipliers.shape[0], -1)
        out = {}
        for k in w:
            wdims = w[k].dim() - 1
            ex = lambda a, v: a * v.reshape(v.shape + (1,) * wdims)  # noqa: E731
            tx = ex(f_dx[k] + gw_dx[k], xt).sum(dim=(1, 2))
            tu = ex(f_du[k] + gw_du[k], ut).sum(dim=(1, 2))
            tg = ex(g[k], lt).sum(dim=1)
            out[k] = -(tx + tu + tg)
        return out, lin.kkt_multipliers, dbg.num_iterations

    # -- differentiable solve -----------------------------------------------------
    def solve(self, guess, problem_params, weights=None):
        """Forward solve whose outputs carry gradients to ``weights`` (custom VJP)."""
        weights = weights or {}
        keys = list(weights.keys())
        vals = [torch.as_tensor(weights[k], dtype=torch.float64) for k in keys]
        holder = []
        states, controls, dual, dbg_out = _SolveFn.apply(
            self, guess, problem_params, keys, holder, guess.dual_backward_guess, *vals
        )
        sol = holder[0]
        return sol._replace(states=states, controls=controls, dual=dual, dual_backward_guess=dbg_out)


class _SolveFn(torch.autograd.Function):
    """custom_vjp pairing of ``_solve`` and ``_solve_bwd`` (sqp.py:572-802)."""

    @staticmethod
    def forward(ctx, solver, guess, problem_params, keys, holder, dbg, *vals):
        weights = dict(zip(keys, [v.detach() for v in vals]))
        sol = solver._solve(guess, problem_params, weights)
        ctx.solver = solver
        ctx.sol = sol
        ctx.keys = keys
        ctx.weights = weights
        ctx.problem_params = problem_params
        holder.append(sol)
        return sol.states.clone(), sol.controls.clone(), sol.dual.clone(), dbg.detach().clone()

    @staticmethod
    def backward(ctx, g_states, g_controls, g_dual, g_dbg):
        solver = ctx.solver
        if g_states is None:
            g_states = torch.zeros_like(ctx.sol.states)
        if g_controls is None:
            g_controls = torch.zeros_like(ctx.sol.controls)
        if g_dbg is None:
            g_dbg = torch.zeros_like(ctx.sol.dual)
        grads, dual_bwd, _ = solver.solve_bwd(
            ctx.sol, ctx.weights, ctx.problem_params, g_states, g_controls, g_dbg
        )
        return (None, None, None, None, None, dual_bwd) + tuple(grads[k] for k in ctx.keys)
