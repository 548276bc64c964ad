"""Schur-complement PCG restatement (oracle, float64, batched).

Follows diffmpc/solvers/pcg.py.  Every function takes tensors with a leading
batch dimension ``B``; the PCG ``while_loop`` (pcg.py:397-436) runs until no
lane is active and freezes finished lanes with a select, which is what
``jax.vmap`` of ``lax.while_loop`` does.  Per-lane results therefore equal the
unbatched reference.
"""

from typing import NamedTuple

import torch


class QPDynamicsParameters(NamedTuple):  # pcg.py:13-20
    As_next: torch.Tensor  # (B, N, nx, nx)
    As: torch.Tensor  # (B, N, nx, nx)
    Bs: torch.Tensor  # (B, N, nx, nu)
    Cs: torch.Tensor  # (B, N+1, nx)


class QPCostParameters(NamedTuple):  # pcg.py:23-30
    Qinv: torch.Tensor  # (B, N+1, nx, nx)
    qvec: torch.Tensor  # (B, N+1, nx)
    Rinv: torch.Tensor  # (B, N, nu, nu)
    rvec: torch.Tensor  # (B, N, nu)


class QPParameters(NamedTuple):  # pcg.py:33-37
    dynamics: QPDynamicsParameters
    cost: QPCostParameters


class QPSolution(NamedTuple):  # pcg.py:40-46
    states: torch.Tensor  # (B, N+1, nx)
    controls: torch.Tensor  # (B, N+1, nu), last row zero
    kkt_multipliers: torch.Tensor  # (B, N+1, nx)


class QPDynamicsCostPremultipliedMatrices(NamedTuple):  # pcg.py:49-52
    As_x_Qinv: torch.Tensor
    Asnext_x_Qinvnext: torch.Tensor
    Bs_x_Rinv: torch.Tensor


class SchurComplementMatrices(NamedTuple):  # pcg.py:55-60
    S: torch.Tensor  # (B, N+1, nx, 3 nx)
    preconditioner_Phiinv: torch.Tensor  # (B, N+1, nx, 3 nx)


class PCGDebugOutput(NamedTuple):  # pcg.py:63-67
    num_iterations: torch.Tensor  # (B,) int64
    convergence_eta: torch.Tensor  # (B,)


def _shift3(v):
    """``[v_{t-1}, v_t, v_{t+1}]`` with zero padding, concatenated on the last axis."""
    z = torch.zeros_like(v[..., :1, :])
    prev = torch.cat([z, v[..., :-1, :]], dim=-2)
    nxt = torch.cat([v[..., 1:, :], z], dim=-2)
    return torch.cat([prev, v, nxt], dim=-1)


def block_tridiag_matvec(M, v):
    """Row-block stencil product used for ``S p`` and ``Phi^-1 r`` (pcg.py:384-392)."""
    return torch.einsum("...tij,...tj->...ti", M, _shift3(v))


def premultiplied_matrices(qp):
    """``A Qinv[:-1]``, ``A_next Qinv[1:]``, ``B Rinv`` (sqp.py:247-254)."""
    Qinv = qp.cost.Qinv
    return QPDynamicsCostPremultipliedMatrices(
        qp.dynamics.As @ Qinv[..., :-1, :, :],
        qp.dynamics.As_next @ Qinv[..., 1:, :, :],
        qp.dynamics.Bs @ qp.cost.Rinv,
    )


def compute_S_Phiinv(qp):
    """S and the block-tridiagonal preconditioner Phi^-1 (pcg.py:160-243)."""
    As_next, As, Bs = qp.dynamics.As_next, qp.dynamics.As, qp.dynamics.Bs
    Qinv, Rinv = qp.cost.Qinv, qp.cost.Rinv
    nx = As.shape[-1]
    eye = torch.eye(nx, dtype=As.dtype).expand(*As.shape[:-3], 1, nx, nx)
    As_next_prev = torch.cat([eye, As_next[..., :-1, :, :]], dim=-3)
    A_Qinv = As @ Qinv[..., :-1, :, :]
    An_Qinvn = As_next @ Qinv[..., 1:, :, :]
    B_Rinv = Bs @ Rinv
    thetas = A_Qinv @ As.mT + B_Rinv @ Bs.mT + An_Qinvn @ As_next.mT
    phis = A_Qinv @ As_next_prev.mT
    thetas = torch.cat([Qinv[..., :1, :, :], thetas], dim=-3)
    thetas_inv = torch.linalg.inv(thetas)
    zero = torch.zeros_like(thetas[..., :1, :, :])
    phis_p = torch.cat([zero, phis, zero], dim=-3)
    S = -torch.cat([phis_p[..., :-1, :, :], thetas, phis_p[..., 1:, :, :].mT], dim=-1)
    thinv_p = torch.cat([zero, thetas_inv, zero], dim=-3)
    prev = -thetas_inv @ phis_p[..., :-1, :, :] @ thinv_p[..., :-2, :, :]
    nxt = -thetas_inv @ phis_p[..., 1:, :, :].mT @ thinv_p[..., 2:, :, :]
    Phiinv = torch.cat([prev, thetas_inv, nxt], dim=-1)
    return SchurComplementMatrices(S, Phiinv)


def compute_gamma(premult, Cs, Q0inv, qs, rs):
    """``gamma = C + [Q0^-1 q0; zeta]`` (pcg.py:245-288)."""
    mv = lambda M, v: torch.einsum("...ij,...j->...i", M, v)  # noqa: E731
    zetas = mv(premult.As_x_Qinv, qs[..., :-1, :]) + mv(premult.Bs_x_Rinv, rs) + mv(
        premult.Asnext_x_Qinvnext, qs[..., 1:, :]
    )
    g0 = mv(Q0inv, qs[..., 0, :])
    return Cs + torch.cat([g0[..., None, :], zetas], dim=-2)


def get_states_controls_from_kkt_multipliers(lambdas, qp):
    """``x = -Qinv (q + G_x^T lambda)``, ``u = -Rinv (r + B^T lambda_next)``, u_N = 0 (pcg.py:290-348)."""
    As_next, As, Bs = qp.dynamics.As_next, qp.dynamics.As, qp.dynamics.Bs
    Qinv, q, Rinv, r = qp.cost.Qinv, qp.cost.qvec, qp.cost.Rinv, qp.cost.rvec
    nx, nu = As.shape[-1], Bs.shape[-1]
    mv = lambda M, v: torch.einsum("...ij,...j->...i", M, v)  # noqa: E731
    eye = torch.eye(nx, dtype=As.dtype).expand(*As.shape[:-3], 1, nx, nx)
    An_shift = torch.cat([eye, As_next[..., :-1, :, :]], dim=-3)
    lam, lam_next = lambdas[..., :-1, :], lambdas[..., 1:, :]
    states = -mv(Qinv[..., :-1, :, :], q[..., :-1, :] + mv(An_shift.mT, lam) + mv(As.mT, lam_next))
    controls = -mv(Rinv, r + mv(Bs.mT, lam_next))
    xN = -mv(Qinv[..., -1, :, :], q[..., -1, :] + mv(As_next[..., -1, :, :].mT, lambdas[..., -1, :]))
    states = torch.cat([states, xN[..., None, :]], dim=-2)
    controls = torch.cat([controls, torch.zeros_like(controls[..., :1, :])], dim=-2)
    return QPSolution(states, controls, lambdas)


def _sel(mask, new, old):
    m = mask.reshape(mask.shape + (1,) * (new.dim() - mask.dim()))
    return torch.where(m, new, old)


def solve_KKT_Schur(qp, schur, gammas, lambdas_guess, max_iter, tol_epsilon):
    """PCG on ``S lambda = gamma`` (pcg.py:350-445), batched.

    Stopping rule (pcg.py:397-403): continue while
    ``(|eta| > eps and it <= max_iter - 1) or it < 1``.
    """
    S, Phiinv = schur.S, schur.preconditioner_Phiinv
    lambs = lambdas_guess
    r = gammas - block_tridiag_matvec(S, lambs)
    rt = block_tridiag_matvec(Phiinv, r)
    p = rt.clone()
    eta = torch.sum(r * rt, dim=(-2, -1))
    it = torch.zeros(eta.shape, dtype=torch.int64)
    while True:
        cont = ((eta.abs() > tol_epsilon) & (it <= max_iter - 1)) | (it < 1)
        if not bool(cont.any()):
            break
        ups = block_tridiag_matvec(S, p)
        v = torch.sum(p * ups, dim=(-2, -1))
        alpha = eta / v
        lambs_n = lambs + alpha[..., None, None] * p
        r_n = r - alpha[..., None, None] * ups
        rt_n = block_tridiag_matvec(Phiinv, r_n)
        etap = torch.sum(r_n * rt_n, dim=(-2, -1))
        beta = etap / eta
        p_n = rt_n + beta[..., None, None] * p
        it = torch.where(cont, it + 1, it)
        r = _sel(cont, r_n, r)
        p = _sel(cont, p_n, p)
        eta = torch.where(cont, etap, eta)
        lambs = _sel(cont, lambs_n, lambs)
    sol = get_states_controls_from_kkt_multipliers(lambs, qp)
    return sol, PCGDebugOutput(it, eta)


class PCGOptimalControl:
    """Mirror of PCGOptimalControl's constructor/properties (pcg.py:70-158)."""

    def __init__(self, horizon, num_states, num_controls, solver_params=None):
        if solver_params is None:
            solver_params = {"verbose": False, "max_iter": 10000, "tol_epsilon": 1e-9}
        self._params = solver_params
        self.name = "PCGOptimalControl"
        self.horizon = horizon
        self.num_states = num_states
        self.num_controls = num_controls

    @property
    def params(self):
        return self._params

    def zero_qp_parameters(self, batch=()):
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        z = lambda *s: torch.zeros(*batch, *s, dtype=torch.float64)  # noqa: E731
        return QPParameters(
            QPDynamicsParameters(z(N, nx, nx), z(N, nx, nx), z(N, nx, nu), z(N + 1, nx)),
            QPCostParameters(z(N + 1, nx, nx), z(N + 1, nx), z(N, nu, nu), z(N, nu)),
        )

    def zero_dynamics_cost_premultiplied_matrices(self, batch=()):
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        z = lambda *s: torch.zeros(*batch, *s, dtype=torch.float64)  # noqa: E731
        return QPDynamicsCostPremultipliedMatrices(z(N, nx, nx), z(N, nx, nx), z(N, nx, nu))

    def zero_schur_complement_matrices(self, batch=()):
        N, nx = self.horizon, self.num_states
        z = lambda *s: torch.zeros(*batch, *s, dtype=torch.float64)  # noqa: E731
        return SchurComplementMatrices(z(N + 1, nx, 3 * nx), z(N + 1, nx, 3 * nx))

    def compute_S_Phiinv(self, qp):
        return compute_S_Phiinv(qp)

    def compute_gamma(self, premult, Cs, Q0inv, qs, rs):
        return compute_gamma(premult, Cs, Q0inv, qs, rs)

    def get_states_controls_from_kkt_multipliers(self, kkt_multipliers, qp):
        return get_states_controls_from_kkt_multipliers(kkt_multipliers, qp)

    def solve_KKT_Schur(self, qp, schur, gammas, lambdas_guess):
        return solve_KKT_Schur(
            qp, schur, gammas, lambdas_guess, self.params["max_iter"], self.params["tol_epsilon"]
        )
