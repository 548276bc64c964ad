"""Schur-complement PCG front end (mirror of diffmpc/solvers/pcg.py).

Same NamedTuples, class name, constructor and methods as the reference; each
method runs one kernel of ``libdmpc.so`` on the reference's dense layouts
(``S``, ``Phi^-1`` as ``(N+1, nx, 3 nx)`` block rows).  Inputs may carry a
leading batch dimension; unbatched inputs give unbatched outputs.
"""

from typing import Any, Dict, NamedTuple, Tuple

import torch

from . import _lib

DEFAULT_PCG_SOLVER_PARAMS = {"verbose": False, "max_iter": 10000, "tol_epsilon": 1e-9}  # sqp.yaml pcg


class QPDynamicsParameters(NamedTuple):  # pcg.py:13-20
    As_next: torch.Tensor  # (N, nx, nx)
    As: torch.Tensor  # (N, nx, nx)
    Bs: torch.Tensor  # (N, nx, nu)
    Cs: torch.Tensor  # (N+1, nx)


class QPCostParameters(NamedTuple):  # pcg.py:23-30
    Qinv: torch.Tensor  # (N+1, nx, nx)
    qvec: torch.Tensor  # (N+1, nx)
    Rinv: torch.Tensor  # (N, nu, nu)
    rvec: torch.Tensor  # (N, nu)


class QPParameters(NamedTuple):  # pcg.py:33-37
    dynamics: QPDynamicsParameters
    cost: QPCostParameters


class QPSolution(NamedTuple):  # pcg.py:40-46
    states: torch.Tensor
    controls: torch.Tensor
    kkt_multipliers: torch.Tensor


class QPDynamicsCostPremultipliedMatrices(NamedTuple):  # pcg.py:49-52
    As_x_Qinv: torch.Tensor
    Asnext_x_Qinvnext: torch.Tensor
    Bs_x_Rinv: torch.Tensor


class SchurComplementMatrices(NamedTuple):  # pcg.py:55-60
    S: torch.Tensor
    preconditioner_Phiinv: torch.Tensor


class PCGDebugOutput(NamedTuple):  # pcg.py:63-67
    num_iterations: Any
    convergence_eta: Any


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


class PCGOptimalControl:
    """Mirror of PCGOptimalControl (pcg.py:70-445)."""

    def __init__(self, problem_horizon: int, problem_num_states: int, problem_num_controls: int,
                 solver_params: Dict[str, Any] = DEFAULT_PCG_SOLVER_PARAMS):
        self._params = solver_params
        self._name = "PCGOptimalControl"
        self._problem_horizon = problem_horizon
        self._problem_num_states = problem_num_states
        self._problem_num_controls = problem_num_controls

    @property
    def name(self) -> str:
        return self._name

    @property
    def params(self) -> Dict:
        return self._params

    @property
    def horizon(self) -> int:
        return self._problem_horizon

    @property
    def num_states(self) -> int:
        return self._problem_num_states

    @property
    def num_controls(self) -> int:
        return self._problem_num_controls

    # -- zeros (pcg.py:129-158) -----------------------------------------------
    def _z(self, *shape):
        return torch.zeros(*shape, dtype=torch.float64, device=_dev() if torch.cuda.is_available() else "cpu")

    def zero_qp_parameters(self):
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        z = self._z
        return QPParameters(
            QPDynamicsParameters(z(N, nx, nx), z(N, nx, nx), z(N, nx, nu), z(N + 1, nx)),
            QPCostParameters(z(N + 1, nx, nx), z(N + 1, nx), z(N, nu, nu), z(N, nu)),
        )

    def zero_dynamics_cost_premultiplied_matrices(self):
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        z = self._z
        return QPDynamicsCostPremultipliedMatrices(z(N, nx, nx), z(N, nx, nx), z(N, nx, nu))

    def zero_schur_complement_matrices(self):
        N, nx = self.horizon, self.num_states
        return SchurComplementMatrices(self._z(N + 1, nx, 3 * nx), self._z(N + 1, nx, 3 * nx))

    # -- helpers ---------------------------------------------------------------
    def _prep(self, tensors, unbatched_dims):
        """Returns (batched contiguous float64 CUDA tensors, B, was_unbatched)."""
        first = tensors[0]
        unb = first.dim() == unbatched_dims
        dev = first.device if first.is_cuda else _dev()
        out = []
        B = 1 if unb else first.shape[0]
        for t in tensors:
            t = torch.as_tensor(t, dtype=torch.float64, device=dev)
            if unb:
                t = t[None]
            elif t.shape[0] != B:
                t = t.expand(B, *t.shape[1:])
            out.append(t.contiguous())
        return out, B, unb

    def _qp_tensors(self, qp):
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        d, c = qp.dynamics, qp.cost
        rvec = torch.as_tensor(c.rvec).reshape(*c.rvec.shape[:-1], -1)
        qvec = torch.as_tensor(c.qvec)
        # the reference's tests pass (T+1, 1) / (T, 1) zero cost vectors; broadcast them
        qvec = qvec.expand(*qvec.shape[:-1], nx) if qvec.shape[-1] == 1 else qvec
        rvec = rvec.expand(*rvec.shape[:-1], nu) if rvec.shape[-1] == 1 else rvec
        return [d.As_next, d.As, d.Bs, d.Cs, c.Qinv, qvec, c.Rinv, rvec]

    # -- kernels ---------------------------------------------------------------
    def compute_S_Phiinv(self, qp_parameters: QPParameters) -> SchurComplementMatrices:
        """S and Phi^-1 (pcg.py:160-243) by dmpc_schur_assemble."""
        S, P, _ = self._assemble(qp_parameters)
        return SchurComplementMatrices(S=S, preconditioner_Phiinv=P)

    def _assemble(self, qp):
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        (An, A, Bm, C, Qi, q, Ri, r), B, unb = self._prep(self._qp_tensors(qp), 3)
        if C.shape[-2] != N + 1:  # tests may pass (N, nx) constraint vectors to compute_S_Phiinv
            C = torch.zeros(B, N + 1, nx, dtype=torch.float64, device=A.device)
        dev = A.device
        S = torch.empty(B, N + 1, nx, 3 * nx, dtype=torch.float64, device=dev)
        P = torch.empty_like(S)
        g = torch.empty(B, N + 1, nx, dtype=torch.float64, device=dev)
        lib = _lib.load()
        nws = lib.dmpc_schur_workspace_size(B, N, nx)
        ws = torch.empty(max(nws, 256), dtype=torch.uint8, device=dev)
        _lib.check(
            lib.dmpc_schur_assemble(
                B, N, nx, nu, An.data_ptr(), A.data_ptr(), Bm.data_ptr(), C.data_ptr(), Qi.data_ptr(),
                q.data_ptr(), Ri.data_ptr(), r.data_ptr(), S.data_ptr(), P.data_ptr(), g.data_ptr(),
                ws.data_ptr(), ws.numel(), _stream(dev),
            ),
            "dmpc_schur_assemble",
        )
        if unb:
            return S[0], P[0], g[0]
        return S, P, g

    def compute_gamma(self, dynamics_cost_premultiplied_matrices, Cs, Q0inv, qs, rs):
        """gamma = C + [Q0^-1 q0; zeta] (pcg.py:245-288) by dmpc_compute_gamma."""
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        pm = dynamics_cost_premultiplied_matrices
        (AQ, AnQ, BR), B, unb = self._prep([pm.As_x_Qinv, pm.Asnext_x_Qinvnext, pm.Bs_x_Rinv], 3)
        dev = AQ.device
        rest = []
        for t, ud in ((Cs, 2), (Q0inv, 2), (qs, 2), (rs, 2)):
            t = torch.as_tensor(t, dtype=torch.float64, device=dev)
            t = t[None] if (unb or t.dim() == ud) else t
            rest.append(t.expand(B, *t.shape[1:]).contiguous())
        C, Q0, q, r = rest
        g = torch.empty(B, N + 1, nx, dtype=torch.float64, device=dev)
        lib = _lib.load()
        _lib.check(
            lib.dmpc_compute_gamma(
                B, N, nx, nu, AQ.data_ptr(), AnQ.data_ptr(), BR.data_ptr(), C.data_ptr(), Q0.data_ptr(),
                q.data_ptr(), r.data_ptr(), g.data_ptr(), _stream(dev),
            ),
            "dmpc_compute_gamma",
        )
        return g[0] if unb else g

    def get_states_controls_from_kkt_multipliers(self, kkt_multipliers, qp_parameters) -> QPSolution:
        """(x, u) from lambda (pcg.py:290-348) by dmpc_kkt_recover; u_N = 0."""
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        lam_in = torch.as_tensor(kkt_multipliers, dtype=torch.float64)
        (lam, An, A, Bm, C, Qi, q, Ri, r), B, unb = self._prep([lam_in] + self._qp_tensors(qp_parameters), 2)
        dev = lam.device
        xs = torch.empty(B, N + 1, nx, dtype=torch.float64, device=dev)
        us = torch.empty(B, N + 1, nu, dtype=torch.float64, device=dev)
        lib = _lib.load()
        _lib.check(
            lib.dmpc_kkt_recover(
                B, N, nx, nu, lam.data_ptr(), An.data_ptr(), A.data_ptr(), Bm.data_ptr(), Qi.data_ptr(),
                q.data_ptr(), Ri.data_ptr(), r.data_ptr(), xs.data_ptr(), us.data_ptr(), _stream(dev),
            ),
            "dmpc_kkt_recover",
        )
        if unb:
            return QPSolution(xs[0], us[0], lam[0])
        return QPSolution(xs, us, lam)

    def solve_KKT_Schur(self, qp_parameters, schur_complement_matrices, schur_complement_gammas,
                        kkt_multipliers_guess) -> Tuple[QPSolution, PCGDebugOutput]:
        """FP64 PCG with the reference's stopping rule (pcg.py:350-445) by dmpc_pcg_solve."""
        N, nx, nu = self.horizon, self.num_states, self.num_controls
        sc = schur_complement_matrices
        (S, P, g, l0, An, A, Bm, C, Qi, q, Ri, r), B, unb = self._prep(
            [sc.S, sc.preconditioner_Phiinv, schur_complement_gammas, kkt_multipliers_guess]
            + self._qp_tensors(qp_parameters),
            3,
        )
        dev = S.device
        lam = torch.empty(B, N + 1, nx, dtype=torch.float64, device=dev)
        xs = torch.empty_like(lam)
        us = torch.empty(B, N + 1, nu, dtype=torch.float64, device=dev)
        it = torch.empty(B, dtype=torch.int32, device=dev)
        eta = torch.empty(B, dtype=torch.float64, device=dev)
        lib = _lib.load()
        _lib.check(
            lib.dmpc_pcg_solve(
                B, N, nx, nu, S.data_ptr(), P.data_ptr(), g.data_ptr(), l0.data_ptr(), An.data_ptr(), A.data_ptr(),
                Bm.data_ptr(), Qi.data_ptr(), q.data_ptr(), Ri.data_ptr(), r.data_ptr(),
                int(self.params["max_iter"]), float(self.params["tol_epsilon"]),
                lam.data_ptr(), xs.data_ptr(), us.data_ptr(), it.data_ptr(), eta.data_ptr(), _stream(dev),
            ),
            "dmpc_pcg_solve",
        )
        if unb:
            return QPSolution(xs[0], us[0], lam[0]), PCGDebugOutput(it[0], eta[0])
        return QPSolution(xs, us, lam), PCGDebugOutput(it, eta)
