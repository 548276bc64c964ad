"""PCG-level API on the GPU: the assertions of the reference's
tests/test_solver_pcg.py plus parity with the oracle's restatement of pcg.py."""

import numpy as np
import pytest
import torch

from diffmpc_b200 import (
    PCGOptimalControl,
    QPCostParameters,
    QPDynamicsCostPremultipliedMatrices,
    QPDynamicsParameters,
    QPParameters,
)
from oracle import pcg as OP
from tests.oracle_util import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"
F64 = torch.float64


def test_constructor_and_properties():
    solver_params = {"max_iter": 50, "tol_epsilon": 1e-5}
    oc = PCGOptimalControl(10, 4, 2, solver_params)
    assert oc.name == "PCGOptimalControl"
    assert (oc.horizon, oc.num_states, oc.num_controls) == (10, 4, 2)
    assert oc.params == solver_params


def test_zero_shapes():
    oc = PCGOptimalControl(5, 3, 2)
    qp = oc.zero_qp_parameters()
    assert qp.dynamics.As_next.shape == (5, 3, 3) and qp.dynamics.Bs.shape == (5, 3, 2)
    assert qp.dynamics.Cs.shape == (6, 3) and qp.cost.Qinv.shape == (6, 3, 3)
    assert qp.cost.Rinv.shape == (5, 2, 2) and qp.cost.rvec.shape == (5, 2)
    oc = PCGOptimalControl(4, 2, 1)
    assert oc.zero_dynamics_cost_premultiplied_matrices().Bs_x_Rinv.shape == (4, 2, 1)
    assert oc.zero_schur_complement_matrices().S.shape == (5, 2, 6)


def _identity_qp(T, nx, nu):
    eye = lambda n: torch.eye(n, dtype=F64, device=DEV)  # noqa: E731
    return QPParameters(
        QPDynamicsParameters(
            As_next=eye(nx).expand(T, nx, nx), As=eye(nx).expand(T, nx, nx),
            Bs=torch.ones(T, nx, nu, dtype=F64, device=DEV), Cs=torch.ones(T, nx, dtype=F64, device=DEV),
        ),
        QPCostParameters(
            Qinv=eye(nx).repeat(T + 1, 1, 1), qvec=torch.zeros(T + 1, nx, dtype=F64, device=DEV),
            Rinv=eye(nu).repeat(T, 1, 1), rvec=torch.zeros(T, nu, dtype=F64, device=DEV),
        ),
    )


@pytest.mark.parametrize("T", [2, 5])
@pytest.mark.parametrize("nx", [1, 5])
@pytest.mark.parametrize("nu", [1, 5])
def test_compute_S_Phiinv_identity_dynamics(T, nx, nu):
    oc = PCGOptimalControl(T, nx, nu, {"max_iter": 10, "tol_epsilon": 1e-8})
    schur = oc.compute_S_Phiinv(_identity_qp(T, nx, nu))
    assert schur.S.shape == (T + 1, nx, 3 * nx)
    assert schur.preconditioner_Phiinv.shape[0] == T + 1
    assert not torch.isnan(schur.S).any()


@pytest.mark.parametrize("T", [2, 5])
@pytest.mark.parametrize("nx", [1, 5])
@pytest.mark.parametrize("nu", [1, 5])
def test_compute_gamma_zeros(T, nx, nu):
    oc = PCGOptimalControl(T, nx, nu)
    dyn_cost = oc.zero_dynamics_cost_premultiplied_matrices()
    z = lambda *s: torch.zeros(*s, dtype=F64, device=DEV)  # noqa: E731
    gamma = oc.compute_gamma(dyn_cost, z(T + 1, nx), torch.eye(nx, dtype=F64, device=DEV), z(T + 1, nx), z(T, nu))
    assert gamma.shape == (T + 1, nx)
    assert torch.allclose(gamma, z(T + 1, nx))


@pytest.mark.parametrize("T", [2, 5])
@pytest.mark.parametrize("nx", [1, 5])
@pytest.mark.parametrize("nu", [1, 5])
def test_get_states_controls_from_zero_multipliers(T, nx, nu):
    oc = PCGOptimalControl(T, nx, nu)
    og = oc.zero_qp_parameters()
    qp = QPParameters(
        og.dynamics,
        QPCostParameters(
            Qinv=torch.eye(nx, dtype=F64, device=DEV).repeat(T + 1, 1, 1), qvec=torch.zeros(T + 1, 1, dtype=F64, device=DEV),
            Rinv=torch.eye(nu, dtype=F64, device=DEV).repeat(T, 1, 1), rvec=torch.zeros(T, 1, dtype=F64, device=DEV),
        ),
    )
    sol = oc.get_states_controls_from_kkt_multipliers(torch.zeros(T + 1, nx, dtype=F64, device=DEV), qp)
    assert sol.states.shape == (T + 1, nx) and sol.controls.shape == (T + 1, nu)
    assert torch.allclose(sol.states, torch.zeros_like(sol.states))
    assert torch.allclose(sol.controls, torch.zeros_like(sol.controls))


@pytest.mark.parametrize("T", [2, 3])
@pytest.mark.parametrize("nx", [1, 2])
@pytest.mark.parametrize("nu", [1, 2])
def test_solve_KKT_Schur_trivial(T, nx, nu):
    oc = PCGOptimalControl(T, nx, nu, {"max_iter": 10, "tol_epsilon": 1e-8})
    qp = _identity_qp(T, nx, nu)
    schur = oc.compute_S_Phiinv(qp)
    dyn_cost = oc.zero_dynamics_cost_premultiplied_matrices()
    z = lambda *s: torch.zeros(*s, dtype=F64, device=DEV)  # noqa: E731
    gammas = oc.compute_gamma(dyn_cost, torch.ones(T + 1, nx, dtype=F64, device=DEV),
                              torch.eye(nx, dtype=F64, device=DEV), z(T + 1, nx), z(T, nu))
    sol, debug = oc.solve_KKT_Schur(qp, schur, gammas, z(T + 1, nx))
    assert sol.states.shape == (T + 1, nx) and sol.controls.shape == (T + 1, nu)
    assert int(debug.num_iterations) <= 10
    assert float(debug.convergence_eta) >= 0.0


def test_solve_KKT_Schur_warmstart():
    T, nx, nu = 3, 4, 5
    np.random.seed(0)
    oc = PCGOptimalControl(T, nx, nu, {"max_iter": 20, "tol_epsilon": 1e-13})
    d = lambda v: torch.diag(torch.tensor(v, dtype=F64, device=DEV))  # noqa: E731
    qp = QPParameters(
        QPDynamicsParameters(
            As=d(np.random.rand(nx)).expand(T, nx, nx), As_next=d(np.random.rand(nx)).expand(T, nx, nx),
            Bs=torch.ones(T, nx, nu, dtype=F64, device=DEV), Cs=torch.ones(T, nx, dtype=F64, device=DEV),
        ),
        QPCostParameters(
            Qinv=d(np.random.rand(nx)).repeat(T + 1, 1, 1), qvec=torch.zeros(T + 1, nx, dtype=F64, device=DEV),
            Rinv=torch.eye(nu, dtype=F64, device=DEV).repeat(T, 1, 1), rvec=torch.zeros(T, nu, dtype=F64, device=DEV),
        ),
    )
    schur = oc.compute_S_Phiinv(qp)
    z = lambda *s: torch.zeros(*s, dtype=F64, device=DEV)  # noqa: E731
    gammas = oc.compute_gamma(oc.zero_dynamics_cost_premultiplied_matrices(), torch.ones(T + 1, nx, dtype=F64, device=DEV),
                              torch.eye(nx, dtype=F64, device=DEV), z(T + 1, nx), z(T, nu))
    sol, dbg = oc.solve_KKT_Schur(qp, schur, gammas, z(T + 1, nx))
    assert int(dbg.num_iterations) <= 10
    sol_w, dbg_w = oc.solve_KKT_Schur(qp, schur, gammas, sol.kkt_multipliers)
    assert torch.allclose(sol.states - sol_w.states, z(T + 1, nx))
    assert torch.allclose(sol.controls - sol_w.controls, z(T + 1, nu))
    assert torch.allclose(sol.kkt_multipliers - sol_w.kkt_multipliers, z(T + 1, nx))
    assert int(dbg_w.num_iterations) < int(dbg.num_iterations)


def _random_qp(B, T, nx, nu, seed):
    g = torch.Generator().manual_seed(seed)
    r = lambda *s: torch.randn(*s, generator=g, dtype=F64)  # noqa: E731
    A = torch.eye(nx, dtype=F64) + 0.2 * r(B, T, nx, nx)
    An = -torch.eye(nx, dtype=F64).expand(B, T, nx, nx) + 0.05 * r(B, T, nx, nx)
    Bm = 0.5 * r(B, T, nx, nu)
    M = r(B, T + 1, nx, nx)
    Q = M @ M.mT + nx * torch.eye(nx, dtype=F64)
    Mr = r(B, T, nu, nu)
    R = Mr @ Mr.mT + nu * torch.eye(nu, dtype=F64)
    qp = OP.QPParameters(
        OP.QPDynamicsParameters(An, A, Bm, r(B, T + 1, nx)),
        OP.QPCostParameters(torch.linalg.inv(Q), r(B, T + 1, nx), torch.linalg.inv(R), r(B, T, nu)),
    )
    return qp


def _to(qp, dev):
    return QPParameters(
        QPDynamicsParameters(*[t.to(dev) for t in qp.dynamics]), QPCostParameters(*[t.to(dev) for t in qp.cost])
    )


@pytest.mark.parametrize("T,nx,nu", [(5, 3, 2), (12, 13, 4), (20, 6, 3)])
def test_pcg_api_matches_oracle(T, nx, nu):
    B = 3
    qp = _random_qp(B, T, nx, nu, seed=T * 100 + nx)
    oschur = OP.compute_S_Phiinv(qp)
    opm = OP.premultiplied_matrices(qp)
    ogam = OP.compute_gamma(opm, qp.dynamics.Cs, qp.cost.Qinv[:, 0], qp.cost.qvec, qp.cost.rvec)
    osol, odbg = OP.solve_KKT_Schur(qp, oschur, ogam, torch.zeros(B, T + 1, nx, dtype=F64), 10000, 1e-20)

    oc = PCGOptimalControl(T, nx, nu, {"max_iter": 10000, "tol_epsilon": 1e-20})
    gqp = _to(qp, DEV)
    schur = oc.compute_S_Phiinv(gqp)
    assert rel_err(schur.S, oschur.S) < 1e-13
    assert rel_err(schur.preconditioner_Phiinv, oschur.preconditioner_Phiinv) < 1e-11
    pm = QPDynamicsCostPremultipliedMatrices(*[t.to(DEV) for t in opm])
    gam = oc.compute_gamma(pm, gqp.dynamics.Cs, gqp.cost.Qinv[:, 0], gqp.cost.qvec, gqp.cost.rvec)
    assert rel_err(gam, ogam) < 1e-13
    sol, dbg = oc.solve_KKT_Schur(gqp, schur, gam, torch.zeros(B, T + 1, nx, dtype=F64, device=DEV))
    assert rel_err(sol.kkt_multipliers, osol.kkt_multipliers) < 1e-9
    assert rel_err(sol.states, osol.states) < 1e-9
    assert rel_err(sol.controls, osol.controls) < 1e-9
    assert (dbg.num_iterations.cpu().long() - odbg.num_iterations).abs().max() <= 1
    rec = oc.get_states_controls_from_kkt_multipliers(osol.kkt_multipliers.to(DEV), gqp)
    assert rel_err(rec.states, osol.states) < 1e-12 and rel_err(rec.controls, osol.controls) < 1e-12
