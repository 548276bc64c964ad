"""Seeded synthetic workloads for the benchmark and parity cases.

Each builder returns ``(dynamics, static_params, batched_params, solver_params)``:
``static_params`` is a parameter dict valid for ``OptimalControlProblem``
(instance 0's values), ``batched_params`` holds every per-instance value with a
leading batch dimension (float64, CPU tensors), ``solver_params`` follows
``params/sqp.yaml``.  Random draws use ``numpy.random.default_rng(seed)``.

Workloads (the reference's ``horizon`` N; K = N + 1 knots):

* ``linear_lti``      nx=6, nu=3, N=20, B=1, Euler dt=1 (the discrete A is I + A_c)
* ``attitude``        spacecraft attitude nx=7, nu=3, N=50, dt=0.1, B=1024, 10 SQP
* ``quadrotor``       nx=13, nu=4, N=60, RK4 dt=0.05, B=4096, loss = sum u_0^2
* ``mixed_uneven``    50% linear nx=12 / 50% quadrotor, N ~ U{20..100}, B=8192
* ``linear_stress``   nx=24, nu=8, N=128, diag Q with log10 entries ~ U[-3,3], B=16384
"""

import copy
import math

import numpy as np
import torch

from .dynamics import LinearDynamics, QuadrotorDynamics, SpacecraftAttitudeDynamics, SpacecraftDynamics
from .problem import load_solver_params

F64 = torch.float64


def _t(a):
    return torch.as_tensor(np.asarray(a), dtype=F64)


def random_stable_linear(rng, B, nx, nu, rho_max=1.05):
    """A_d = I + 0.1 N(0,1)/sqrt(nx) rescaled to spectral radius <= rho_max; B = 0.1 N(0,1).

    With Euler and dt = 1 the continuous-time A of ``x_dot = A x + B u`` is A_d - I.
    """
    Ad = np.eye(nx)[None] + 0.1 * rng.standard_normal((B, nx, nx)) / math.sqrt(nx)
    rho = np.abs(np.linalg.eigvals(Ad)).max(axis=-1)
    scale = np.where(rho > rho_max, rho_max / rho, 1.0)
    Ad = Ad * scale[:, None, None]
    Bm = 0.1 * rng.standard_normal((B, nx, nu))
    return Ad - np.eye(nx)[None], Bm


def _unit_quat(rng, B):
    q = rng.standard_normal((B, 4))
    return q / np.linalg.norm(q, axis=-1, keepdims=True)


def _base(N, dt, scheme, x0, xf, xref, uref, wx, wu, wf, pen, extra):
    p = {
        "horizon": N,
        "discretization_resolution": _t(dt),
        "discretization_scheme": scheme,
        "initial_state": _t(x0),
        "final_state": _t(xf),
        "reference_state_trajectory": _t(xref),
        "reference_control_trajectory": _t(uref),
        "penalize_control_reference": pen,
        "weights_penalization_reference_state_trajectory": _t(wx),
        "weights_penalization_control_squared": _t(wu),
        "weights_penalization_final_state": _t(wf),
    }
    p.update({k: _t(v) for k, v in extra.items()})
    return p


def _static_of(batched):
    out = {}
    for k, v in batched.items():
        out[k] = v[0] if isinstance(v, torch.Tensor) and v.dim() > 0 else v
    return out


def linear_lti(B=1, seed=1000, nx=6, nu=3, N=20, wx=1.0, wu=0.1, wf=9.0, log10_wx=None):
    """Linear time-invariant MPC (Q = wx I, R = wu I, terminal (wx + wf) I)."""
    rng = np.random.default_rng(seed)
    A, Bm = random_stable_linear(rng, B, nx, nu)
    x0 = rng.standard_normal((B, nx))
    if log10_wx is not None:
        wxv = 10.0 ** rng.uniform(-log10_wx, log10_wx, size=(B, nx))
    else:
        wxv = np.full((B, nx), wx)
    K = N + 1
    batched = _base(
        N, np.ones(B), 0, x0, np.zeros((B, nx)), np.zeros((B, K, nx)), np.zeros((B, K, nu)),
        wxv, np.full((B, nu), wu), np.full((B, nx), wf), False,
        {"A": A, "B": Bm, "b": np.zeros((B, nx))},
    )
    dyn = LinearDynamics({
        "num_states": nx, "num_controls": nu,
        "names_states": [f"x{i}" for i in range(nx)], "names_controls": [f"u{i}" for i in range(nu)],
    })
    sp = load_solver_params("sqp.yaml")
    sp["pcg"]["tol_epsilon"] = 1e-10
    sp["num_scp_iteration_max"] = 2
    return dyn, _static_of(batched), batched, sp


def linear_stress(B=16384, seed=1004, nx=24, nu=8, N=128):
    dyn, st, bt, sp = linear_lti(B=B, seed=seed, nx=nx, nu=nu, N=N, wu=1e-2, wf=0.0, log10_wx=3.0)
    return dyn, st, bt, sp


def shrunk_stable_matrix(rng, nx, margin=1e-2):
    """I + 0.1 N(0,1) with every eigenvalue of modulus >= 1 - margin divided by
    (modulus + margin), so the spectrum lies strictly inside the unit circle
    (benchmarking/reinforcement-learning/utils.py:34-48 describes this construction)."""
    A = np.eye(nx) + 0.1 * rng.standard_normal((nx, nx))
    lam, V = np.linalg.eig(A)
    mod = np.abs(lam)
    lam = np.where(mod < 1.0 - margin, lam, lam / (mod + margin))
    return (V @ np.diag(lam) @ np.linalg.inv(V)).real


def rl_linear(B=1024, seed=1005, nx=8, nu=4, N=39, warm_start=True):
    """Closed-loop benchmark problem of the reference's reinforcement-learning scripts
    (benchmark_diffmpc.py:40-100, utils.py): one stable discrete system shared by the batch
    (A, B ~ N(0,1), b ~ 0.01 N(0,1)), x0 ~ 5 N(0,1), Q = I, R = I, no terminal weight, MPC
    horizon N = 39 (40 knots) with dt = 1 Euler, so the MPC model's continuous-time A is
    A - I; one SQP iteration with the line search at alpha = 1, PCG tolerance 1e-12.
    Returns (dynamics, static params, batched params, solver params, (A, B, b))."""
    rng = np.random.default_rng(seed)
    A = shrunk_stable_matrix(rng, nx)
    Bm = rng.standard_normal((nx, nu))
    b = 0.01 * rng.standard_normal(nx)
    x0 = 5.0 * rng.standard_normal((B, nx))
    K = N + 1
    tile = lambda a: np.repeat(a[None], B, axis=0)  # noqa: E731
    batched = _base(
        N, np.ones(B), 0, x0, np.zeros((B, nx)), np.zeros((B, K, nx)), np.zeros((B, K, nu)),
        np.ones((B, nx)), np.ones((B, nu)), np.zeros((B, nx)), False,
        {"A": tile(A - np.eye(nx)), "B": tile(Bm), "b": tile(b)},
    )
    dyn = LinearDynamics({
        "num_states": nx, "num_controls": nu,
        "names_states": [f"x{i}" for i in range(nx)], "names_controls": [f"u{i}" for i in range(nu)],
    })
    sp = load_solver_params("sqp.yaml")
    sp["num_scp_iteration_max"] = 1
    sp["pcg"]["tol_epsilon"] = 1e-12
    sp["warm_start_backward"] = bool(warm_start)
    sp["linesearch"] = True
    sp["linesearch_alphas"] = [1.0]
    return dyn, _static_of(batched), batched, sp, (_t(A), _t(Bm), _t(b))


def rl_spacecraft(B=16, seed=1006, N=39):
    """Closed-loop benchmark problem of the reference's spacecraft script
    (spacecraft/benchmark_diffmpc.py:30-60, spacecraft/utils.py): angular-rate spacecraft with
    one inertia vector shared by the batch, inertia ~ U[1, 10]^3, x0 ~ U[-0.1, 0.1]^3, the
    spacecraft.yaml weights (Q = I, R = I, dt = 0.1, Euler), zero references and terminal
    weight, horizon N = 39 (40 knots); one SQP iteration with the line search at alpha = 1,
    PCG tolerance 1e-12.  The rollout simulates with the model's own Euler step and the cost
    10 |x|^2 + |u|^2.  Returns (dynamics, static params, batched params, solver params)."""
    rng = np.random.default_rng(seed)
    J = 1.0 + 9.0 * rng.random(3)
    x0 = -0.1 + 0.2 * rng.random((B, 3))
    K = N + 1
    batched = _base(
        N, np.full(B, 0.1), 0, x0, np.zeros((B, 3)), np.zeros((B, K, 3)), np.zeros((B, K, 3)),
        np.ones((B, 3)), np.ones((B, 3)), np.zeros((B, 3)), False,
        {"inertia_vector": np.repeat(J[None], B, axis=0)},
    )
    sp = load_solver_params("sqp.yaml")
    sp["num_scp_iteration_max"] = 1
    sp["pcg"]["tol_epsilon"] = 1e-12
    sp["linesearch"] = True
    sp["linesearch_alphas"] = [1.0]
    return SpacecraftDynamics(), _static_of(batched), batched, sp


def attitude(B=1024, seed=1001, N=50):
    """Spacecraft attitude (quaternion + rate), random goal attitude."""
    rng = np.random.default_rng(seed)
    J = rng.uniform(1.0, 3.0, size=(B, 3))
    q0 = _unit_quat(rng, B)
    w0 = 0.1 * rng.standard_normal((B, 3))
    qg = _unit_quat(rng, B)
    x0 = np.concatenate([q0, w0], axis=1)
    xg = np.concatenate([qg, np.zeros((B, 3))], axis=1)
    K = N + 1
    batched = _base(
        N, np.full(B, 0.1), 0, x0, xg, np.repeat(xg[:, None], K, axis=1), np.zeros((B, K, 3)),
        np.tile([10.0, 10, 10, 10, 1, 1, 1], (B, 1)), np.full((B, 3), 0.01), np.zeros((B, 7)), False,
        {"inertia_vector": J},
    )
    sp = load_solver_params("sqp.yaml")
    sp["num_scp_iteration_max"] = 10
    sp["pcg"]["tol_epsilon"] = 1e-8
    return SpacecraftAttitudeDynamics(), _static_of(batched), batched, sp


def quadrotor(B=4096, seed=1002, N=60):
    """Quadrotor RK4 with random mass/inertia, perturbed hover start, random goal position."""
    rng = np.random.default_rng(seed)
    mass = rng.uniform(0.5, 1.5, size=(B, 1))
    Jd = rng.uniform(0.005, 0.02, size=(B, 3))
    inertia = np.zeros((B, 9))
    inertia[:, 0], inertia[:, 4], inertia[:, 8] = Jd[:, 0], Jd[:, 1], Jd[:, 2]
    hover = np.array([0.0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0])
    x0 = hover[None] + 0.3 * rng.standard_normal((B, 13))
    x0[:, 6:10] /= np.linalg.norm(x0[:, 6:10], axis=1, keepdims=True)
    goal = np.repeat(hover[None], B, axis=0)
    goal[:, :3] = rng.uniform(-2.0, 2.0, size=(B, 3))
    wx = np.exp(rng.uniform(-2.0, 2.0, size=(B, 13)))
    wu = np.exp(rng.uniform(-2.0, 2.0, size=(B, 4)))
    K = N + 1
    uref = np.zeros((B, K, 4))
    uref[:, :, 0] = mass * 9.81
    batched = _base(
        N, np.full(B, 0.05), 2, x0, goal, np.repeat(goal[:, None], K, axis=1), uref,
        wx, wu, np.zeros((B, 13)), True, {"mass": mass, "inertia": inertia},
    )
    sp = load_solver_params("sqp.yaml")
    return QuadrotorDynamics(), _static_of(batched), batched, sp


def subset(batched, idx):
    """Per-instance slice of a batched parameter dict (static keys kept)."""
    out = {}
    for k, v in batched.items():
        out[k] = v[idx] if isinstance(v, torch.Tensor) and v.dim() > 0 else v
    return out


def to_device(batched, device):
    return {k: (v.to(device) if isinstance(v, torch.Tensor) else v) for k, v in batched.items()}


def clone_params(p):
    return copy.copy(p)
