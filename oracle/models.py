"""Continuous-time dynamics ``state_dot(x, u, params)`` (oracle, float64).

Each function takes one instance (``x`` of shape ``(nx,)``, ``u`` of shape
``(nu,)``) and a dict of that instance's parameters, and is written with
plain torch ops so that ``torch.func`` transforms (jvp/jacfwd/vmap) apply,
mirroring how the reference differentiates its JAX ``state_dot``.
"""

import torch

GRAVITY = 9.81  # quadrotor_dynamics.py:112


def _cat(xs):
    return torch.cat([x.reshape(-1) for x in xs])


def linear_state_dot(x, u, p):
    """``x_dot = A x + B u + b`` (linear_dynamics.py:69)."""
    return p["A"] @ x + p["B"] @ u + p["b"]


def _skew(a):
    """Skew matrix with ``S(a) b = a x b`` (quadrotor_dynamics.py:35-36)."""
    z = torch.zeros((), dtype=a.dtype)
    return torch.stack(
        [
            torch.stack([z, -a[2], a[1]]),
            torch.stack([a[2], z, -a[0]]),
            torch.stack([-a[1], a[0], z]),
        ]
    )


def _q_left(q):
    """Left quaternion-product matrix, scalar first (quadrotor_dynamics.py:40-48)."""
    w, x, y, z = q[0], q[1], q[2], q[3]
    return torch.stack(
        [
            torch.stack([w, -x, -y, -z]),
            torch.stack([x, w, -z, y]),
            torch.stack([y, z, w, -x]),
            torch.stack([z, -y, x, w]),
        ]
    )


def _rotation(q):
    """Rotation matrix of a unit quaternion (quadrotor_dynamics.py:57-69)."""
    qw, qx, qy, qz = q[0], q[1], q[2], q[3]
    qw2, qx2, qy2, qz2 = qw * qw, qx * qx, qy * qy, qz * qz
    return torch.stack(
        [
            torch.stack([qw2 + qx2 - qy2 - qz2, 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)]),
            torch.stack([2 * (qx * qy + qw * qz), qw2 - qx2 + qy2 - qz2, 2 * (qy * qz - qw * qx)]),
            torch.stack([2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), qw2 - qx2 - qy2 + qz2]),
        ]
    )


def quadrotor_state_dot(x, u, p):
    """13-state quadrotor ``[p, v, q, w]`` with controls ``[thrust, tau]``.

    Follows quadrotor_dynamics.py:84-133: the 3x3 inertia comes from the
    9-vector key ``"inertia"`` and is inverted on every call, the quaternion
    is normalised inside ``state_dot``, ``v_dot = -g e3 + (f/m) R e3``,
    ``q_dot = 0.5 q_left(q) [0; w]`` and ``w_dot = J^-1 (S(J w) w + tau)``.
    """
    inertia = p["inertia"].reshape(3, 3)
    inertia_inv = torch.linalg.inv(inertia)
    m = p["mass"].reshape(-1)[0]
    v = x[3:6]
    q = x[6:10]
    w = x[10:13]
    f = u[0]
    tau = u[1:4]
    q = q / torch.linalg.norm(q)
    rot = _rotation(q)
    e3 = torch.tensor([0.0, 0.0, 1.0], dtype=x.dtype)
    p_dot = v
    v_dot = -GRAVITY * e3 + (f / m) * (rot @ e3)
    q_dot = 0.5 * _q_left(q) @ _cat([torch.zeros(1, dtype=x.dtype), w])
    w_dot = inertia_inv @ (_skew(inertia @ w) @ w + tau)
    return _cat([p_dot, v_dot, q_dot, w_dot])


def spacecraft_state_dot(x, u, p):
    """Rigid-body rate dynamics, nx = 3 (spacecraft_dynamics.py:54-66)."""
    inertia = p["inertia_vector"]
    omega_cross = _skew(x)
    return (1.0 / inertia) * (u - omega_cross @ (inertia * x))


def attitude_state_dot(x, u, p):
    """Spacecraft attitude model, nx = 7: ``[q (scalar first), w]``, nu = 3.

    The reference has no such model; it combines the quadrotor's quaternion
    kinematics (normalise, ``q_dot = 0.5 q_left(q)[0; w]``,
    quadrotor_dynamics.py:122,129) with the spacecraft's Euler equation for a
    diagonal inertia ``w_dot = J^-1 (tau - w x J w)`` (spacecraft_dynamics.py:63).
    """
    inertia = p["inertia_vector"]
    q = x[0:4]
    w = x[4:7]
    q = q / torch.linalg.norm(q)
    q_dot = 0.5 * _q_left(q) @ _cat([torch.zeros(1, dtype=x.dtype), w])
    w_dot = (1.0 / inertia) * (u - _skew(w) @ (inertia * w))
    return _cat([q_dot, w_dot])


def cartpole_state_dot(x, u, p):
    """Gym-style cart-pole (cartpole_dynamics.py:59-80)."""
    x_dot, theta, theta_dot = x[1], x[2], x[3]
    force = u[0]
    m_c = p["masscart"].reshape(-1)[0]
    m_p = p["masspole"].reshape(-1)[0]
    length = p["length"].reshape(-1)[0]
    g = p["gravity"].reshape(-1)[0]
    total_mass = m_c + m_p
    polemass_length = m_p * length
    sin_t = torch.sin(theta)
    cos_t = torch.cos(theta)
    temp = (force + polemass_length * theta_dot**2 * sin_t) / total_mass
    theta_acc = (g * sin_t - cos_t * temp) / (
        length * (4.0 / 3.0 - (m_p * cos_t**2) / total_mass)
    )
    x_acc = temp - polemass_length * theta_acc * cos_t / total_mass
    return torch.stack([x_dot, x_acc, theta_dot, theta_acc])


class Model:
    """Static description of a dynamics model: dimensions and ``state_dot``."""

    def __init__(self, name, num_states, num_controls, state_dot, param_keys):
        self.name = name
        self.num_states = num_states
        self.num_controls = num_controls
        self.state_dot = state_dot
        self.param_keys = tuple(param_keys)


def make_model(name, nx=None, nu=None):
    if name == "linear":
        return Model("linear", nx, nu, linear_state_dot, ("A", "B", "b"))
    if name == "quadrotor":
        return Model("quadrotor", 13, 4, quadrotor_state_dot, ("mass", "inertia"))
    if name == "spacecraft":
        return Model("spacecraft", 3, 3, spacecraft_state_dot, ("inertia_vector",))
    if name == "attitude":
        return Model("attitude", 7, 3, attitude_state_dot, ("inertia_vector",))
    if name == "cartpole":
        return Model(
            "cartpole", 4, 1, cartpole_state_dot, ("masscart", "masspole", "length", "gravity")
        )
    raise NotImplementedError(name)
