"""Optimal control problem restatement (oracle, float64, one instance).

Follows diffmpc/problems/optimal_control_problem.py and
diffmpc/dynamics/integrators.py.  Every method works on ONE instance;
batching is done by the solver with ``torch.func.vmap``.
"""

import torch
from torch.func import grad, hessian, jacfwd, vmap

EULER, MIDPOINT, RUNGEKUTTA4 = 0, 1, 2  # integrators.py:12-17

REQUIRED_KEYS = (  # required_parameters.yaml:1-15
    "horizon",
    "discretization_resolution",
    "discretization_scheme",
    "initial_state",
    "final_state",
    "reference_state_trajectory",
    "reference_control_trajectory",
    "penalize_control_reference",
    "weights_penalization_reference_state_trajectory",
    "weights_penalization_final_state",
    "weights_penalization_control_squared",
)
STATIC_KEYS = ("horizon", "discretization_scheme", "penalize_control_reference")


def predict_next_state(model, dt, scheme, params, x, u):
    """One integration step (integrators.py:20-71).

    The Euler step is always evaluated first and then overwritten for the
    midpoint and RK4 schemes, exactly as the reference does.
    """
    x_next = x + dt * model.state_dot(x, u, params)
    if scheme == MIDPOINT:
        x_mid = x + 0.5 * dt * model.state_dot(x, u, params)
        x_next = x + dt * model.state_dot(x_mid, u, params)
    elif scheme == RUNGEKUTTA4:
        k1 = model.state_dot(x, u, params)
        k2 = model.state_dot(x + 0.5 * dt * k1, u, params)
        k3 = model.state_dot(x + 0.5 * dt * k2, u, params)
        k4 = model.state_dot(x + dt * k3, u, params)
        x_next = x + (1.0 / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4) * dt
    return x_next


def check_parameters(params):
    """Raises like load_params.py:89-101."""
    if params is None:
        raise ValueError("[OptimalControlProblem] params should be a dictionary.")
    for key in REQUIRED_KEYS:
        if key not in params:
            raise KeyError("[OptimalControlProblem]", key, "is not in params dictionary")
    return True


class OptimalControlProblem:
    """Restatement of OptimalControlProblem (optimal_control_problem.py:16-398)."""

    def __init__(self, model, params, check_parameters_are_valid=True):
        if check_parameters_are_valid:
            check_parameters(params)
        self.model = model
        self.params = dict(params)
        self.horizon = int(params["horizon"])
        self.scheme = int(params["discretization_scheme"])
        self.penalize_control_reference = bool(params["penalize_control_reference"])
        self.num_state_variables = model.num_states
        self.num_control_variables = model.num_controls

    # -- initial guess (:82-102) ------------------------------------------
    def initial_guess(self, params):
        N = self.horizon
        x0 = params["initial_state"]
        xf = params["final_state"]
        t = torch.arange(N + 1, dtype=torch.float64)
        a1 = ((N - t) / N)[:, None]
        a2 = (t / N)[:, None]
        states = x0[None] * a1 + xf[None] * a2 + 1e-6
        controls = torch.zeros(N + 1, self.num_control_variables, dtype=torch.float64) + 1e-6
        return states, controls

    # -- dynamics -----------------------------------------------------------
    def next_state(self, params, x, u):
        return predict_next_state(
            self.model, params["discretization_resolution"], self.scheme, params, x, u
        )

    def equality_constraints(self, states, controls, params):
        """``[x_0 - x0; f(x_t, u_t) - x_{t+1}]`` flattened (:104-151)."""
        N = self.horizon
        c0 = states[0] - params["initial_state"]
        nxt = vmap(lambda x, u: self.next_state(params, x, u))(states[:N], controls[:N])
        return torch.cat([c0, (nxt - states[1:]).reshape(-1)])

    def get_dynamics_linearized_matrices(self, states, controls, params):
        """``As_next = -I``, ``As, Bs`` by forward-mode Jacobian, ``Cs`` (:325-398)."""
        N, nx = self.horizon, self.num_state_variables

        def f(z):
            return self.next_state(params, z[:nx], z[nx:])

        zs = torch.cat([states[:N], controls[:N]], dim=-1)
        nxt = vmap(f)(zs)
        jac = vmap(jacfwd(f))(zs)
        As = jac[:, :, :nx]
        Bs = jac[:, :, nx:]
        Cs = torch.cat(
            [
                params["initial_state"][None],
                -nxt
                + torch.einsum("tij,tj->ti", As, states[:N])
                + torch.einsum("tij,tj->ti", Bs, controls[:N]),
            ]
        )
        As_next = -torch.eye(nx, dtype=torch.float64).expand(N, nx, nx).clone()
        return As_next, As, Bs, Cs

    # -- cost (:153-323) ------------------------------------------------------
    def step_cost(self, x, u, p):
        nu = self.num_control_variables
        if self.penalize_control_reference:
            ref = torch.cat([p["reference_state_trajectory"], p["reference_control_trajectory"]])
        else:
            ref = torch.cat(
                [p["reference_state_trajectory"], torch.zeros(nu, dtype=torch.float64)]
            )
        w = torch.cat(
            [
                p["weights_penalization_reference_state_trajectory"],
                p["weights_penalization_control_squared"],
            ]
        )
        z = torch.cat([x, u])
        return torch.sum(w * (z - ref) ** 2)

    def final_cost(self, x, p):
        w = p["weights_penalization_reference_state_trajectory"] + p[
            "weights_penalization_final_state"
        ]
        return torch.sum(w * (x - p["final_state"]) ** 2)

    _KEYS_REF = ("reference_state_trajectory", "reference_control_trajectory")
    _KEYS_W = (
        "weights_penalization_reference_state_trajectory",
        "weights_penalization_control_squared",
        "weights_penalization_final_state",
        "final_state",
    )

    def _split_cost_params(self, params):
        N = self.horizon
        step = {k: params[k][:-1] for k in self._KEYS_REF}
        step.update({k: params[k][None].expand(N, *params[k].shape) for k in self._KEYS_W})
        final = {k: params[k][-1] for k in self._KEYS_REF}
        final.update({k: params[k] for k in self._KEYS_W})
        return step, final

    def cost(self, states, controls, params):
        step, final = self._split_cost_params(params)
        sc = vmap(self.step_cost)(states[:-1], controls[:-1], step)
        return torch.sum(sc) + self.final_cost(states[-1], final)

    def get_cost_linearized_matrices(self, states, controls, params):
        """QN, qN, Q, q, R, r with ``q = J - x^T H`` on the unprojected H (:249-323)."""
        step, final = self._split_cost_params(params)
        Jx, Ju = vmap(grad(self.step_cost, argnums=(0, 1)))(states[:-1], controls[:-1], step)
        Hxx = vmap(hessian(self.step_cost, argnums=0))(states[:-1], controls[:-1], step)
        Huu = vmap(hessian(self.step_cost, argnums=1))(states[:-1], controls[:-1], step)
        JT = grad(self.final_cost, argnums=0)(states[-1], final)
        HT = hessian(self.final_cost, argnums=0)(states[-1], final)
        QN = HT
        qN = JT - states[-1] @ HT
        q = Jx - torch.einsum("ti,tij->tj", states[:-1], Hxx)
        r = Ju - torch.einsum("ti,tij->tj", controls[:-1], Huu)
        return QN, qN, Hxx, q, Huu, r
