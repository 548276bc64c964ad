"""Problem definition and parameter loading (mirror of
diffmpc/problems/optimal_control_problem.py and diffmpc/utils/load_params.py).

The problem object carries the static configuration of the path (model,
horizon, discretization scheme, whether the control reference is penalized)
and the default parameter dict; the numerical work runs in ``libdmpc.so``.
"""

import copy
import os
from typing import Any, Dict

import torch
import yaml

from .dynamics import Dynamics

_PARAMS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "params")

# load_params.py:65-70: entries kept as python scalars
NOT_TENSOR_KEYS = ("horizon", "discretization_scheme", "penalize_control_reference", "rescale_optimization_variables")


def load_params(path: str) -> Dict[str, Any]:
    """yaml.safe_load of a parameter file (load_params.py:10-23)."""
    with open(path, "r") as f:
        return yaml.safe_load(f)


def load_solver_params(filename: str = "sqp.yaml") -> Dict[str, Any]:
    """Solver parameters from the package's params folder (load_params.py:26-43)."""
    return load_params(os.path.join(_PARAMS_DIR, filename))


def load_problem_params(filename: str) -> Dict[str, Any]:
    """Problem parameters as float64 tensors, references repeated over horizon+1
    (load_params.py:46-86)."""
    params = load_params(os.path.join(_PARAMS_DIR, filename))
    for key in list(params):
        if key not in NOT_TENSOR_KEYS:
            params[key] = torch.as_tensor(params[key], dtype=torch.float64)
    K = int(params["horizon"]) + 1
    for key in ("reference_state_trajectory", "reference_control_trajectory"):
        params[key] = params[key][None].repeat(K, *([1] * params[key].dim()))
    return params


def check_parameters_dictionary_or_raise_errors(params: Dict[str, Any]) -> bool:
    """Raises ValueError / KeyError like load_params.py:89-101."""
    if params is None:
        raise ValueError("[OptimalControlProblem] params should be a dictionary.")
    for key in load_params(os.path.join(_PARAMS_DIR, "required_parameters.yaml")):
        if key not in params:
            raise KeyError("[OptimalControlProblem]", key, "is not in params dictionary")
    return True


class OptimalControlProblem:
    """Mirror of OptimalControlProblem (optimal_control_problem.py:16-80).

    Cost: sum_t w_x.(x_t - xref_t)^2 + w_u.(u_t - uref_t)^2 (t < N) plus
    (w_x + w_f).(x_N - x_final)^2; constraints x_0 = x_init and
    x_{t+1} = F(x_t, u_t) with F one step of the chosen integrator.
    """

    def __init__(self, dynamics: Dynamics, params: Dict[str, Any] = None, check_parameters_are_valid: bool = True):
        if check_parameters_are_valid:
            check_parameters_dictionary_or_raise_errors(params)
        self._dynamics = dynamics
        self._params = copy.copy(params)
        self._discretization_scheme = int(params["discretization_scheme"])
        if self._discretization_scheme not in (0, 1, 2):
            raise ValueError(f"discretization_scheme {self._discretization_scheme} is not 0, 1 or 2")
        self._num_variables = (self.num_control_variables + self.num_state_variables) * (self.horizon + 1)
        self._num_constraints = self.num_state_variables * (self.horizon + 1)
        self.name = "OptimalControlProblem"

    @property
    def dynamics(self) -> Dynamics:
        return self._dynamics

    @property
    def params(self) -> Dict[str, Any]:
        return self._params

    @property
    def horizon(self) -> int:
        return int(self._params["horizon"])

    @property
    def discretization_scheme(self) -> int:
        return self._discretization_scheme

    @property
    def penalize_control_reference(self) -> bool:
        return bool(self._params["penalize_control_reference"])

    @property
    def num_variables(self) -> int:
        return self._num_variables

    @property
    def num_constraints(self) -> int:
        return self._num_constraints

    @property
    def num_state_variables(self) -> int:
        return self._dynamics.num_states

    @property
    def num_control_variables(self) -> int:
        return self._dynamics.num_controls

    def initial_guess(self, params: Dict[str, Any] = None, device=None):
        """Straight line from initial to final state (+1e-6), controls 1e-6
        (optimal_control_problem.py:82-102).  Batched when initial_state is (B, nx)."""
        if params is None:
            params = self._params
        x0 = torch.as_tensor(params["initial_state"], dtype=torch.float64, device=device)
        xf = torch.as_tensor(params["final_state"], dtype=torch.float64, device=device)
        N = self.horizon
        t = torch.arange(N + 1, dtype=torch.float64, device=x0.device)
        a1 = ((N - t) / N)[:, None]
        a2 = (t / N)[:, None]
        states = x0[..., None, :] * a1 + xf[..., None, :] * a2 + 1e-6
        lead = states.shape[:-2]
        controls = torch.zeros(*lead, N + 1, self.num_control_variables, dtype=torch.float64, device=x0.device) + 1e-6
        return states, controls
