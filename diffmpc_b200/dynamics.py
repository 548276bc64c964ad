"""Dynamics model descriptors (mirror of diffmpc/dynamics/*.py).

The arithmetic of each model lives in ``csrc/models.cuh``; these classes carry
what the host needs: dimensions, state/control names (base_dynamics.py:16-106)
and the packing of the model's parameter dict into the flat per-instance
parameter vector of the C ABI.
"""

from typing import Any, Dict, List

import torch

from . import _lib


class Dynamics:
    """Mirror of diffmpc.dynamics.base_dynamics.Dynamics (base_dynamics.py:16-131)."""

    model_name = None
    param_keys: tuple = ()

    def __init__(self, parameters: Dict[str, Any]):
        self._params = parameters
        self._state_name_to_state_index_dict = {n: i for i, n in enumerate(parameters["names_states"])}
        self._control_name_to_control_index_dict = {n: i for i, n in enumerate(parameters["names_controls"])}

    @property
    def params(self):
        return self._params

    @property
    def num_states(self) -> int:
        return self._params["num_states"]

    @property
    def num_controls(self) -> int:
        return self._params["num_controls"]

    @property
    def names_states(self) -> List[str]:
        return self._params["names_states"]

    @property
    def names_controls(self) -> List[str]:
        return self._params["names_controls"]

    @property
    def state_name_to_state_index_dict(self):
        return self._state_name_to_state_index_dict

    @property
    def control_name_to_control_index_dict(self):
        return self._control_name_to_control_index_dict

    def get_state_variable_at_state_name(self, states, name):
        return states[..., self._state_name_to_state_index_dict[name]]

    def get_control_variable_at_control_name(self, controls, name):
        return controls[..., self._control_name_to_control_index_dict[name]]

    @property
    def model_id(self) -> int:
        return _lib.MODEL_IDS[self.model_name]

    # -- parameter packing ------------------------------------------------------
    def param_shapes(self) -> Dict[str, tuple]:
        raise NotImplementedError

    def num_model_params(self) -> int:
        n = 0
        for shape in self.param_shapes().values():
            k = 1
            for s in shape:
                k *= s
            n += k
        return n

    def param_slices(self) -> Dict[str, slice]:
        out, o = {}, 0
        for key, shape in self.param_shapes().items():
            k = 1
            for s in shape:
                k *= s
            out[key] = slice(o, o + k)
            o += k
        return out

    def defaults(self) -> Dict[str, Any]:
        return {}

    def pack_params(self, params: Dict[str, Any], batch: int, device) -> torch.Tensor:
        """(batch, P) float64 parameter vectors; each entry may be shared or batched."""
        cols = []
        for key, shape in self.param_shapes().items():
            v = params.get(key, self.defaults().get(key))
            if v is None:
                raise KeyError(f"[{type(self).__name__}] missing dynamics parameter '{key}'")
            t = torch.as_tensor(v, dtype=torch.float64, device=device)
            base = 1
            for s in shape:
                base *= s
            if t.numel() == base:
                t = t.reshape(1, base).expand(batch, base)
            else:
                t = t.reshape(batch, base)
            cols.append(t)
        return torch.cat(cols, dim=1).contiguous()


class LinearDynamics(Dynamics):
    """``x_dot = A x + B u + b`` (linear_dynamics.py:46-70); nx, nu free."""

    model_name = "linear"

    def __init__(self, parameters=None):
        if parameters is None:
            parameters = {
                "num_states": 4,
                "num_controls": 2,
                "names_states": ["pos_x", "pos_y", "vel_x", "vel_y"],
                "names_controls": ["force_x", "force_x"],
            }
        super().__init__(parameters)

    def param_shapes(self):
        nx, nu = self.num_states, self.num_controls
        return {"A": (nx, nx), "B": (nx, nu), "b": (nx,)}

    def defaults(self):
        return {"b": torch.zeros(self.num_states, dtype=torch.float64)}


class QuadrotorDynamics(Dynamics):
    """13-state quadrotor [p, v, q, w], controls [thrust, tau] (quadrotor_dynamics.py:8-133)."""

    model_name = "quadrotor"

    def __init__(self, parameters=None):
        if parameters is None:
            parameters = {
                "num_states": 13,
                "num_controls": 4,
                "names_states": [
                    "pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z",
                    "q_0", "q_1", "q_2", "q_3", "omega_x", "omega_y", "omega_z",
                ],
                "names_controls": ["thrust", "torque_x", "torque_y", "torque_z"],
            }
        super().__init__(parameters)

    def param_shapes(self):
        return {"mass": (1,), "inertia": (9,)}

    def defaults(self):
        # quadrotor_dynamics.py:28-31
        return {
            "mass": torch.tensor([0.1], dtype=torch.float64),
            "inertia": torch.tensor([0.1, 0.01, 0.01, 0.01, 0.1, 0.01, 0.01, 0.01, 0.1], dtype=torch.float64),
        }


class SpacecraftDynamics(Dynamics):
    """Angular-rate dynamics, nx = 3 (spacecraft_dynamics.py:9-66)."""

    model_name = "spacecraft"

    def __init__(self, parameters=None):
        if parameters is None:
            parameters = {
                "num_states": 3,
                "num_controls": 3,
                "names_states": ["omega_x", "omega_y", "omega_z"],
                "names_controls": ["torque_x", "torque_y", "torque_z"],
            }
        super().__init__(parameters)

    def param_shapes(self):
        return {"inertia_vector": (3,)}

    def defaults(self):
        return {"inertia_vector": torch.tensor([5.0, 2.0, 1.0], dtype=torch.float64)}


class SpacecraftAttitudeDynamics(Dynamics):
    """Attitude model, nx = 7: unit quaternion (scalar first) + body rate; nu = 3 torques.

    No reference counterpart: it combines the quadrotor's quaternion kinematics
    with the spacecraft's Euler equation for a diagonal inertia.
    """

    model_name = "attitude"

    def __init__(self, parameters=None):
        if parameters is None:
            parameters = {
                "num_states": 7,
                "num_controls": 3,
                "names_states": ["q_0", "q_1", "q_2", "q_3", "omega_x", "omega_y", "omega_z"],
                "names_controls": ["torque_x", "torque_y", "torque_z"],
            }
        super().__init__(parameters)

    def param_shapes(self):
        return {"inertia_vector": (3,)}

    def defaults(self):
        return {"inertia_vector": torch.tensor([1.0, 1.0, 1.0], dtype=torch.float64)}


class CartpoleDynamics(Dynamics):
    """Gym-style cart-pole, nx = 4, nu = 1 (cartpole_dynamics.py:8-80)."""

    model_name = "cartpole"

    def __init__(self, parameters=None):
        if parameters is None:
            parameters = {
                "num_states": 4,
                "num_controls": 1,
                "names_states": ["x", "x_dot", "theta", "theta_dot"],
                "names_controls": ["force"],
            }
        super().__init__(parameters)

    def param_shapes(self):
        return {"masscart": (1,), "masspole": (1,), "length": (1,), "gravity": (1,)}

    def defaults(self):
        return {
            "masscart": torch.tensor([1.0], dtype=torch.float64),
            "masspole": torch.tensor([0.1], dtype=torch.float64),
            "length": torch.tensor([0.5], dtype=torch.float64),
            "gravity": torch.tensor([9.81], dtype=torch.float64),
        }
