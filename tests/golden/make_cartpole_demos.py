"""Generates tests/golden/cartpole_demos.npz from the reference's
benchmarking/imitation-learning/demonstrations.pkl (run once, where the reference
is mounted; the fixture is committed, the pickle is not read at test time).

The pickle holds 32 dicts {"x0": jax.Array (4,), "ctrl_traj": jax.Array (101, 1)}
written by the reference's collect_expert_data.py:21-59 (cartpole.yaml, N=100,
SQP max 501 iterations, line search on, PCG tolerance 1e-24).  jax is not
installed here, so the unpickler maps jax's array reconstructor to numpy.
"""

import os
import pickle
import sys

import numpy as np

SRC = "/root/reference/benchmarking/imitation-learning/demonstrations.pkl"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cartpole_demos.npz")


def _reconstruct(fun, args, state, aval=None):
    obj = fun(*args)
    obj.__setstate__(state)
    return obj


class _Unpickler(pickle.Unpickler):
    def find_class(self, module, name):
        if module.startswith("jax") and name == "_reconstruct_array":
            return _reconstruct
        if module.startswith("jax"):
            # abstract-value / sharding helpers carry no array data
            return lambda *a, **k: None
        return super().find_class(module, name)


def main(src=SRC):
    with open(src, "rb") as f:
        data = _Unpickler(f).load()
    x0 = np.stack([np.asarray(d["x0"], dtype=np.float64) for d in data])
    u = np.stack([np.asarray(d["ctrl_traj"], dtype=np.float64) for d in data])
    np.savez_compressed(OUT, x0=x0, ctrl_traj=u)
    print(OUT, x0.shape, u.shape)


if __name__ == "__main__":
    main(*sys.argv[1:])
