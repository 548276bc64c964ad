"""JAX front end: ``jax.custom_vjp`` over the same solver (needs jax and jaxlib).

``make_jax_solve(solver)`` returns ``solve(x0, weights) -> (states, controls)``.
- It is differentiable with ``jax.grad`` w.r.t. ``weights``, a dict of float64 arrays.
- Its forward and backward run the CUDA kernels through ``jax.pure_callback``, handing the arrays over via host memory. This keeps existing JAX code (``jit``, ``grad``) working unchanged.
- A zero-copy binding registers the C entry points as XLA FFI custom calls instead
  (``register_ffi_targets``).  The handlers that map XLA buffers onto the C ABI are in
  ``csrc/xla_ffi.cc`` (operand orders in ``include/dmpc_xla.h``); their core is built into
  ``libdmpc.so`` and tested from C, the XLA-facing symbols only when the library is built with
  ``DMPC_XLA_INCLUDE`` pointing at jaxlib's include directory.

JAX and jaxlib are not installed in the image this library is built in, so this module is
import-guarded and untested there.  ``make_jax_solve`` raises ImportError without jax.
"""

from typing import Dict

try:  # pragma: no cover - exercised only where jax is installed
    import jax
    import jax.numpy as jnp
except ImportError:  # pragma: no cover
    jax = None
    jnp = None


FFI_TARGETS = (("dmpc_solve_fwd", "dmpc_xla_fwd_handler"), ("dmpc_solve_adj", "dmpc_xla_adj_handler"))


def register_ffi_targets():
    """Registers the library's XLA FFI handlers as the CUDA custom-call targets "dmpc_solve_fwd" and
    "dmpc_solve_adj".  Needs jax and a ``libdmpc.so`` built with ``DMPC_XLA_INCLUDE`` (so that
    ``csrc/xla_ffi.cc`` compiles its XLA part); unvalidated, since neither exists where this
    library is built."""
    if jax is None:
        raise ImportError("diffmpc_b200.jax_shim needs jax and jaxlib (not installed)")
    from diffmpc_b200 import _lib

    lib = _lib.load()
    for target, sym in FFI_TARGETS:
        if not hasattr(lib, sym):
            raise RuntimeError(f"{sym} is not in libdmpc.so: rebuild with DMPC_XLA_INCLUDE=<jaxlib>/include")
        jax.ffi.register_ffi_target(target, jax.ffi.pycapsule(getattr(lib, sym)), platform="CUDA")


def ffi_attributes(solver, batch: int):
    """The custom calls' attributes for ``solver`` and a batch: the problem's integers and the
    solver parameters as the raw bytes of a dmpc_solver_params."""
    import numpy as np

    from diffmpc_b200.sqp import solver_params_struct

    prog = solver.program
    dyn = prog.dynamics
    return {
        "model": dyn.model_id, "nx": prog.num_state_variables, "nu": prog.num_control_variables,
        "horizon": prog.horizon, "batch": int(batch), "scheme": prog.discretization_scheme,
        "penalize_control_reference": int(bool(prog.penalize_control_reference)),
        "n_model_params": dyn.num_model_params(),
        "solver_params": np.frombuffer(bytes(solver_params_struct(solver.params)), dtype=np.uint8),
    }


def make_jax_solve(solver, problem_params: Dict):
    if jax is None:
        raise ImportError("diffmpc_b200.jax_shim needs jax and jaxlib (not installed)")
    import numpy as np
    import torch

    prog = solver.program
    K, nx, nu = prog.horizon + 1, prog.num_state_variables, prog.num_control_variables

    def _torch_solve(x0, wvals, keys, want_grad, gx, gu):
        dev = torch.device("cuda", torch.cuda.current_device())
        p = {k: (torch.as_tensor(np.asarray(v), device=dev) if hasattr(v, "shape") else v)
             for k, v in problem_params.items()}
        p["initial_state"] = torch.as_tensor(np.asarray(x0), dtype=torch.float64, device=dev)
        w = {k: torch.as_tensor(np.asarray(v), dtype=torch.float64, device=dev).requires_grad_(want_grad)
             for k, v in zip(keys, wvals)}
        sol = solver.solve(solver.initial_guess(p), p, w)
        if not want_grad:
            return sol.states.detach().cpu().numpy(), sol.controls.detach().cpu().numpy()
        gx_t = torch.as_tensor(np.asarray(gx), device=dev)
        gu_t = torch.as_tensor(np.asarray(gu), device=dev)
        torch.autograd.backward([sol.states, sol.controls], [gx_t, gu_t])
        return tuple(w[k].grad.detach().cpu().numpy() for k in keys)

    @jax.custom_vjp
    def solve(x0, weights):
        keys = sorted(weights)
        lead = x0.shape[:-1]
        shapes = (jax.ShapeDtypeStruct(lead + (K, nx), jnp.float64), jax.ShapeDtypeStruct(lead + (K, nu), jnp.float64))
        return jax.pure_callback(
            lambda x, *ws: _torch_solve(x, ws, keys, False, None, None), shapes, x0, *[weights[k] for k in keys]
        )

    def fwd(x0, weights):
        return solve(x0, weights), (x0, weights)

    def bwd(res, cot):
        x0, weights = res
        keys = sorted(weights)
        shapes = tuple(jax.ShapeDtypeStruct(weights[k].shape, jnp.float64) for k in keys)
        grads = jax.pure_callback(
            lambda x, gx, gu, *ws: _torch_solve(x, ws, keys, True, gx, gu), shapes, x0, cot[0], cot[1],
            *[weights[k] for k in keys],
        )
        return None, dict(zip(keys, grads))

    solve.defvjp(fwd, bwd)
    return solve
