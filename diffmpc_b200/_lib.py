"""ctypes binding of ``libdmpc.so`` (the C ABI declared in ``include/dmpc.h``).

The shared library is built in-tree (``diffmpc_b200/libdmpc.so``) by
``diffmpc_b200/build.py``.  Loading fails loudly when it is missing: there is
no CPU fallback for the solver.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdmpc.so")

ABI_VERSION = 3
DMPC_OK = 0
DMPC_ERR_INVALID = 1
DMPC_ERR_CUDA = 3
DMPC_MAX_NX = 32
DMPC_MAX_NU = 16
DMPC_MAX_ALPHAS = 8
DMPC_MAX_PARAM_GRADS = 64
DMPC_MAX_GROUPS = 8
DMPC_NOALLOC_SCRATCH_BYTES = 32 * 1024 * 1024

MODEL_IDS = {"linear": 0, "quadrotor": 1, "spacecraft": 2, "attitude": 3, "cartpole": 4}
PREC_FP64, PREC_MIXED = 0, 1
CTA_AUTO, CTA_WIDE, CTA_ROWS, CTA_DUAL = 0, 1, 2, 3
SIM_LINEAR, SIM_MODEL, SIM_MODEL_SCHEME = 0, 1, 2

EXPORTED_SYMBOLS = (
    "dmpc_abi_version",
    "dmpc_error_string",
    "dmpc_last_cuda_error",
    "dmpc_workspace_size",
    "dmpc_default_params",
    "dmpc_solve_fwd",
    "dmpc_solve_adj",
    "dmpc_linearize",
    "dmpc_schur_assemble",
    "dmpc_schur_workspace_size",
    "dmpc_pcg_solve",
    "dmpc_compute_gamma",
    "dmpc_kkt_recover",
    "dmpc_probe_fp32_fma",
    "dmpc_solve_fwd_noalloc",
    "dmpc_rollout_fwd",
    "dmpc_rollout_adj",
    "dmpc_psd_project",
)

_p = ctypes.c_void_p
_i32 = ctypes.c_int32
_f64 = ctypes.c_double


class SolverParams(ctypes.Structure):
    _fields_ = [
        ("tol_convergence", _f64),
        ("num_scp_iteration_max", _i32),
        ("linesearch", _i32),
        ("linesearch_eta", _f64),
        ("n_alphas", _i32),
        ("alphas", _f64 * DMPC_MAX_ALPHAS),
        ("warm_start_backward", _i32),
        ("pcg_max_iter", _i32),
        ("pcg_tol_epsilon", _f64),
        ("precision", _i32),
        ("max_refinement", _i32),
        ("inner_rel_tol", _f64),
        ("threads_per_block", _i32),
        ("blocks_in_smem", _i32),
        ("cta_config", _i32),
    ]


class Group(ctypes.Structure):
    _fields_ = [
        ("model", _i32),
        ("nx", _i32),
        ("nu", _i32),
        ("horizon", _i32),
        ("batch", _i32),
        ("scheme", _i32),
        ("penalize_control_reference", _i32),
        ("n_model_params", _i32),
        ("horizons", _p),
        ("dt", _p),
        ("initial_state", _p),
        ("final_state", _p),
        ("reference_state", _p),
        ("reference_control", _p),
        ("w_x", _p),
        ("w_u", _p),
        ("w_f", _p),
        ("model_params", _p),
        ("states", _p),
        ("controls", _p),
        ("dual", _p),
        ("convergence_error", _p),
        ("status", _p),
        ("num_iter", _p),
        ("convergence_errors", _p),
        ("linesearch_alphas", _p),
        ("num_pcg_iters", _p),
        ("lin_states", _p),
        ("lin_controls", _p),
        ("num_pcg_corrections", _p),
        ("num_pcg_fp64_iters", _p),
    ]


class Adjoint(ctypes.Structure):
    _fields_ = [
        ("dl_dstates", _p),
        ("dl_dcontrols", _p),
        ("dual_backward_guess", _p),
        ("dual_backward", _p),
        ("num_pcg_iter", _p),
        ("g_initial_state", _p),
        ("g_final_state", _p),
        ("g_w_x", _p),
        ("g_w_u", _p),
        ("g_w_f", _p),
        ("g_reference_state", _p),
        ("g_reference_control", _p),
        ("n_param_grads", _i32),
        ("param_grad_index", ctypes.POINTER(_i32)),
        ("g_model_params", _p),
        ("adj_states", _p),
        ("adj_controls", _p),
        ("num_pcg_corrections", _p),
        ("num_pcg_fp64_iter", _p),
    ]


class Rollout(ctypes.Structure):
    _fields_ = [
        ("num_steps", _i32),
        ("warm_start", _i32),
        ("simulator", _i32),
        ("reserved", _i32),
        ("cost_state_weights", _p),
        ("cost_control_weights", _p),
        ("cost_state_ref", _p),
        ("cost_control_ref", _p),
        ("sim_A", _p),
        ("sim_B", _p),
        ("sim_b", _p),
        ("step_initial_state", _p),
        ("step_states", _p),
        ("step_controls", _p),
        ("step_dual", _p),
        ("step_lin_states", _p),
        ("step_lin_controls", _p),
        ("step_status", _p),
        ("step_num_iter", _p),
        ("step_convergence_error", _p),
        ("step_convergence_errors", _p),
        ("step_linesearch_alphas", _p),
        ("step_num_pcg_iters", _p),
        ("running_cost", _p),
    ]


class RolloutAdjoint(ctypes.Structure):
    _fields_ = [
        ("cost_cotangent", _p),
        ("through_state", _i32),
        ("scratch_dl_dcontrols", _p),
        ("scratch_dual", _p),
        ("g_initial_state", _p),
    ]


class DmpcError(RuntimeError):
    pass


_lib = None


def load():
    """Loads ``libdmpc.so``; raises ``DmpcError`` if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise DmpcError(
            f"{LIB_PATH} is missing: build it with `python -m diffmpc_b200.build` "
            "(the solver has no CPU fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    lib.dmpc_abi_version.restype = ctypes.c_int
    lib.dmpc_error_string.restype = ctypes.c_char_p
    lib.dmpc_error_string.argtypes = [ctypes.c_int]
    lib.dmpc_last_cuda_error.restype = ctypes.c_char_p
    lib.dmpc_last_cuda_error.argtypes = []
    lib.dmpc_workspace_size.restype = ctypes.c_size_t
    lib.dmpc_workspace_size.argtypes = [ctypes.c_int, ctypes.POINTER(Group), ctypes.POINTER(SolverParams)]
    lib.dmpc_default_params.restype = None
    lib.dmpc_default_params.argtypes = [ctypes.POINTER(SolverParams)]
    lib.dmpc_solve_fwd.restype = ctypes.c_int
    lib.dmpc_solve_fwd.argtypes = [
        ctypes.c_int, ctypes.POINTER(Group), ctypes.POINTER(SolverParams), _p, ctypes.c_size_t, _p,
    ]
    lib.dmpc_solve_adj.restype = ctypes.c_int
    lib.dmpc_solve_adj.argtypes = [
        ctypes.c_int, ctypes.POINTER(Group), ctypes.POINTER(Adjoint), ctypes.POINTER(SolverParams),
        _p, ctypes.c_size_t, _p,
    ]
    lib.dmpc_linearize.restype = ctypes.c_int
    lib.dmpc_linearize.argtypes = [ctypes.POINTER(Group), ctypes.POINTER(SolverParams)] + [_p] * 7 + [
        _p, ctypes.c_size_t, _p,
    ]
    lib.dmpc_schur_workspace_size.restype = ctypes.c_size_t
    lib.dmpc_schur_workspace_size.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.dmpc_schur_assemble.restype = ctypes.c_int
    lib.dmpc_schur_assemble.argtypes = [ctypes.c_int] * 4 + [_p] * 11 + [_p, ctypes.c_size_t, _p]
    lib.dmpc_pcg_solve.restype = ctypes.c_int
    lib.dmpc_pcg_solve.argtypes = [ctypes.c_int] * 4 + [_p] * 11 + [ctypes.c_int, _f64] + [_p] * 5 + [_p]
    lib.dmpc_compute_gamma.restype = ctypes.c_int
    lib.dmpc_compute_gamma.argtypes = [ctypes.c_int] * 4 + [_p] * 8 + [_p]
    lib.dmpc_kkt_recover.restype = ctypes.c_int
    lib.dmpc_kkt_recover.argtypes = [ctypes.c_int] * 4 + [_p] * 10 + [_p]
    lib.dmpc_probe_fp32_fma.restype = ctypes.c_double
    lib.dmpc_probe_fp32_fma.argtypes = [ctypes.c_int, ctypes.c_int, _p, _p]
    lib.dmpc_solve_fwd_noalloc.restype = ctypes.c_int
    lib.dmpc_solve_fwd_noalloc.argtypes = [ctypes.c_int, ctypes.POINTER(Group), ctypes.POINTER(SolverParams), _p]
    lib.dmpc_rollout_fwd.restype = ctypes.c_int
    lib.dmpc_rollout_fwd.argtypes = [
        ctypes.POINTER(Group), ctypes.POINTER(Rollout), ctypes.POINTER(SolverParams), _p, ctypes.c_size_t, _p,
    ]
    lib.dmpc_rollout_adj.restype = ctypes.c_int
    lib.dmpc_rollout_adj.argtypes = [
        ctypes.POINTER(Group), ctypes.POINTER(Rollout), ctypes.POINTER(Adjoint), ctypes.POINTER(RolloutAdjoint),
        ctypes.POINTER(SolverParams), _p, ctypes.c_size_t, _p,
    ]
    lib.dmpc_psd_project.restype = ctypes.c_int
    lib.dmpc_psd_project.argtypes = [ctypes.c_int, ctypes.c_int, _p, _f64, _p, _p]
    if lib.dmpc_abi_version() != ABI_VERSION:
        raise DmpcError("libdmpc.so ABI version mismatch")
    _lib = lib
    return lib


def check(rc, what):
    if rc != DMPC_OK:
        lib = load()
        msg = lib.dmpc_error_string(rc).decode()
        if rc == DMPC_ERR_CUDA:
            msg += " " + lib.dmpc_last_cuda_error().decode()
        raise DmpcError(f"{what} failed: {msg} (code {rc})")
