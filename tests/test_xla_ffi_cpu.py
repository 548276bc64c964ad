"""The XLA custom-call handler core (include/dmpc_xla.h, csrc/xla_ffi.cc) on the CPU: the library
exports every function the header declares, and a C program linked against it checks the
operand lists, the workspace size and the validation of malformed operand lists (tests/c).
The XLA handler symbols themselves need jaxlib's headers, which this image does not have:
that part is unvalidated."""

import os
import re
import shutil
import subprocess

import pytest

from diffmpc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
XLA_HEADER = os.path.join(ROOT, "include", "dmpc_xla.h")


def xla_header_functions():
    text = open(XLA_HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(dmpc_xla_\w+)\(", text, re.M)))


def test_library_exports_every_xla_header_symbol():
    lib = _lib.load()
    names = xla_header_functions()
    assert names == ["dmpc_xla_adj_operands", "dmpc_xla_fwd_operands", "dmpc_xla_solve_adj",
                     "dmpc_xla_solve_fwd", "dmpc_xla_workspace_size"]
    for n in names:
        assert hasattr(lib, n), n


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_handler_core_from_c(tmp_path):
    lib = _lib.load()
    libdir = os.path.dirname(lib._name)
    exe = str(tmp_path / "test_xla_ffi")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "test_xla_ffi.c"), "-L", libdir, "-ldmpc",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"


def test_ffi_attributes_carry_the_solver_parameters():
    import ctypes

    from diffmpc_b200 import OptimalControlProblem, SQPSolver, jax_shim, workloads

    dyn, st, bt, sp = workloads.quadrotor(B=2, N=10, seed=3)
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp, device="cpu")
    at = jax_shim.ffi_attributes(solver, 2)
    assert (at["model"], at["nx"], at["nu"], at["horizon"], at["batch"]) == (_lib.MODEL_IDS["quadrotor"], 13, 4, 10, 2)
    raw = at["solver_params"]
    assert raw.dtype.itemsize == 1 and raw.size == ctypes.sizeof(_lib.SolverParams)
    back = _lib.SolverParams.from_buffer_copy(raw.tobytes())
    assert back.pcg_tol_epsilon == sp["pcg"]["tol_epsilon"] and back.num_scp_iteration_max == sp["num_scp_iteration_max"]
