"""C ABI checks that need no GPU: the library loads, exports every symbol
declared in include/dmpc.h, its structs match ctypes, and host-side
validation rejects bad descriptors without launching anything."""

import ctypes
import os
import re
import shutil
import subprocess

import pytest

from diffmpc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dmpc.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|void|double|const char\*)\s+(dmpc_\w+)\(", text, re.M)))


def test_library_loads_and_exports_every_header_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTED_SYMBOLS)
    assert lib.dmpc_abi_version() == _lib.ABI_VERSION == 3


def test_defaults_match_reference_yaml():
    p = _lib.SolverParams()
    _lib.load().dmpc_default_params(p)
    assert p.tol_convergence == 1e-8 and p.num_scp_iteration_max == 15
    assert p.linesearch == 0 and p.linesearch_eta == 0.4
    assert list(p.alphas)[: p.n_alphas] == [0.01, 0.1, 0.3, 0.7, 1.0]
    assert p.warm_start_backward == 1 and p.pcg_max_iter == 10000 and p.pcg_tol_epsilon == 1e-9


def test_mixed_precision_defaults_agree_everywhere():
    """The C defaults, the Python fallbacks and the package's sqp.yaml give the same mixed-path
    knobs, so a solver built from the YAML runs the tuned configuration."""
    from diffmpc_b200.problem import load_solver_params
    from diffmpc_b200.sqp import solver_params_struct

    c = _lib.SolverParams()
    _lib.load().dmpc_default_params(c)
    from_yaml = solver_params_struct(load_solver_params("sqp.yaml"))
    from_empty = solver_params_struct({})
    for q in (from_yaml, from_empty):
        assert q.inner_rel_tol == c.inner_rel_tol == 1e-3
        assert q.max_refinement == c.max_refinement == 30
        assert q.precision == c.precision == _lib.PREC_MIXED


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc missing")
def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "%s"\n'
        "int main(){printf(\"%%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu\\n\","
        "sizeof(dmpc_solver_params),sizeof(dmpc_group),sizeof(dmpc_adjoint),"
        "offsetof(dmpc_solver_params,blocks_in_smem),offsetof(dmpc_group,lin_controls),"
        "offsetof(dmpc_adjoint,param_grad_index),offsetof(dmpc_adjoint,adj_controls),"
        "sizeof(dmpc_rollout),offsetof(dmpc_rollout,sim_A),offsetof(dmpc_rollout,running_cost));}\n" % HEADER
    )
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [
        ctypes.sizeof(_lib.SolverParams), ctypes.sizeof(_lib.Group), ctypes.sizeof(_lib.Adjoint),
        _lib.SolverParams.blocks_in_smem.offset, _lib.Group.lin_controls.offset,
        _lib.Adjoint.param_grad_index.offset, _lib.Adjoint.adj_controls.offset,
        ctypes.sizeof(_lib.Rollout), _lib.Rollout.sim_A.offset, _lib.Rollout.running_cost.offset,
    ]
    assert got == want


def _group(model=1, nx=13, nu=4, N=10, batch=2, P=10):
    g = _lib.Group()
    g.model, g.nx, g.nu, g.horizon, g.batch, g.scheme, g.n_model_params = model, nx, nu, N, batch, 2, P
    return g


def test_host_validation_rejects_bad_descriptors():
    lib = _lib.load()
    p = _lib.SolverParams()
    lib.dmpc_default_params(p)
    assert lib.dmpc_workspace_size(1, _group(), p) > 0
    assert lib.dmpc_workspace_size(1, _group(nx=12), p) == 0          # quadrotor needs nx = 13
    assert lib.dmpc_workspace_size(1, _group(P=9), p) == 0            # wrong parameter count
    assert lib.dmpc_workspace_size(1, _group(model=9), p) == 0        # unknown model
    assert lib.dmpc_workspace_size(0, _group(), p) == 0               # no groups
    g = _group(nx=12)
    assert lib.dmpc_solve_fwd(1, g, p, None, 0, None) == 4            # DMPC_ERR_UNSUPPORTED
    assert lib.dmpc_solve_fwd(1, _group(), p, None, 0, None) == 2     # DMPC_ERR_WORKSPACE
    bad = _lib.SolverParams()
    lib.dmpc_default_params(bad)
    bad.n_alphas = 0
    assert lib.dmpc_solve_fwd(1, _group(), bad, None, 0, None) == 1   # DMPC_ERR_INVALID
    assert lib.dmpc_error_string(2) == b"workspace too small or misaligned"


@pytest.mark.timeout(120)
def test_calls_return_a_named_cuda_error_without_a_device():
    """With no usable device every entry point returns DMPC_ERR_CUDA promptly (it never
    blocks) and dmpc_last_cuda_error names the runtime's error."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the no-device error path")
    lib = _lib.load()
    p = _lib.SolverParams()
    lib.dmpc_default_params(p)
    n = lib.dmpc_workspace_size(1, _group(), p)
    fake = 1 << 20  # 256-byte aligned; the failed launch never dereferences it
    assert lib.dmpc_solve_fwd(1, _group(), p, fake, n, None) == 3
    assert lib.dmpc_last_cuda_error() not in (b"cudaSuccess", b"")
    assert lib.dmpc_solve_fwd_noalloc(1, _group(), p, None) == 3
    with pytest.raises(_lib.DmpcError, match="CUDA runtime error cuda"):
        _lib.check(3, "dmpc_solve_fwd")


def test_workspace_grows_with_resident_ctas_not_with_batch():
    """The workspace is a 256-byte work counter plus one slot per CTA that can be resident: it
    grows with the batch up to that count and then stays put (persistent launch)."""
    lib = _lib.load()
    p = _lib.SolverParams()
    lib.dmpc_default_params(p)
    a = lib.dmpc_workspace_size(1, _group(batch=1), p)
    b = lib.dmpc_workspace_size(1, _group(batch=4), p)
    c = lib.dmpc_workspace_size(1, _group(batch=1, N=20), p)
    big = lib.dmpc_workspace_size(1, _group(batch=100000), p)
    huge = lib.dmpc_workspace_size(1, _group(batch=1000000), p)
    slot = a - 256
    assert b - 256 == 4 * slot and c > a and slot % 256 == 0
    assert big == huge and (big - 256) % slot == 0 and (big - 256) // slot <= 4 * 1024


def test_jax_shim_is_import_guarded():
    from diffmpc_b200 import jax_shim

    if jax_shim.jax is None:
        with pytest.raises(ImportError):
            jax_shim.make_jax_solve(None, {})


def test_automatic_launch_shape_puts_two_headline_instances_on_an_sm():
    """Mixed precision, quadrotor N=60 (K ceil(13/4) = 244 > 128 threads of the one-CTA row
    layout), more instances than SMs: the automatic choice is the two-CTA configuration, whose
    workspace holds two slots per SM (148 SMs assumed without a device), twice the one-CTA row
    configuration's.  FP64 precision keeps one CTA per SM, and a batch of at most one instance per
    SM takes one slot per instance."""
    lib = _lib.load()
    p = _lib.SolverParams()
    lib.dmpc_default_params(p)
    assert p.precision == _lib.PREC_MIXED and p.cta_config == _lib.CTA_AUTO
    g = _group(N=60, batch=4096)
    auto = lib.dmpc_workspace_size(1, g, p)
    p.cta_config = _lib.CTA_ROWS
    rows = lib.dmpc_workspace_size(1, g, p)
    p.cta_config = _lib.CTA_DUAL
    dual = lib.dmpc_workspace_size(1, g, p)
    assert auto == dual and (auto - 256) == 2 * (rows - 256)
    p.cta_config = _lib.CTA_AUTO
    assert lib.dmpc_workspace_size(1, _group(N=60, batch=100), p) - 256 == 100 * (rows - 256) // 148
    p.precision = _lib.PREC_FP64
    assert lib.dmpc_workspace_size(1, g, p) == rows
