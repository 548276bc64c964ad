"""Allocation-free forward solve, called through the C ABI.

Some callers cannot allocate device memory at solve time.
- A real-time MPC loop cannot afford a cudaMalloc stalling the device for an unknown time.
- A host framework may own the device allocator and only lend the library a stream.

`dmpc_solve_fwd_noalloc` serves them from a fixed scratch array inside libdmpc.so.
These tests check three things through the C ABI:
- two calls in a row each reproduce what `dmpc_solve_fwd` gives with a caller-allocated workspace;
- a problem too large for the fixed array is refused;
- the refusal launches nothing.

This file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""

import pytest
import torch

from diffmpc_b200 import OptimalControlProblem, SQPSolver, _lib, workloads
from diffmpc_b200.sqp import _Call

pytestmark = pytest.mark.gpu

DMPC_ERR_WORKSPACE = 2


def _fresh_call(solver, params):
    guess = solver.initial_guess(params)
    return _Call(solver, guess, params, guess.states.shape[0], guess.states.device)


def _solver(B, N, seed):
    dyn, st, bt, sp = workloads.quadrotor(B=B, N=N, seed=seed)
    sp["pcg"]["tol_epsilon"] = 1e-11
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp)
    return solver, workloads.to_device(bt, "cuda")


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    lib = _lib.load()
    solver, p = _solver(B=4, N=20, seed=31)
    stream = torch.cuda.current_stream().cuda_stream

    ref = _fresh_call(solver, p)
    n = lib.dmpc_workspace_size(1, ref.group, solver._c_params)
    assert 0 < n <= _lib.DMPC_NOALLOC_SCRATCH_BYTES
    ws = torch.empty(n, dtype=torch.uint8, device="cuda")
    assert lib.dmpc_solve_fwd(1, ref.group, solver._c_params, ws.data_ptr(), n, stream) == 0
    torch.cuda.synchronize()

    for _ in range(2):  # the second call reuses the scratch the first call left behind
        c = _fresh_call(solver, p)
        assert lib.dmpc_solve_fwd_noalloc(1, c.group, solver._c_params, stream) == 0
        torch.cuda.synchronize()
        for name in ("states", "controls", "dual", "lin_states", "lin_controls", "conv"):
            a, b = getattr(c, name), getattr(ref, name)
            assert torch.allclose(a, b, rtol=1e-12, atol=1e-14), name
        assert torch.equal(c.status, ref.status)
        assert torch.equal(c.num_iter, ref.num_iter)
        assert torch.equal(c.pcg_hist, ref.pcg_hist)


def test_noalloc_refuses_problems_larger_than_its_scratch():
    lib = _lib.load()
    solver, p = _solver(B=64, N=60, seed=32)  # about 43 MB of scratch, above the 32 MiB array
    stream = torch.cuda.current_stream().cuda_stream
    c = _fresh_call(solver, p)
    assert lib.dmpc_workspace_size(1, c.group, solver._c_params) > _lib.DMPC_NOALLOC_SCRATCH_BYTES
    before = c.states.clone()
    assert lib.dmpc_solve_fwd_noalloc(1, c.group, solver._c_params, stream) == DMPC_ERR_WORKSPACE
    torch.cuda.synchronize()
    assert torch.equal(c.states, before)  # refused before any launch
    assert int(c.num_iter.abs().sum()) == 0
