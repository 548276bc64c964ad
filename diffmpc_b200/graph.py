"""CUDA-graph capture of the forward solve.

For a closed-loop controller that re-solves the same problem shape every control
period (the reference's ``lax.scan`` rollouts), the per-call host work matters:
building descriptors and launching.  ``GraphedForward`` captures ONE
``dmpc_solve_fwd`` launch on static device buffers.  Each call then copies the new
initial state and warm start into those buffers and replays the graph: one graph
launch, no host-side descriptor building.

It is not differentiable.  ``CapturedStep`` captures a whole differentiable step instead:
forward solves, the loss, and the adjoint launches of its backward pass (``solve_groups``
over ragged groups, ``ClosedLoopRollout``, or plain ``SQPSolver.solve``), so that a training
or evaluation loop on a fixed shape replays it as one graph.
"""

from typing import Optional

import torch

from . import _lib
from .sqp import SQPSolution, SQPSolver, _Call


class GraphedForward:
    """Replays a captured forward solve of ``solver`` on a fixed batch shape.

    ``problem_params`` and ``initial_guess`` (batched) fix the buffers.  Every
    subsequent ``__call__`` may change the initial state and the warm start; other
    parameters can be updated in place through ``self.call`` (its tensors are the graph's
    inputs).
    """

    def __init__(self, solver: SQPSolver, initial_guess: SQPSolution, problem_params: dict):
        lib = _lib.load()
        dev = initial_guess.states.device
        self.solver = solver
        B = initial_guess.states.shape[0]
        self.call = _Call(solver, initial_guess, problem_params, B, dev)
        n = lib.dmpc_workspace_size(1, self.call.group, solver._c_params)
        self.ws = torch.empty(max(n, 256), dtype=torch.uint8, device=dev)
        self._guess_states = self.call.states.clone()
        self._guess_controls = self.call.controls.clone()
        self._guess_dual = self.call.dual.clone()
        self._guess_conv = self.call.conv.clone()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            # one eager launch outside the capture: sets the kernel's shared-memory
            # attribute and loads the module before capture begins
            self._restore()
            _lib.check(self._launch(lib, side.cuda_stream), "dmpc_solve_fwd")
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
            self._restore()
            rc = self._launch(lib, torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(rc, "dmpc_solve_fwd (capture)")

    def _launch(self, lib, stream):
        return lib.dmpc_solve_fwd(1, self.call.group, self.solver._c_params, self.ws.data_ptr(), self.ws.numel(), stream)

    def _restore(self):
        # the kernel solves in place: reload the warm start before every launch
        self.call.states.copy_(self._guess_states)
        self.call.controls.copy_(self._guess_controls)
        self.call.dual.copy_(self._guess_dual)
        self.call.conv.copy_(self._guess_conv)

    def __call__(self, initial_state: Optional[torch.Tensor] = None, warm_start: Optional[SQPSolution] = None) -> SQPSolution:
        if initial_state is not None:
            self.call.x0.copy_(initial_state.reshape(self.call.x0.shape))
        if warm_start is not None:
            self._guess_states.copy_(warm_start.states.reshape(self._guess_states.shape))
            self._guess_controls.copy_(warm_start.controls.reshape(self._guess_controls.shape))
            self._guess_dual.copy_(warm_start.dual.reshape(self._guess_dual.shape))
        self.graph.replay()
        c = self.call
        return SQPSolution(c.states, c.controls, c.dual, None, None, None, c.status, c.num_iter, c.conv,
                           c.conv_hist, c.alpha_hist, c.pcg_hist, None, c.lin_states, c.lin_controls)


class CapturedStep:
    """One CUDA graph of a whole step: ``fn()`` run once under capture, then ``replay()``.

    ``fn`` takes no arguments.  It reads its inputs from tensors that outlive the capture (the
    caller refills them in place between replays) and returns the tensors it produced (solution,
    loss, gradients); it must not synchronise with the host (no ``.item()``, ``.cpu()`` or
    printing of device values).  Take gradients with ``torch.autograd.grad`` rather than
    ``backward()``: ``.grad`` accumulation would be captured as an accumulation.  ``warmup``
    eager calls on a side stream come first: they set the kernels' launch attributes and
    allocate the solver workspace and autograd buffers outside the capture.  ``replay()``
    re-runs every captured launch (the solver kernels, their workspace resets and the loss's
    torch kernels) and returns the tensors ``fn`` returned during capture, refreshed in place.
    """

    def __init__(self, fn, warmup: int = 3, device=None):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.fn = fn
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(max(1, int(warmup))):
                fn()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
            self.outputs = fn()

    def replay(self):
        self.graph.replay()
        return self.outputs

    __call__ = replay

