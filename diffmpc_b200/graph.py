"""CUDA-graph capture of the forward solve.

For a closed-loop controller that re-solves the same problem shape every control
period (the reference's ``lax.scan`` rollouts), the per-call host work matters:
building descriptors and launching.  ``GraphedForward`` captures ONE
``dmpc_solve_fwd`` launch on static device buffers.  Each call then copies the new
initial state and warm start into those buffers and replays the graph: one graph
launch, no host-side descriptor building.

It is not differentiable.  Use ``SQPSolver.solve`` when gradients are needed.
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
