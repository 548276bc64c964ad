"""SQP solver front end (mirror of diffmpc/solvers/sqp.py) on the B200 library.

``SQPSolver.solve(initial_guess, problem_params, weights)`` has the reference's
signature and semantics (sqp.py:436-560 forward, sqp.py:562-802 custom VJP):
gradients flow to ``weights`` only, ``initial_guess`` and ``problem_params``
are treated as constants, and the cotangent of ``dual_backward_guess`` carries
the adjoint multipliers back (the reference's warm-start threading through
``lax.scan``).  Inputs are torch tensors; a leading batch dimension solves a
batch in one kernel launch (the reference batches with ``jax.vmap``).

The forward solve writes the iterate of the last linearization; the adjoint
recomputes the Schur blocks from it instead of storing them.
"""

import copy
import enum
from typing import Any, Dict, NamedTuple

import torch

from . import _lib
from .pcg import (PCGOptimalControl, QPCostParameters, QPDynamicsCostPremultipliedMatrices,
                  QPDynamicsParameters, QPParameters)
from .problem import OptimalControlProblem, load_solver_params

DEFAULT_SOLVER_PARAMS = load_solver_params("sqp.yaml")


class SolverReturnStatus(enum.IntEnum):  # sqp.py:31-35
    SUCCESS = 0
    ERROR = -100


class SQPSolution(NamedTuple):  # sqp.py:38-57
    states: torch.Tensor
    controls: torch.Tensor
    dual: torch.Tensor
    qp_parameters: Any
    dynamics_cost_premultiplied_matrices: Any
    schur_complement_matrices: Any
    status: torch.Tensor
    num_iter: torch.Tensor
    convergence_error: torch.Tensor
    convergence_errors: torch.Tensor
    linesearch_alphas: torch.Tensor
    num_pcg_iters: torch.Tensor
    dual_backward_guess: torch.Tensor = None
    # iterate at which the last QP was linearized (the adjoint rebuilds S, Phi^-1 there)
    linearization_states: torch.Tensor = None
    linearization_controls: torch.Tensor = None


COST_GRAD_KEYS = {
    "initial_state": "g_initial_state",
    "final_state": "g_final_state",
    "weights_penalization_reference_state_trajectory": "g_w_x",
    "weights_penalization_control_squared": "g_w_u",
    "weights_penalization_final_state": "g_w_f",
    "reference_state_trajectory": "g_reference_state",
    "reference_control_trajectory": "g_reference_control",
}


def solver_params_struct(params: Dict[str, Any]) -> _lib.SolverParams:
    """Reference solver dict (sqp.yaml keys) -> C struct."""
    p = _lib.SolverParams()
    lib = _lib.load()
    lib.dmpc_default_params(p)
    p.tol_convergence = float(params.get("tol_convergence", 1e-8))
    p.num_scp_iteration_max = int(params.get("num_scp_iteration_max", 15))
    p.linesearch = 1 if params.get("linesearch", False) else 0
    p.linesearch_eta = float(params.get("linesearch_eta", 0.4))
    alphas = list(params.get("linesearch_alphas", [0.01, 0.1, 0.3, 0.7, 1.0]))
    if not 1 <= len(alphas) <= _lib.DMPC_MAX_ALPHAS:
        raise ValueError(f"linesearch_alphas must have 1..{_lib.DMPC_MAX_ALPHAS} entries")
    p.n_alphas = len(alphas)
    for i, a in enumerate(alphas):
        p.alphas[i] = float(a)
    p.warm_start_backward = 1 if params.get("warm_start_backward", True) else 0
    pcg = params.get("pcg", {})
    p.pcg_max_iter = int(pcg.get("max_iter", 10000))
    p.pcg_tol_epsilon = float(pcg.get("tol_epsilon", 1e-9))
    prec = params.get("precision", "mixed")
    p.precision = _lib.PREC_FP64 if prec in ("fp64", _lib.PREC_FP64) else _lib.PREC_MIXED
    p.max_refinement = int(params.get("max_refinement", 30))
    p.inner_rel_tol = float(params.get("inner_rel_tol", 1e-3))
    p.threads_per_block = int(params.get("threads_per_block", 0))
    p.blocks_in_smem = int(params.get("blocks_in_smem", -1))
    p.cta_config = int(params.get("cta_config", 0))
    return p


def _ptr(t):
    return 0 if t is None else t.data_ptr()


def _batched(v, base_shape, B, device, dtype=torch.float64):
    """Broadcast a shared (base_shape) or per-instance (B, *base_shape) value to (B, *base).  A
    Python number is filled on the device (no host-to-device copy, so that the call can be
    captured in a CUDA graph)."""
    if isinstance(v, (int, float)) and not isinstance(v, bool):
        return torch.full((B, *base_shape), float(v), dtype=dtype, device=device)
    t = torch.as_tensor(v, dtype=dtype, device=device)
    n = 1
    for s in base_shape:
        n *= s
    if t.numel() == n:
        return t.reshape(1, *base_shape).expand(B, *base_shape).contiguous()
    return t.reshape(B, *base_shape).contiguous()


class _Call:
    """Per-call device buffers of one group and the C descriptor that points at them."""

    def __init__(self, solver, guess, params, B, device):
        prog = solver.program
        dyn = prog.dynamics
        nx, nu, N = prog.num_state_variables, prog.num_control_variables, prog.horizon
        K = N + 1
        mi = solver.maxiter
        self.B, self.K, self.nx, self.nu, self.N = B, K, nx, nu, N
        f = lambda v, *shape: _batched(v, shape, B, device)  # noqa: E731
        self.dt = f(params["discretization_resolution"])
        self.x0 = f(params["initial_state"], nx)
        self.xf = f(params["final_state"], nx)
        self.xref = f(params["reference_state_trajectory"], K, nx)
        self.uref = f(params["reference_control_trajectory"], K, nu)
        self.wx = f(params["weights_penalization_reference_state_trajectory"], nx)
        self.wu = f(params["weights_penalization_control_squared"], nu)
        self.wf = f(params["weights_penalization_final_state"], nx)
        self.mp = dyn.pack_params(params, B, device)
        hz = params.get("horizons", None)
        self.horizons = None
        if hz is not None:
            t = torch.as_tensor(hz)
            if t.device.type == "cpu" and t.numel() > 0 and (int(t.min()) < 1 or int(t.max()) > N):
                raise ValueError("per-instance horizons must lie in [1, horizon]")
            # a device tensor is not read back (no host sync): the kernels mark an instance
            # whose horizon lies outside [1, horizon] with status ERROR and leave it unsolved
            self.horizons = t.to(device=device, dtype=torch.int32).reshape(B).contiguous()
        # guess -> outputs (the kernel works in place)
        self.states = f(guess.states, K, nx).clone()
        self.controls = f(guess.controls, K, nu).clone()
        self.dual = f(guess.dual, K, nx).clone()
        ce = guess.convergence_error
        self.conv = f(0.0 if ce is None else ce).clone()
        self.status = torch.zeros(B, dtype=torch.int32, device=device)
        self.num_iter = torch.zeros(B, dtype=torch.int32, device=device)

        def hist(v, dtype):
            if v is not None:
                t = torch.as_tensor(v, device=device)
                if t.shape[-1] == mi:
                    return _batched(t, (mi,), B, device, dtype).clone()
            return torch.zeros(B, mi, dtype=dtype, device=device)

        self.conv_hist = hist(guess.convergence_errors, torch.float64)
        self.alpha_hist = hist(guess.linesearch_alphas, torch.float64)
        self.pcg_hist = hist(guess.num_pcg_iters, torch.int32)
        # per QP solve: FP64 residual replacements, and iterations of the FP64 recurrence
        self.pcg_record = torch.zeros(2, B, mi, dtype=torch.int32, device=device)
        self.lin_states = torch.empty(B, K, nx, dtype=torch.float64, device=device)
        self.lin_controls = torch.empty(B, K, nu, dtype=torch.float64, device=device)
        g = _lib.Group()
        g.model = dyn.model_id
        g.nx, g.nu, g.horizon, g.batch = nx, nu, N, B
        g.scheme = prog.discretization_scheme
        g.penalize_control_reference = 1 if prog.penalize_control_reference else 0
        g.n_model_params = dyn.num_model_params()
        g.horizons = _ptr(self.horizons)
        g.dt, g.initial_state, g.final_state = _ptr(self.dt), _ptr(self.x0), _ptr(self.xf)
        g.reference_state, g.reference_control = _ptr(self.xref), _ptr(self.uref)
        g.w_x, g.w_u, g.w_f, g.model_params = _ptr(self.wx), _ptr(self.wu), _ptr(self.wf), _ptr(self.mp)
        g.states, g.controls, g.dual = _ptr(self.states), _ptr(self.controls), _ptr(self.dual)
        g.convergence_error, g.status, g.num_iter = _ptr(self.conv), _ptr(self.status), _ptr(self.num_iter)
        g.convergence_errors, g.linesearch_alphas = _ptr(self.conv_hist), _ptr(self.alpha_hist)
        g.num_pcg_iters = _ptr(self.pcg_hist)
        g.lin_states, g.lin_controls = _ptr(self.lin_states), _ptr(self.lin_controls)
        g.num_pcg_corrections, g.num_pcg_fp64_iters = _ptr(self.pcg_record[0]), _ptr(self.pcg_record[1])
        self.group = g


class AdjointSpec:
    """dmpc_adjoint descriptor of one group plus the device buffers it points at.

    Gradients of the cost keys come from the first launch; model-parameter gradients
    are requested in chunks of at most DMPC_MAX_PARAM_GRADS indices per launch."""

    def __init__(self, dyn, call, g_states, g_controls, g_dbg, keys):
        dev = call.states.device
        B, K, nx, nu = call.B, call.K, call.nx, call.nu
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=dev)  # noqa: E731
        self.dlx = (g_states if g_states is not None else z(B, K, nx)).to(torch.float64).contiguous()
        self.dlu = (g_controls if g_controls is not None else z(B, K, nu)).to(torch.float64).contiguous()
        self.dbg = None if g_dbg is None else g_dbg.to(torch.float64).contiguous()
        self.dual_backward = z(B, K, nx)
        self.adj_iters = torch.zeros(B, dtype=torch.int32, device=dev)
        self.adj_record = torch.zeros(2, B, dtype=torch.int32, device=dev)
        adj = _lib.Adjoint()
        adj.num_pcg_iter = self.adj_iters.data_ptr()
        adj.num_pcg_corrections, adj.num_pcg_fp64_iter = self.adj_record[0].data_ptr(), self.adj_record[1].data_ptr()
        adj.dl_dstates, adj.dl_dcontrols = self.dlx.data_ptr(), self.dlu.data_ptr()
        adj.dual_backward_guess = _ptr(self.dbg)
        adj.dual_backward = self.dual_backward.data_ptr()
        shapes = {
            "g_initial_state": (B, nx), "g_final_state": (B, nx), "g_w_x": (B, nx), "g_w_u": (B, nu),
            "g_w_f": (B, nx), "g_reference_state": (B, K, nx), "g_reference_control": (B, K, nu),
        }
        self.keys = list(keys)
        self.slices = dyn.param_slices()
        self.bufs = {}
        param_idx = []
        for k in self.keys:
            if k in COST_GRAD_KEYS:
                f = COST_GRAD_KEYS[k]
                self.bufs[k] = z(*shapes[f])
                setattr(adj, f, self.bufs[k].data_ptr())
            elif k in self.slices:
                sl = self.slices[k]
                param_idx.extend(range(sl.start, sl.stop))
            else:
                raise NotImplementedError(f"gradient with respect to '{k}' is not supported")
        m = _lib.DMPC_MAX_PARAM_GRADS
        self.chunks = [param_idx[i:i + m] for i in range(0, len(param_idx), m)] or [[]]
        self.chunk_bufs = [z(B, max(1, len(c))) for c in self.chunks]
        self.chunk_idx = [(_lib.ctypes.c_int32 * max(1, len(c)))(*c) for c in self.chunks]
        self.adj = adj

    @property
    def n_chunks(self):
        return len(self.chunks)

    def select_chunk(self, ci):
        adj = self.adj
        chunk = self.chunks[ci]
        adj.n_param_grads = len(chunk)
        adj.param_grad_index = self.chunk_idx[ci]
        adj.g_model_params = self.chunk_bufs[ci].data_ptr() if chunk else 0
        if ci > 0:  # cost-key gradients were produced by the first launch
            for f in COST_GRAD_KEYS.values():
                setattr(adj, f, 0)

    def gradients(self):
        out = {"__dual_backward__": self.dual_backward}
        out.update(self.bufs)
        per_index = {}
        for chunk, buf in zip(self.chunks, self.chunk_bufs):
            for j, idx in enumerate(chunk):
                per_index[idx] = buf[:, j]
        for k in self.keys:
            if k in self.slices:
                sl = self.slices[k]
                out[k] = torch.stack([per_index[i] for i in range(sl.start, sl.stop)], dim=1)
        return out


class _SQPFunction(torch.autograd.Function):
    """custom_vjp of the solve (sqp.py:572-802): forward = dmpc_solve_fwd, backward = dmpc_solve_adj."""

    @staticmethod
    def forward(ctx, solver, guess, problem_params, keys, holder, dbg, *vals):
        params = dict(problem_params)
        params.update({k: v.detach() for k, v in zip(keys, vals)})
        B = guess.states.shape[0]
        call = _Call(solver, guess, params, B, guess.states.device)
        solver._run_fwd(call)
        holder["call"] = call
        ctx.solver = solver
        ctx.call = call
        ctx.keys = keys
        ctx.shapes = [v.shape for v in vals]
        return call.states.clone(), call.controls.clone(), call.dual.clone(), dbg.detach().clone()

    @staticmethod
    def backward(ctx, g_states, g_controls, g_dual, g_dbg):
        call = ctx.call
        grads = ctx.solver._run_adj(call, g_states, g_controls, g_dbg, ctx.keys)
        out = []
        for k, shape in zip(ctx.keys, ctx.shapes):
            g = grads.get(k)
            if g is None:
                out.append(None)
                continue
            n = 1
            for s in shape:
                n *= s
            g = g.reshape(call.B, -1)
            if g.shape[1] == n:  # shared across the batch
                out.append(g.sum(0).reshape(shape))
            else:
                out.append(g.reshape(shape))
        return (None, None, None, None, None, grads["__dual_backward__"]) + tuple(out)


class SQPSolver:
    """Mirror of SQPSolver (sqp.py:60-802) backed by libdmpc.so."""

    _supported_program_types = [OptimalControlProblem]

    def __init__(self, program: OptimalControlProblem, name: str = "SQPSolver", params: Dict = None, device=None):
        if params is None:
            params = copy.deepcopy(DEFAULT_SOLVER_PARAMS)
        if params.get("verbose", False):
            print("Initializing Solver with")
            print("> name    =", name)
            print("> program =", program)
        if not any(isinstance(program, t) for t in self._supported_program_types):
            raise NotImplementedError(str(getattr(program, "name", program)) + " is not supported.")
        self._verbose = params.get("verbose", False)
        self._params = params
        self._program = program
        self._name = name
        self._device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device() if torch.cuda.is_available() else 0)
        self._pcg = PCGOptimalControl(
            program.horizon, program.num_state_variables, program.num_control_variables, params["pcg"]
        )
        self._c_params = solver_params_struct(params)
        self._ws = None
        # optional list collecting (name, start_event, end_event) around each kernel launch
        self.kernel_events = None
        # adjoint PCG iteration counts of the most recent backward pass, (B,) int32
        self.last_adjoint_pcg_iters = None
        # precision record of the most recent forward solve, (2, B, num_scp_iteration_max) int32:
        # [0] FP64 residual replacements of each QP's FP32 PCG, [1] iterations of the FP64
        # recurrence (all of num_pcg_iters in FP64; > 0 in mixed precision when the FP32 PCG
        # handed the QP over); and of the most recent backward pass, (2, B)
        self.last_forward_pcg_record = None
        self.last_adjoint_pcg_record = None
        self.solve = self._solve_differentiable

    # -- properties (sqp.py:100-133) ------------------------------------------
    @property
    def name(self) -> str:
        return self._name

    @property
    def params(self) -> Dict:
        return self._params

    @property
    def problem_params(self) -> Dict:
        return self._program.params

    @property
    def maxiter(self) -> int:
        return int(self._params["num_scp_iteration_max"])

    @property
    def program(self) -> OptimalControlProblem:
        return self._program

    @property
    def verbose(self) -> bool:
        return self._verbose

    @property
    def pcg(self) -> PCGOptimalControl:
        return self._pcg

    # -- guesses (sqp.py:135-158) ------------------------------------------------
    def initial_guess_primal(self, params=None):
        return self._program.initial_guess(params, device=self._device)

    def initial_guess_dual(self, batch=()):
        p = self._program
        return torch.zeros(*batch, p.horizon + 1, p.num_state_variables, dtype=torch.float64, device=self._device)

    def initial_guess(self, params=None) -> SQPSolution:
        x, u = self.initial_guess_primal(params)
        lead = tuple(x.shape[:-2])
        mi = self.maxiter
        dev = self._device
        return SQPSolution(
            x,
            u,
            self.initial_guess_dual(lead),
            None,
            None,
            None,
            torch.zeros(lead, dtype=torch.int32, device=dev),
            torch.zeros(lead, dtype=torch.int32, device=dev),
            torch.zeros(lead, dtype=torch.float64, device=dev),
            torch.zeros(*lead, mi, dtype=torch.float64, device=dev),
            torch.zeros(*lead, mi, dtype=torch.float64, device=dev),
            torch.zeros(*lead, mi, dtype=torch.int32, device=dev),
            self.initial_guess_dual(lead),
        )

    def make_params_with_weights(self, weights, problem_params=None):
        new = copy.copy(self.problem_params if problem_params is None else problem_params)
        for k, v in weights.items():
            new[k] = v
        return new

    # -- library calls -----------------------------------------------------------
    def _workspace(self, nbytes, device):
        if self._ws is None or self._ws.numel() < nbytes or self._ws.device != device:
            self._ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
        return self._ws

    def _run_fwd(self, call: _Call):
        lib = _lib.load()
        n = lib.dmpc_workspace_size(1, call.group, self._c_params)
        if n == 0 and call.B > 0:
            raise ValueError("invalid problem description for the B200 solver")
        ws = self._workspace(n, call.states.device)
        stream = torch.cuda.current_stream(call.states.device).cuda_stream
        ev = self._event_pair()
        _lib.check(lib.dmpc_solve_fwd(1, call.group, self._c_params, ws.data_ptr(), ws.numel(), stream), "dmpc_solve_fwd")
        self._event_end(ev, "k_sqp_fwd")
        self.last_forward_pcg_record = call.pcg_record

    def _event_pair(self):
        if self.kernel_events is None:
            return None
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record()
        return e0

    def _event_end(self, e0, name):
        if e0 is None:
            return
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record()
        self.kernel_events.append((name, e0, e1))

    def _run_adj(self, call: _Call, g_states, g_controls, g_dbg, keys):
        lib = _lib.load()
        dev = call.states.device
        spec = AdjointSpec(self._program.dynamics, call, g_states, g_controls, g_dbg, keys)
        ws_n = lib.dmpc_workspace_size(1, call.group, self._c_params)
        ws = self._workspace(ws_n, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        for ci in range(spec.n_chunks):
            spec.select_chunk(ci)
            ev = self._event_pair()
            _lib.check(
                lib.dmpc_solve_adj(1, call.group, spec.adj, self._c_params, ws.data_ptr(), ws.numel(), stream),
                "dmpc_solve_adj",
            )
            self._event_end(ev, "k_sqp_adj")
        self.last_adjoint_pcg_iters = spec.adj_iters
        self.last_adjoint_pcg_record = spec.adj_record
        return spec.gradients()

    # -- solve (sqp.py:436-560, 562-802) -------------------------------------------
    def _solve_differentiable(self, initial_guess: SQPSolution, problem_params: Dict = None, weights: Dict = None):
        if problem_params is None:
            problem_params = self.problem_params
        weights = weights or {}
        unbatched = initial_guess.states.dim() == 2
        g = initial_guess
        if unbatched:
            g = g._replace(
                states=g.states[None],
                controls=g.controls[None],
                dual=g.dual[None],
                convergence_error=None if g.convergence_error is None else torch.as_tensor(g.convergence_error).reshape(1),
                convergence_errors=None if g.convergence_errors is None else torch.as_tensor(g.convergence_errors)[None],
                linesearch_alphas=None if g.linesearch_alphas is None else torch.as_tensor(g.linesearch_alphas)[None],
                num_pcg_iters=None if g.num_pcg_iters is None else torch.as_tensor(g.num_pcg_iters)[None],
                dual_backward_guess=None if g.dual_backward_guess is None else g.dual_backward_guess[None],
            )
        dev = g.states.device
        B = g.states.shape[0]
        dbg = g.dual_backward_guess
        if dbg is None:
            dbg = torch.zeros_like(g.dual, dtype=torch.float64)
        keys = sorted(weights.keys())
        vals = [torch.as_tensor(weights[k], dtype=torch.float64, device=dev) for k in keys]
        holder = {}
        states, controls, dual, dbg_out = _SQPFunction.apply(self, g, problem_params, keys, holder, dbg, *vals)
        c = holder["call"]
        qp = premult = schur = None
        if self._params.get("return_qp_matrices", False) and c.horizons is None:
            qp, premult, schur = self.qp_matrices(c)
        sol = SQPSolution(
            states, controls, dual, qp, premult, schur,
            c.status, c.num_iter, c.conv, c.conv_hist, c.alpha_hist, c.pcg_hist, dbg_out,
            c.lin_states, c.lin_controls,
        )
        if unbatched:
            first = lambda v: v[0] if isinstance(v, torch.Tensor) and v.dim() > 0 else v  # noqa: E731
            sol = SQPSolution(*[
                None if v is None else (type(v)(*[type(w)(*[first(x) for x in w]) if isinstance(w, tuple) else first(w)
                                                  for w in v]) if isinstance(v, tuple) else first(v))
                for v in sol])
        return sol

    def qp_matrices(self, call):
        """QP data of the last SQP iteration, as the reference keeps it in SQPSolution
        (qp_parameters, dynamics_cost_premultiplied_matrices, schur_complement_matrices;
        sqp.py:44-46, set by each iteration of _solve, :436-560): the linearization at the
        iterate the last QP was built at (dmpc_linearize), A_next = -I, the premultiplied
        products (sqp.py:247-254) and S, Phi^-1 (dmpc_schur_assemble).  Uniform horizons only."""
        lib = _lib.load()
        B, K, nx, nu, N = call.B, call.K, call.nx, call.nu, call.N
        dev = call.states.device
        g = _lib.Group.from_buffer_copy(call.group)
        g.states, g.controls = call.lin_states.data_ptr(), call.lin_controls.data_ptr()
        e = lambda *sh: torch.empty(*sh, dtype=torch.float64, device=dev)  # noqa: E731
        As, Bs, Cs, Qinv, qvec = e(B, N, nx, nx), e(B, N, nx, nu), e(B, K, nx), e(B, K, nx, nx), e(B, K, nx)
        Rinv, rvec = e(B, N, nu, nu), e(B, N, nu)
        n = lib.dmpc_workspace_size(1, g, self._c_params)
        ws = self._workspace(n, dev)
        _lib.check(lib.dmpc_linearize(g, self._c_params, As.data_ptr(), Bs.data_ptr(), Cs.data_ptr(), Qinv.data_ptr(),
                                      qvec.data_ptr(), Rinv.data_ptr(), rvec.data_ptr(), ws.data_ptr(), ws.numel(),
                                      torch.cuda.current_stream(dev).cuda_stream), "dmpc_linearize")
        As_next = -torch.eye(nx, dtype=torch.float64, device=dev).expand(B, N, nx, nx).contiguous()
        qp = QPParameters(QPDynamicsParameters(As_next, As, Bs, Cs), QPCostParameters(Qinv, qvec, Rinv, rvec))
        premult = QPDynamicsCostPremultipliedMatrices(As @ Qinv[:, :-1], As_next @ Qinv[:, 1:], Bs @ Rinv)
        return qp, premult, self._pcg.compute_S_Phiinv(qp)
