#!/usr/bin/env python
"""Benchmark: batched forward + adjoint MPC solves/s, quadrotor N=60 (K=61 knots), B=4096.

One step = one batched SQP forward solve (``k_sqp_fwd``: linearize -> Schur
assembly -> PCG -> recover, up to 15 SQP iterations) of 4096 quadrotor MPC
instances plus the hand-written adjoint (``k_sqp_adj``) of the loss
``sum_i ||u_0^i||^2`` with respect to x0, the diag(Q)/diag(R) log-weights and
the mass.  Synthetic, seeded inputs (``diffmpc_b200.workloads.quadrotor``).
PCG tolerance 1e-20 (absolute, on eta = r^T Phi^-1 r): the QPs are solved to
where the 1e-6 control parity against the all-FP64 path is well defined; the
line's ``parity`` block reports it over the whole batch beside two FP64-vs-FP64
controls.

Contract: ``python bench.py --gpus N --steps K --warmup W`` prints ONE JSON line
on rank 0.  N > 1 runs under torchrun, one process per GPU, each rank solving
its own batch of 4096 (weak scaling, no data-path collective: instances are
independent).  ``--impl reference`` times the reference algorithm's CPU
implementation (the float64 oracle restatement; the JAX reference cannot be
installed offline) on the host cores, one instance per step.
"""

import argparse
import copy
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd MPC solves/s, quadrotor T=60 B=4096, vs plain FP64 GPU @1e-6 rel"
WORKLOAD = "quadrotor N=60 (K=61), RK4 dt=0.05, fwd SQP (<=15 it, tol 1e-8) + adjoint, loss sum u0^2"
UNIT = "solves/s"
GRAD_KEYS = ("initial_state", "weights_penalization_reference_state_trajectory",
             "weights_penalization_control_squared", "mass")


CTA_CONFIGS = {"auto": 0, "wide": 1, "rows": 2, "dual": 3}  # DMPC_CTA_*


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--horizon", type=int, default=60)
    ap.add_argument("--pcg-tol", type=float, default=1e-20)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--pcg-max-iter", type=int, default=0, help="pcg.max_iter (0: the workload's own)")
    ap.add_argument("--cpu-sample", type=int, default=16, help="instances per CPU-baseline run (and pool size cap)")
    ap.add_argument("--cpu-runs", type=int, default=3, help="CPU-baseline runs (median reported)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--fp64-sample", type=int, default=8, help="instances timed one-per-launch in FP64")
    ap.add_argument("--no-extras", action="store_true", help="skip cpu baseline / fp64 / e2e legs")
    ap.add_argument("--no-other", action="store_true", help="skip the other workload shapes in the headline run")
    ap.add_argument("--cta-config", default="auto", choices=["auto", "wide", "rows", "dual"],
                    help="CTA shape of the solver kernels (dmpc_solver_params.cta_config)")
    ap.add_argument("--threads", type=int, default=0,
                    help="dmpc_solver_params.threads_per_block (0: automatic)")
    ap.add_argument("--blocks-in-smem", type=int, default=-1, choices=[-1, 0, 1],
                    help="dmpc_solver_params.blocks_in_smem (-1: shared memory when they fit)")
    ap.add_argument("--workload", default="quadrotor", choices=["quadrotor", "attitude", "mixed", "stress", "rollout", "rollout_spacecraft"],
                    help="quadrotor = the headline; the others report the remaining workload shapes")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None):
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        if device is not None and device.type == "cuda":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons every 200 ms while active."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ workload
def launch_shape(sp, args):
    """The launch-shape overrides of the command line (automatic by default)."""
    sp["cta_config"] = CTA_CONFIGS[args.cta_config]
    sp["threads_per_block"] = args.threads
    sp["blocks_in_smem"] = args.blocks_in_smem


def build(args, rank):
    from diffmpc_b200 import workloads

    dyn, st, bt, sp = workloads.quadrotor(B=args.batch, N=args.horizon, seed=1002 + rank)
    sp["precision"] = args.precision
    sp["pcg"]["tol_epsilon"] = args.pcg_tol
    launch_shape(sp, args)
    return dyn, st, bt, sp


def algorithmic_flops(nx, nu, N, B, sqp_iters, pcg_iters, adj_pcg_iters, rk4=True):
    """Algorithmic FLOPs of the reference's dense algorithm for the executed iteration
    counts (totals over the batch of B instances): F_pcg = 12 K nx^2 + 10 K nx per PCG
    iteration, F_setup = K (16 nx^3 + 4 nx^2 nu) per QP assembly, F_lin = N (nx + nu) s F_f
    per linearization (s = 4 for RK4, F_f = 130 flops for the quadrotor state_dot).  The
    adjoint assembles once per instance.  Also returns the FLOPs the scaled-basis FP32
    iteration executes, 8 K nx^2 + 12 K nx (two off-diagonal block matvecs, unit diagonal)."""
    K = N + 1
    f_pcg = 12 * K * nx * nx + 10 * K * nx
    f_pcg_exec = 8 * K * nx * nx + 12 * K * nx
    f_setup = K * (16 * nx**3 + 4 * nx * nx * nu)
    f_lin = N * (nx + nu) * (4 if rk4 else 1) * 130
    fwd = sqp_iters * (f_setup + f_lin) + pcg_iters * f_pcg
    adj = B * (f_setup + f_lin) + adj_pcg_iters * f_pcg
    fwd_exec = sqp_iters * (f_setup + f_lin) + pcg_iters * f_pcg_exec
    return fwd, adj, f_pcg, fwd_exec


def fp32_peak_tflops(torch, lib):
    """Measured FP32 FMA throughput of this GPU (libdmpc's probe kernel, CUDA events)."""
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    blocks = props.multi_processor_count * 8
    out = torch.zeros(blocks, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    lib.dmpc_probe_fp32_fma(blocks, 256, out.data_ptr(), stream)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        flops = lib.dmpc_probe_fp32_fma(blocks, 4096, out.data_ptr(), stream)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, flops / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def headline_step(solver, params):
    """One step of the headline: batched forward solve + adjoint of sum ||u_0||^2 with respect to
    x0, the diagonal log-weights and the mass.  Returns (solution, gradients)."""
    import torch

    lw_x = torch.log(params["weights_penalization_reference_state_trajectory"]).detach().requires_grad_(True)
    lw_u = torch.log(params["weights_penalization_control_squared"]).detach().requires_grad_(True)
    x0 = params["initial_state"].detach().clone().requires_grad_(True)
    mass = params["mass"].detach().clone().requires_grad_(True)
    weights = {
        "initial_state": x0,
        "weights_penalization_reference_state_trajectory": torch.exp(lw_x),
        "weights_penalization_control_squared": torch.exp(lw_u),
        "mass": mass,
    }
    guess = solver.initial_guess(params)
    sol = solver.solve(guess, params, weights)
    loss = (sol.controls[:, 0] ** 2).sum()
    loss.backward()
    return sol, {"initial_state": x0.grad, "log_w_x": lw_x.grad, "log_w_u": lw_u.grad, "mass": mass.grad}


def _grad_matrix(grads):
    """(B, 31) per-instance gradient vector: x0, log w_x, log w_u, mass."""
    import torch

    B = grads["initial_state"].shape[0]
    return torch.cat([grads[k].detach().reshape(B, -1) for k in ("initial_state", "log_w_x", "log_w_u", "mass")], 1)


def _rel_per_instance(a, b):
    """max |a - b| / max |b| per instance (leading dimension)."""
    B = a.shape[0]
    a, b = a.detach().double().reshape(B, -1), b.detach().double().reshape(B, -1)
    return (a - b).abs().amax(1) / b.abs().amax(1).clamp_min(1e-300)


def _dist(v, bar):
    import torch

    v = v.double().cpu()
    return {"p50": float(torch.quantile(v, 0.5)), "p99": float(torch.quantile(v, 0.99)), "max": float(v.max()),
            "n_above_bar": int((v > bar).sum()), "bar": bar}


def _sqp_stats(sol):
    import torch

    c = sol.convergence_error.double().cpu()
    return {"status_success": int((sol.status == 0).sum()), "conv_err_p50": float(torch.quantile(c, 0.5)),
            "conv_err_p90": float(torch.quantile(c, 0.9)),
            "pcg_iters_per_instance": float(sol.num_pcg_iters.double().sum() / sol.status.numel())}


def precision_record(solver, sol):
    """What the FP64 corrections of the mixed PCG did in the solver's last step: FP64 residual
    replacements per QP solve, the QP solves the FP32 PCG handed to the FP64 recurrence, and the
    FP64 recurrence's share of all PCG iterations (forward QPs, and the adjoint QP)."""
    import torch

    rec = solver.last_forward_pcg_record
    if rec is None:
        return None
    mi = rec.shape[-1]
    ran = torch.arange(mi, device=rec.device)[None, :] < sol.num_iter.to(rec.device).long()[:, None]
    corr, f64 = rec[0][ran].double(), rec[1][ran].double()
    its = sol.num_pcg_iters.to(rec.device)[ran].double()
    out = {"qp_solves": int(ran.sum()), "replacements_per_qp": float(corr.mean()),
           "qp_handed_to_fp64": int((f64 > 0).sum()), "fp64_iter_share": float(f64.sum() / its.sum().clamp_min(1))}
    a, ai = solver.last_adjoint_pcg_record, solver.last_adjoint_pcg_iters
    if isinstance(a, torch.Tensor) and isinstance(ai, torch.Tensor):  # (per-group lists after solve_groups)
        out["adjoint"] = {"qp_solves": int(a.shape[1]), "replacements_per_qp": float(a[0].double().mean()),
                          "qp_handed_to_fp64": int((a[1] > 0).sum()),
                          "fp64_iter_share": float(a[1].double().sum() / ai.double().sum().clamp_min(1))}
    return out


def parity_block(sp, dyn, st, p, sol, grads):
    """Parity of the timed mixed-precision result over the whole batch against the all-FP64 path
    (the reference recurrence, same parameters).  Two FP64-vs-FP64 controls stand beside it for
    every instance: the FP64 path with another CTA size (another summation order of its
    reductions), and the FP64 path with a 100x tighter PCG tolerance (how far the reference's own
    answer moves inside its tolerance).  An instance above the bar is matched when either control
    moves the FP64 answer at least as much.  Also the FP64 path's device time on the batch
    (fp64_batched: what the FP32 iterations buy)."""
    import copy

    import torch

    from diffmpc_b200 import OptimalControlProblem, SQPSolver

    dev = sol.controls.device
    B = sol.controls.shape[0]
    sp64 = copy.deepcopy(sp)
    sp64["precision"] = "fp64"
    s64 = SQPSolver(OptimalControlProblem(dyn, st), params=sp64, device=dev)
    headline_step(s64, p)  # warm-up (workspace, launch attributes)
    torch.cuda.synchronize()
    s64.kernel_events = []
    sol64, g64 = headline_step(s64, p)
    torch.cuda.synchronize()
    fp64_ms = sum(a.elapsed_time(b) for _, a, b in s64.kernel_events)
    s64.kernel_events = None
    spc = copy.deepcopy(sp64)
    spc["threads_per_block"] = 384
    sc = SQPSolver(OptimalControlProblem(dyn, st), params=spc, device=dev)
    solc, gc = headline_step(sc, p)
    spt = copy.deepcopy(sp64)
    spt["pcg"] = dict(sp64["pcg"])
    spt["pcg"]["tol_epsilon"] = sp64["pcg"]["tol_epsilon"] * 1e-2
    stt = SQPSolver(OptimalControlProblem(dyn, st), params=spt, device=dev)
    solt, gt = headline_step(stt, p)
    torch.cuda.synchronize()
    u_mix = _rel_per_instance(sol.controls, sol64.controls)
    g_mix = _rel_per_instance(_grad_matrix(grads), _grad_matrix(g64))
    u_ctl = _rel_per_instance(solc.controls, sol64.controls)
    g_ctl = _rel_per_instance(_grad_matrix(gc), _grad_matrix(g64))
    u_tgt = _rel_per_instance(solt.controls, sol64.controls)
    g_tgt = _rel_per_instance(_grad_matrix(gt), _grad_matrix(g64))
    u_any, g_any = torch.maximum(u_ctl, u_tgt), torch.maximum(g_ctl, g_tgt)
    bad = torch.nonzero(u_mix > 1e-6).flatten().tolist()
    bad_g = torch.nonzero(g_mix > 1e-5).flatten().tolist()
    unexplained = [i for i in bad if float(u_any[i]) < float(u_mix[i])]
    unexplained_g = [i for i in bad_g if float(g_any[i]) < float(g_mix[i])]
    outliers = [{"i": i, "mixed": float(u_mix[i]), "fp64_reordered": float(u_ctl[i]),
                 "fp64_tighter_eps": float(u_tgt[i]), "status": int(sol.status[i]),
                 "conv_err": float(sol.convergence_error[i])} for i in bad[:12]]
    return {
        "reference": "all-FP64 GPU path (reference recurrence and stopping rule) at the same parameters, whole batch",
        "instances": B,
        "controls_mixed_vs_fp64": _dist(u_mix, 1e-6),
        "grads_mixed_vs_fp64": _dist(g_mix, 1e-5),
        "controls_fp64_vs_fp64_reordered": _dist(u_ctl, 1e-6),
        "grads_fp64_vs_fp64_reordered": _dist(g_ctl, 1e-5),
        "controls_fp64_vs_fp64_tighter_eps": _dist(u_tgt, 1e-6),
        "grads_fp64_vs_fp64_tighter_eps": _dist(g_tgt, 1e-5),
        "control_outliers_not_matched_by_fp64_controls": len(unexplained),
        "grad_outliers_not_matched_by_fp64_controls": len(unexplained_g),
        "control_outliers": outliers,
        "mixed": _sqp_stats(sol),
        "fp64": _sqp_stats(sol64),
    }, {"value": B / (fp64_ms * 1e-3), "unit": UNIT, "device_ms": fp64_ms,
        "sample": f"all {B} instances, one batched fwd + adjoint, all-FP64 PCG (device time of its kernels)"}


# ------------------------------------------------------------------ CPU oracle (process pool)
def _pool_init():
    import torch

    torch.set_num_threads(1)


def _oracle_job(job):
    """fwd + adjoint of the float64 oracle on one instance in a pool worker:
    job = (model name, nx, nu, static params, one-instance batched params, solver params)."""
    name, nx, nu, st, sub, sp = job
    import torch

    from oracle.models import make_model
    from oracle.ocp import STATIC_KEYS, OptimalControlProblem
    from oracle.sqp import SQPSolver as OracleSolver

    w = {k: sub[k] for k in GRAD_KEYS}
    t0 = time.perf_counter()
    s = OracleSolver(OptimalControlProblem(make_model(name, nx, nu), st), params=sp)
    sol = s._solve(s.initial_guess({k: v for k, v in sub.items() if k not in STATIC_KEYS}), sub, w)
    dlu = torch.zeros_like(sol.controls)
    dlu[:, 0] = 2 * sol.controls[:, 0]
    g, _, _ = s.solve_bwd(sol, w, sub, torch.zeros_like(sol.states), dlu, torch.zeros_like(sol.dual))
    return sol.controls, g, time.perf_counter() - t0


def _jobs(dyn, st, bt, sp, idx):
    from diffmpc_b200 import workloads

    return [(dyn.model_name, dyn.num_states, dyn.num_controls, st, workloads.subset(bt, slice(i, i + 1)), sp)
            for i in idx]


def oracle_pool(workers):
    """A spawn-started pool of single-threaded oracle workers (spawn: a child forked from a process
    that has touched the GPU can hang)."""
    import multiprocessing as mp

    return mp.get_context("spawn").Pool(workers, initializer=_pool_init)


def cpu_baseline(args, sol, grads, bt, dyn, st, sp, pool, workers):
    """The float64 oracle on the host cores: `workers` single-threaded processes, runs of
    `args.cpu_sample` instances, median of `args.cpu_runs` runs; the oracle's controls and gradients
    of every sampled instance are compared with the timed GPU result."""
    import torch

    S, R = args.cpu_sample, args.cpu_runs
    pool.map(_oracle_job, _jobs(dyn, st, bt, sp, range(workers)))  # warm-up: imports, first solve per worker
    walls, rel_c, rel_g = [], [], []
    gm = _grad_matrix(grads).cpu()
    for r in range(R):
        idx = [(r * S + j) % args.batch for j in range(S)]
        t0 = time.perf_counter()
        outs = pool.map(_oracle_job, _jobs(dyn, st, bt, sp, idx))
        walls.append(time.perf_counter() - t0)
        for i, (c, g, _) in zip(idx, outs):
            gpu_c = sol.controls[i:i + 1].detach().cpu()
            rel_c.append(float((gpu_c - c).abs().max() / c.abs().max()))
            og = torch.cat([g["initial_state"].reshape(1, -1),
                            (g["weights_penalization_reference_state_trajectory"] *
                             bt["weights_penalization_reference_state_trajectory"][i:i + 1]).reshape(1, -1),
                            (g["weights_penalization_control_squared"] *
                             bt["weights_penalization_control_squared"][i:i + 1]).reshape(1, -1),
                            g["mass"].reshape(1, -1)], 1)
            rel_g.append(float((gm[i:i + 1] - og).abs().max() / og.abs().max()))
    med = statistics.median(walls)
    return {
        "value": S / med, "unit": UNIT, "cores": workers, "kind": "port",
        "sample": f"{S} instances per run on {workers} single-threaded processes, median of {R} runs "
                  f"(instances 0..{R * S - 1}), fwd+adjoint, float64 oracle restatement (torch CPU)",
        "run_seconds": walls,
        "oracle_check": {"instances": len(rel_c), "max_rel_control_err": max(rel_c), "max_rel_grad_err": max(rel_g),
                         "bars": {"controls": 1e-6, "grads": 1e-5}},
    }


def run_ours(args):
    import copy

    import torch
    import torch.distributed as dist

    from diffmpc_b200 import OptimalControlProblem, SQPSolver, _lib, workloads

    rank, world, local = dist_env()
    # the oracle's process pool starts before the first GPU call (rank 0 only)
    workers = min(os.cpu_count() or 1, args.cpu_sample)
    pool = oracle_pool(workers) if (rank == 0 and not args.no_extras and not args.no_cpu) else None
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)
    lib = _lib.load()
    dyn, st, bt, sp = build(args, rank)
    B, N, nx, nu = args.batch, args.horizon, dyn.num_states, dyn.num_controls
    solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp, device=device)
    p = workloads.to_device(bt, device)
    l2_flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    # ---- warm-up
    for _ in range(args.warmup):
        sol, grads = headline_step(solver, p)
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs, kernel events on the launching stream
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    step_ms, fwd_ms, adj_ms = [], [], []
    barrier(device)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        l2_flush.zero_()  # > L2 (126 MB): every step starts cold
        solver.kernel_events = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sol, grads = headline_step(solver, p)
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        for name, a, b in solver.kernel_events:
            (fwd_ms if name == "k_sqp_fwd" else adj_ms).append(a.elapsed_time(b))
    barrier(device)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    solver.kernel_events = None
    total_ms = max_over_ranks(sum(step_ms), device)
    ms_per_step = total_ms / args.steps
    value = world * B * args.steps / (total_ms * 1e-3)
    gpu_launches = args.steps * 2

    # ---- roofline of the dominant kernel (k_sqp_fwd)
    sqp_iters = float(sol.num_iter.double().sum())
    pcg_iters = float(sol.num_pcg_iters.double().sum())
    adj_iters = float(solver.last_adjoint_pcg_iters.double().sum()) if solver.last_adjoint_pcg_iters is not None else 0.0
    f_fwd, f_adj, f_pcg, f_fwd_exec = algorithmic_flops(nx, nu, N, B, sqp_iters, pcg_iters, adj_iters)
    fwd_avg = statistics.mean(fwd_ms)
    peak = fp32_peak_tflops(torch, lib)
    achieved = f_fwd / (fwd_avg * 1e-3) / 1e12
    traffic = None
    prof = os.path.join(ROOT, "profiles", "k_sqp_fwd_traffic.json")
    if os.path.exists(prof):
        try:
            t = json.load(open(prof))
            if abs(float(t.get("pcg_tol_epsilon", 0.0)) - args.pcg_tol) <= 1e-3 * args.pcg_tol:
                traffic = t["dram_bytes_per_instance"] * B
        except (ValueError, KeyError):
            traffic = None
    roofline = {
        "bound": "fp32", "kernel": "k_sqp_fwd", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
        "frac": achieved / peak if peak > 0 else None, "traffic": traffic,
        "peak_source": "measured: libdmpc FP32 FMA probe on this GPU (MEASURED_PEAKS.json has no FP32 figure)",
        "algorithmic_flops_per_launch": f_fwd, "kernel_ms": fwd_avg,
        "adj_kernel_ms": statistics.mean(adj_ms) if adj_ms else None,
        "pcg_iters_per_instance": pcg_iters / B, "sqp_iters_per_instance": sqp_iters / B,
        "adj_pcg_iters_per_instance": adj_iters / B,
        "adj_achieved_tflops": (f_adj / (statistics.mean(adj_ms) * 1e-3) / 1e12) if adj_ms else None,
        "executed_flops_per_launch": f_fwd_exec,
        "executed_tflops": f_fwd_exec / (fwd_avg * 1e-3) / 1e12,
    }

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": {
            "workload": WORKLOAD,
            "batch_per_gpu": B, "horizon": N, "nx": nx, "nu": nu, "pcg_tol_epsilon": args.pcg_tol,
            "precision": args.precision, "parallelism": f"replicas x{world}",
            "l2": "512 MB buffer written between timed steps; solver workspace one slot per resident CTA",
        },
        "roofline": roofline, "clocks": clocks, "gpu_launches": gpu_launches,
        "precision_record": precision_record(solver, sol),
    }

    if not args.no_extras:
        # ---- e2e through the public API with host buffers (pinned), copies inside the region
        host = {k: (v.pin_memory() if isinstance(v, torch.Tensor) else v) for k, v in bt.items()}
        h2d = sum(v.numel() * v.element_size() for v in host.values() if isinstance(v, torch.Tensor))
        out_host = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in grads.items()}
        u0_host = torch.empty((B, nu), dtype=torch.float64, pin_memory=True)
        d2h = sum(v.numel() * v.element_size() for v in out_host.values()) + u0_host.numel() * 8
        e2e_ms = []
        for it in range(args.warmup + args.steps):
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            pd = {k: (v.to(device, non_blocking=True) if isinstance(v, torch.Tensor) else v) for k, v in host.items()}
            s2, g2 = headline_step(solver, pd)
            for k in out_host:
                out_host[k].copy_(g2[k], non_blocking=True)
            u0_host.copy_(s2.controls[:, 0], non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            if it >= args.warmup:
                e2e_ms.append(e0.elapsed_time(e1))
        e2e_total = max_over_ranks(sum(e2e_ms), device)
        line["e2e"] = {"value": world * B * args.steps / (e2e_total * 1e-3), "unit": UNIT,
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    if rank == 0 and not args.no_extras:
        # ---- whole-batch parity against the all-FP64 path, and that path's batched throughput
        line["parity"], line["fp64_batched"] = parity_block(sp, dyn, st, p, sol, grads)
        line["fp64_batched"]["speedup_of_value"] = value / (world * line["fp64_batched"]["value"])
        # ---- plain all-FP64 one-instance-per-launch GPU path (the metric's denominator)
        sp64 = copy.deepcopy(sp)
        sp64["precision"] = "fp64"
        solver64 = SQPSolver(OptimalControlProblem(dyn, st), params=sp64, device=device)
        S = min(args.fp64_sample, B)

        def one64(i):
            return headline_step(solver64, workloads.subset(p, slice(i, i + 1)))[0]

        one64(0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sols64 = [one64(i) for i in range(S)]
        e1.record()
        torch.cuda.synchronize()
        fp64_rate = S / (e0.elapsed_time(e1) * 1e-3)
        ctrl64 = torch.cat([s.controls.detach() for s in sols64]).cpu()
        rel64 = float((sol.controls[:S].detach().cpu() - ctrl64).abs().max() / ctrl64.abs().max())
        line["fp64_one_per_launch"] = {
            "value": fp64_rate, "unit": UNIT, "sample": f"{S} instances, one fwd+adj launch pair each",
            "speedup_of_value": value / (world * fp64_rate) if fp64_rate > 0 else None,
            "max_rel_control_diff_mixed_vs_fp64": rel64,
        }
        # ---- CPU baseline: float64 oracle on the host cores, with the oracle check
        if pool is not None:
            line["cpu_baseline"] = cpu_baseline(args, sol, grads, bt, dyn, st, sp, pool, workers)
        # ---- the other workload shapes, one GPU
        if world == 1 and not args.no_other:
            line["other_workloads"] = other_workloads(args)
    if pool is not None:
        pool.close()
        pool.join()

    if world > 1:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args):
    """Reference arm: the reference algorithm on the host CPU (float64 oracle restatement), one
    instance per step, the steps spread over single-threaded worker processes on every host core."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    workers = min(os.cpu_count() or 1, max(1, args.steps))
    pool = oracle_pool(workers)
    dyn, st, bt, sp = build(args, 0)
    W = max(args.warmup, workers)  # at least one warm-up per worker (imports, first solve)
    pool.map(_oracle_job, _jobs(dyn, st, bt, sp, range(W)))
    idx = [(W + j) % args.batch for j in range(args.steps)]
    t0 = time.perf_counter()
    outs = pool.map(_oracle_job, _jobs(dyn, st, bt, sp, idx))
    wall = time.perf_counter() - t0
    pool.close()
    pool.join()
    value = args.steps / wall
    per_instance = statistics.median([o[2] for o in outs])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "batch_per_gpu": args.batch, "horizon": args.horizon,
                   "pcg_tol_epsilon": args.pcg_tol, "instances_per_step": 1},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"{args.steps} instances (one per step) on {workers} single-threaded processes, "
                                   f"{W} warm-up instances first; float64 oracle restatement of the reference JAX "
                                   f"solver (JAX is not installable offline); median single-instance time "
                                   f"{per_instance:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed(fn, steps, warmup):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, out


def run_other_workload(args):
    """Throughput / precision of the non-headline workload shapes (one GPU, one line)."""
    import numpy as np
    import torch

    from diffmpc_b200 import OptimalControlProblem, SQPSolver, workloads
    from diffmpc_b200.batch import solve_groups
    from diffmpc_b200.sqp import SQPSolution

    dev = torch.device("cuda", 0)
    line = {"impl": "ours", "workload": args.workload, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "data": "synthetic"}
    if args.workload == "attitude":
        B = args.batch if args.batch != 4096 else 1024
        dyn, st, bt, sp = workloads.attitude(B=B)
        launch_shape(sp, args)
        res = {}
        for prec in ("mixed", "fp64"):
            sp2 = dict(sp, precision=prec)
            solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp2, device=dev)
            p = workloads.to_device(bt, dev)
            ms, sol = _timed(lambda: solver.solve(solver.initial_guess(p), p), args.steps, args.warmup)
            res[prec] = (ms, sol.controls.detach().cpu(), sol.num_pcg_iters.sum(dim=1).double().mean().item())
        c64 = res["fp64"][1]
        line.update(metric="batched forward MPC solves/s, attitude nx=7 N=50 B=%d, 10 SQP, eps 1e-8" % B,
                    value=B / (res["mixed"][0] * 1e-3), fp64_value=B / (res["fp64"][0] * 1e-3),
                    pcg_iters_mixed=res["mixed"][2], pcg_iters_fp64=res["fp64"][2],
                    max_rel_control_diff_mixed_vs_fp64=float((res["mixed"][1] - c64).abs().max() / c64.abs().max()))
    elif args.workload == "mixed":
        B = args.batch if args.batch != 4096 else 8192
        rng = np.random.default_rng(1003)
        groups = []
        for which in ("linear", "quadrotor"):
            if which == "linear":
                dyn, st, bt, sp = workloads.linear_lti(B=B // 2, nx=12, nu=4, N=100, seed=1013)
            else:
                dyn, st, bt, sp = workloads.quadrotor(B=B // 2, N=100, seed=1023)
            sp["pcg"]["tol_epsilon"] = args.pcg_tol
            sp["num_scp_iteration_max"] = 15
            sp["precision"] = args.precision
            solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp, device=dev)
            p = workloads.to_device(bt, dev)
            p["horizons"] = torch.tensor(rng.integers(20, 101, size=B // 2), dtype=torch.int32, device=dev)
            groups.append((solver, p))

        def step():
            probs, ws = [], []
            for solver, p in groups:
                w = p["initial_state"].clone().requires_grad_(True)
                ws.append(w)
                probs.append((solver, solver.initial_guess(p), p, {"initial_state": w}))
            sols = solve_groups(probs)
            grads = torch.autograd.grad(sum((s.controls[:, 0] ** 2).sum() for s in sols), ws)
            return sols, grads

        from diffmpc_b200.autotune import tune_step
        from diffmpc_b200.graph import CapturedStep

        # launch shape: autotuned on this step (forward + adjoint, both groups), then the whole
        # step (2 persistent launches and the loss) captured as one CUDA graph
        ms_default, _ = _timed(step, 1, 1)
        best = tune_step(groups[0][0], step, tag=f"mixed{B}", repeats=1, use_cache=False)
        ms_eager, (sols, _) = _timed(step, args.steps, args.warmup)
        cap = CapturedStep(step, warmup=args.warmup)
        ms, (sols, _) = _timed(cap.replay, args.steps, args.warmup)
        iters = torch.cat([s.num_pcg_iters.sum(dim=1) for s in sols]).double().cpu()
        line.update(metric="fwd+bwd MPC solves/s, 50% linear nx=12 / 50% quadrotor, N~U{20..100}, "
                           "one persistent launch per direction, CUDA graph, autotuned",
                    value=B / (ms * 1e-3), ms_per_step=ms, batch=B,
                    eager_solves_per_s=B / (ms_eager * 1e-3), untuned_eager_solves_per_s=B / (ms_default * 1e-3),
                    launch_shape={"cta_config": int(best[0]), "threads_per_block": int(best[1])},
                    pcg_iters_per_instance_p50=float(iters.quantile(0.5)),
                    pcg_iters_per_instance_p99=float(iters.quantile(0.99)),
                    status_success=int(sum(int((s.status == 0).sum()) for s in sols)),
                    precision_record=[precision_record(s_, sol_) for (s_, _), sol_ in zip(groups, sols)])
    elif args.workload == "rollout":
        from diffmpc_b200.rollout import ClosedLoopRollout

        B = args.batch if args.batch != 4096 else 64
        T = 50
        dyn, st, bt, sp, (A, Bm, b) = workloads.rl_linear(B=B)
        solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp, device=dev)
        p = workloads.to_device(bt, dev)
        Ad, Bd, bd = A.to(dev), Bm.to(dev), b.to(dev)
        key = "weights_penalization_reference_state_trajectory"
        roll = ClosedLoopRollout(solver, Ad, Bd, bd, T, warm_start=True)
        roll_cold = ClosedLoopRollout(solver, Ad, Bd, bd, T, warm_start=False)

        def fused(grad, r=roll):
            w = {key: p[key].clone().requires_grad_(grad)}
            c = r(p["initial_state"], p, w)
            if grad:
                c.sum().backward()
            return c

        def host_loop():
            w = {key: p[key].clone().requires_grad_(True)}
            guess0 = solver.initial_guess(p)
            guess, x, c = guess0, p["initial_state"], 0.0
            for _ in range(T):
                q = dict(p)
                q["initial_state"] = x.detach()
                sol = solver.solve(guess, q, w)
                u = sol.controls[:, 0]
                x = x @ Ad.T + u @ Bd.T + bd
                c = c + (x ** 2).sum(-1) + (u ** 2).sum(-1)
                guess = SQPSolution(*[v.detach() if isinstance(v, torch.Tensor) else v for v in sol])
            c.sum().backward()
            return c

        ms_f, c_f = _timed(lambda: fused(False), args.steps, args.warmup)
        ms_fb, c_fb = _timed(lambda: fused(True), args.steps, args.warmup)
        ms_h, c_h = _timed(host_loop, args.steps, args.warmup)
        ms_cold, _ = _timed(lambda: fused(True, roll_cold), args.steps, args.warmup)
        line.update(metric="closed-loop MPC rollout, linear nx=8 nu=4 N=39, 50 steps, warm start, B=%d: "
                           "MPC solves/s (B*steps per second), fwd+bwd through the rollout" % B,
                    value=B * T / (ms_fb * 1e-3), ms_per_step=ms_fb, batch=B, sim_steps=T,
                    fwd_only_solves_per_s=B * T / (ms_f * 1e-3), fwd_only_ms=ms_f,
                    host_loop_solves_per_s=B * T / (ms_h * 1e-3), host_loop_ms=ms_h,
                    cold_start_solves_per_s=B * T / (ms_cold * 1e-3),
                    reference_recorded={
                        "fwd_solves_per_s": 23847, "fwd_bwd_solves_per_s": 14651,
                        "config": "B=64, 40 knots, 50 steps, PCG 1e-12, warm start, FP64 JAX on an unrecorded GPU",
                        "source": "benchmarking/reinforcement-learning/timing_results/"
                                  "timing_64_40_12_pcg=1e-12_warmstart=True/diffmpc_cuda:0_{fwd,bwd}.npy (median of 100)"},
                    max_rel_cost_diff_fused_vs_host_loop=float((c_fb - c_h).abs().max() / c_h.abs().max()),
                    pcg_iters_per_solve=float(roll.last.pcg_hist.double().sum() / (B * T)))
    elif args.workload == "rollout_spacecraft":
        from diffmpc_b200.rollout import ClosedLoopRollout

        B = args.batch if args.batch != 4096 else 16
        T = 20
        dyn, st, bt, sp = workloads.rl_spacecraft(B=B)
        solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp, device=dev)
        p = workloads.to_device(bt, dev)
        keys = ["weights_penalization_reference_state_trajectory", "weights_penalization_control_squared"]
        roll = ClosedLoopRollout(solver, num_sim_steps=T, simulator="euler", state_weight=10.0)

        def run(grad):
            w = {k: p[k].clone().requires_grad_(grad) for k in keys}
            c = roll(p["initial_state"], p, w)
            if grad:
                c.sum().backward()
            return c

        ms_f, _ = _timed(lambda: run(False), args.steps, args.warmup)
        ms_fb, _ = _timed(lambda: run(True), args.steps, args.warmup)
        line.update(metric="closed-loop MPC rollout, spacecraft nx=3 N=39, 20 steps, model Euler simulator, "
                           "B=%d: MPC solves/s (B*steps per second), fwd+bwd through the rollout" % B,
                    value=B * T / (ms_fb * 1e-3), ms_per_step=ms_fb, batch=B, sim_steps=T,
                    fwd_only_solves_per_s=B * T / (ms_f * 1e-3), fwd_only_ms=ms_f,
                    reference_recorded={
                        "fwd_ms_per_rollout": 5.5, "fwd_bwd_ms_per_rollout": 8.8,
                        "config": "batch and horizon unrecorded (script defaults B=16, 40 knots, 20 steps), "
                                  "FP64 JAX on CPU (TFRT_CPU_0)",
                        "source": "benchmarking/reinforcement-learning/spacecraft/timing_results/spacecraft_timing/"
                                  "diffmpc_TFRT_CPU_0_{fwd,bwd}.npy (median)"},
                    pcg_iters_per_solve=float(roll.last.pcg_hist.double().sum() / (B * T)))
    else:  # stress
        B = args.batch if args.batch != 4096 else 16384
        dyn, st, bt, sp = workloads.linear_stress(B=B)
        sp["pcg"]["tol_epsilon"] = args.pcg_tol
        if args.pcg_max_iter > 0:
            sp["pcg"]["max_iter"] = args.pcg_max_iter
        sp["num_scp_iteration_max"] = 2
        out = {}
        for prec in ("mixed", "fp64"):
            sp2 = dict(sp, precision=prec)
            solver = SQPSolver(OptimalControlProblem(dyn, st), params=sp2, device=dev)
            p = workloads.to_device(bt, dev)

            def step():
                w = {"weights_penalization_reference_state_trajectory":
                     p["weights_penalization_reference_state_trajectory"].clone().requires_grad_(True)}
                sol = solver.solve(solver.initial_guess(p), p, w)
                (sol.controls[:, 0] ** 2).sum().backward()
                return sol, w

            ms, (sol, w) = _timed(step, args.steps, args.warmup)
            # QP solves whose FP64 recurrence ran out of pcg.max_iter before the stopping test held
            its64 = solver.last_forward_pcg_record[1].cpu() if prec == "mixed" else sol.num_pcg_iters.cpu()
            at_budget = (its64 >= sp["pcg"]["max_iter"]).any(dim=1)
            out[prec] = (ms, sol.controls.detach().cpu(), w["weights_penalization_reference_state_trajectory"].grad.cpu(),
                         sol.num_pcg_iters.sum(dim=1).double().mean().item(), precision_record(solver, sol), at_budget)
        c64, g64 = out["fp64"][1], out["fp64"][2]
        rel_c = _rel_per_instance(out["mixed"][1], c64)
        outl = [int(i) for i in torch.nonzero(rel_c > 1e-6).flatten()]
        line.update(qp_budget_exhausted={"mixed_instances": int(out["mixed"][5].sum()),
                                         "fp64_instances": int(out["fp64"][5].sum()),
                                         "control_outliers_with_a_qp_at_budget": sum(
                                             1 for i in outl if bool(out["mixed"][5][i] or out["fp64"][5][i])),
                                         "control_outliers": len(outl)})
        line.update(metric="fwd+bwd MPC solves/s, linear nx=24 nu=8 N=128, diag Q 1e-3..1e3, B=%d" % B,
                    pcg_max_iter=sp["pcg"]["max_iter"],
                    value=B / (out["mixed"][0] * 1e-3), fp64_value=B / (out["fp64"][0] * 1e-3),
                    max_rel_control_diff_mixed_vs_fp64=float((out["mixed"][1] - c64).abs().max() / c64.abs().max()),
                    max_rel_grad_diff_mixed_vs_fp64=float((out["mixed"][2] - g64).abs().max() / g64.abs().max()),
                    controls_mixed_vs_fp64=_dist(_rel_per_instance(out["mixed"][1], c64), 1e-6),
                    grads_mixed_vs_fp64=_dist(_rel_per_instance(out["mixed"][2], g64), 1e-5),
                    pcg_iters_mixed=out["mixed"][3], pcg_iters_fp64=out["fp64"][3],
                    refinement_steps=out["mixed"][4]["replacements_per_qp"], precision_record=out["mixed"][4])
    return line


# The other workload shapes measured inside the default run (one GPU, after the headline), so that
# the line the default run prints carries them too: (workload, batch or None for its default,
# steps, warm-up steps).  The precision-stress shape runs on a 1024-instance slice of its
# 16384-instance batch to keep the run within minutes (`--workload stress` runs all of it).
OTHER_WORKLOADS = (("attitude", None, 3, 3), ("rollout", None, 3, 3), ("rollout_spacecraft", None, 3, 3),
                   ("mixed", None, 2, 1), ("stress", 1024, 1, 1))


def other_workloads(args):
    out = {}
    for name, batch, steps, warmup in OTHER_WORKLOADS:
        a = copy.copy(args)
        a.workload, a.steps, a.warmup = name, steps, warmup
        a.batch = batch if batch is not None else 4096  # 4096: the workload's own default batch
        a.cta_config, a.threads, a.blocks_in_smem = "auto", 0, -1
        t0 = time.perf_counter()
        try:
            line = run_other_workload(a)
        except Exception as e:  # noqa: BLE001 - the headline line must still print
            out[name] = {"error": f"{type(e).__name__}: {e}"}
            continue
        line["wall_s"] = time.perf_counter() - t0
        for k in ("impl", "unit", "n_gpus", "data", "workload"):
            line.pop(k, None)
        out[name] = line
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "quadrotor":
        print(json.dumps(run_other_workload(args)), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
