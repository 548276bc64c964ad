"""Launch-shape autotuner for the fused solver kernels.

One CTA solves one instance, so the tunables are the CTA size (how many warps work on one
instance) and the CTA configuration (``cta_config``: how many registers a thread gets and how
many CTAs share an SM -- WIDE one CTA of up to 512 threads, ROWS one of 256..384 threads with
up to 255 registers for the row PCG, DUAL two CTAs of 256 threads).  Shared memory can further
limit the CTAs per SM.  A candidate is ``threads`` (with the automatic configuration) or
``(cta_config, threads)``.  ``tune`` times a forward solve of a sample of the caller's batch for
every candidate; ``tune_step`` times any step (for example forward + adjoint of several ragged
groups through ``solve_groups``, whose launches take the first solver's parameters).  The
fastest goes into the solver's parameters.  A JSON cache keyed by (model, nx, nu, N, precision,
GPU name, and the caller's tag for ``tune_step``) makes later calls free.
"""

import json
import os
from typing import Dict, Iterable, Optional

import torch

from . import _lib
from .sqp import SQPSolver, solver_params_struct

CACHE_PATH = os.environ.get("DMPC_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "dmpc_autotune.json"))


def _key(solver: SQPSolver) -> str:
    prog = solver.program
    prec = solver.params.get("precision", "mixed")
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return f"{prog.dynamics.model_name}/{prog.num_state_variables}/{prog.num_control_variables}/{prog.horizon}/{prec}/{name}"


def _load_cache() -> Dict[str, int]:
    try:
        with open(CACHE_PATH) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(cache: Dict[str, int]) -> None:
    try:
        os.makedirs(os.path.dirname(CACHE_PATH), exist_ok=True)
        with open(CACHE_PATH, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:
        pass


def candidates(solver: SQPSolver) -> Iterable:
    """Launch shapes worth trying: the automatic choice, WIDE at 256..512 threads, ROWS at 256 and
    384 (mixed precision only: the row PCG is what its registers are for) and DUAL."""
    out = [(_lib.CTA_AUTO, 0), (_lib.CTA_WIDE, 256), (_lib.CTA_WIDE, 384), (_lib.CTA_WIDE, 512), (_lib.CTA_DUAL, 256)]
    if solver.params.get("precision", "mixed") == "mixed":
        out += [(_lib.CTA_ROWS, 256), (_lib.CTA_ROWS, 384)]
    return out


def _as_pair(c):
    return (int(c[0]), int(c[1])) if isinstance(c, (tuple, list)) else (_lib.CTA_AUTO, int(c))


def _apply(solver: SQPSolver, c) -> None:
    cfg, thr = _as_pair(c)
    solver.params["cta_config"] = cfg
    solver.params["threads_per_block"] = thr
    solver._c_params = solver_params_struct(solver.params)


def _time_candidates(solver: SQPSolver, fn, cands, repeats: int):
    """Device time of ``fn`` per candidate launch shape (candidates the library refuses are skipped)."""
    timings = {}
    saved = (solver.params.get("cta_config", 0), solver.params.get("threads_per_block", 0))
    try:
        for c in cands:
            _apply(solver, c)
            try:
                fn()  # warm-up (and validity check)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(repeats):
                    fn()
                e1.record()
                torch.cuda.synchronize()
                timings[c if not isinstance(c, list) else tuple(c)] = e0.elapsed_time(e1) / repeats
            except _lib.DmpcError:
                continue
    finally:
        _apply(solver, saved)
    return timings


def tune_step(solver: SQPSolver, fn, tag: str, repeats: int = 2, use_cache: bool = True,
              cands: Optional[Iterable] = None):
    """Pick the fastest launch shape for the step ``fn()`` (no arguments; it launches with
    ``solver``'s parameters) and store it in ``solver.params``.  ``tag`` names the step in the
    cache key.  Returns the winning candidate."""
    key = _key(solver) + "/" + tag
    cache = _load_cache() if use_cache else {}
    if key in cache:
        best = cache[key]
        best = tuple(best) if isinstance(best, list) else best
    else:
        timings = _time_candidates(solver, fn, list(cands if cands is not None else candidates(solver)), repeats)
        best = min(timings, key=timings.get) if timings else (_lib.CTA_AUTO, 0)
        cache[key] = list(best) if isinstance(best, tuple) else best
        if use_cache:
            _store_cache(cache)
    _apply(solver, best)
    return best


def tune(solver: SQPSolver, problem_params: Dict, sample: int = 296, repeats: int = 2,
         use_cache: bool = True, cands: Optional[Iterable] = None):
    """Pick the fastest launch shape for ``solver`` on ``problem_params``.

    ``problem_params`` is a batched parameter dict as passed to ``solve``; the first
    ``sample`` instances (two waves of 148 SMs by default) are timed.  The winner is
    written into ``solver.params`` (``cta_config``, ``threads_per_block``) and returned in
    the form of the candidates (``threads``, or ``(cta_config, threads)``).
    """
    B = int(torch.as_tensor(problem_params["initial_state"]).reshape(-1, solver.program.num_state_variables).shape[0])
    n = min(sample, B)
    sub = {}
    for k, v in problem_params.items():
        sub[k] = v[:n] if isinstance(v, torch.Tensor) and v.dim() > 0 and v.shape[0] == B else v
    guess = solver.initial_guess(sub)
    return tune_step(solver, lambda: solver.solve(guess, sub), tag=f"fwd{n}", repeats=repeats, use_cache=use_cache,
                     cands=cands)
