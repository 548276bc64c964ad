"""Launch-shape autotuner for the fused solver kernels.

One CTA solves one instance, so the tunable is the CTA size: how many warps work on
one instance.  Shared memory fixes how many CTAs fit per SM: one for the quadrotor
N=60 blocks, more for small instances.  ``tune`` times a forward solve of a sample of the
caller's batch for every candidate CTA size and stores the fastest in the solver's parameters. A JSON cache keyed
by (model, nx, nu, N, precision, GPU name) makes later calls free.
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


def candidates(solver: SQPSolver) -> Iterable[int]:
    """CTA sizes worth trying: the default (0 = automatic) and 128..512 in warps of 64."""
    return [0, 128, 192, 256, 320, 384, 448, 512]


def tune(solver: SQPSolver, problem_params: Dict, sample: int = 296, repeats: int = 2,
         use_cache: bool = True, cands: Optional[Iterable[int]] = None) -> int:
    """Pick the fastest ``threads_per_block`` for ``solver`` on ``problem_params``.

    ``problem_params`` is a batched parameter dict as passed to ``solve``; the first
    ``sample`` instances (two waves of 148 SMs by default) are timed.  The winner is
    written into ``solver.params["threads_per_block"]`` and returned.
    """
    key = _key(solver)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        best = int(cache[key])
    else:
        B = int(torch.as_tensor(problem_params["initial_state"]).reshape(-1, solver.program.num_state_variables).shape[0])
        n = min(sample, B)
        sub = {}
        for k, v in problem_params.items():
            sub[k] = v[:n] if isinstance(v, torch.Tensor) and v.dim() > 0 and v.shape[0] == B else v
        timings = {}
        saved = solver.params.get("threads_per_block", 0)
        for t in (cands if cands is not None else candidates(solver)):
            solver.params["threads_per_block"] = t
            try:
                solver._c_params = solver_params_struct(solver.params)
                guess = solver.initial_guess(sub)
                solver.solve(guess, sub)  # warm-up (and validity check)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(repeats):
                    solver.solve(guess, sub)
                e1.record()
                torch.cuda.synchronize()
                timings[t] = e0.elapsed_time(e1) / repeats
            except _lib.DmpcError:
                continue
        solver.params["threads_per_block"] = saved
        best = min(timings, key=timings.get) if timings else 0
        cache[key] = best
        if use_cache:
            _store_cache(cache)
    solver.params["threads_per_block"] = best
    solver._c_params = solver_params_struct(solver.params)
    return best
