"""The FP32 iterations run PCG in the basis scaled by the Cholesky factors of the
diagonal Schur blocks.  This checks, in float64 on the CPU, the identities that basis
rests on, using the oracle's S and Phi^-1 (pcg.py:160-243):

* L^T Phi^-1 L = I - F^ and L^-1 S L^-T = -(I + F^), with F^ zero on the block diagonal;
* PCG on (S^, I - F^) from r^ = L^-1 r produces the reference recurrence's eta sequence
  and, mapped back by L^-T, its iterates;
* the kernels' mixed-precision recurrence (FP32 PCG with FP64 residual replacement and stall
  detection, sqp_device.cuh: pcg_rows_scaled and pcg_mixed_scaled), restated in numpy with FP32
  vectors, stops on the reference's FP64 test and reaches the solution; it needs fewer FP32
  iterations than restarting refinement, which at the shipped inner tolerance (1e-3) cannot
  meet a 1e4-fold stagnation rule and would hand every solve to the FP64 recurrence;
* on ill-conditioned systems the stall detection hands the solve to the FP64 recurrence after
  a few hundred FP32 iterations instead of half the budget.
"""

import numpy as np
import torch

from oracle import pcg as opcg


def _system(seed, N=20, nx=6, nu=3, qspread=2.0):
    rng = np.random.default_rng(seed)
    K = N + 1
    A = torch.tensor(np.eye(nx) + 0.1 * rng.standard_normal((1, N, nx, nx)))
    Bm = torch.tensor(0.1 * rng.standard_normal((1, N, nx, nu)))
    An = -torch.eye(nx, dtype=torch.float64).expand(1, N, nx, nx).clone()
    Qinv = torch.diag_embed(torch.tensor(10 ** rng.uniform(-qspread, qspread, (1, K, nx))))
    Rinv = torch.diag_embed(torch.tensor(10 ** rng.uniform(-1, 1, (1, N, nu))))
    qp = opcg.QPParameters(
        opcg.QPDynamicsParameters(An, A, Bm, torch.zeros(1, K, nx)),
        opcg.QPCostParameters(Qinv, torch.zeros(1, K, nx), Rinv, torch.zeros(1, N, nu)),
    )
    S, Phi = opcg.compute_S_Phiinv(qp)
    gam = torch.tensor(rng.standard_normal(K * nx))
    return S, Phi, gam, K, nx


def _dense(M, K, nx):
    D = torch.zeros(K * nx, K * nx, dtype=torch.float64)
    for t in range(K):
        for c, tt in enumerate((t - 1, t, t + 1)):
            if 0 <= tt < K:
                D[t * nx:(t + 1) * nx, tt * nx:(tt + 1) * nx] = M[0, t, :, c * nx:(c + 1) * nx]
    return D


def _pcg(Smat, Minv, b, iters):
    x = torch.zeros_like(b)
    r = b.clone()
    z = Minv @ r
    p = z.clone()
    eta = r @ z
    etas, xs = [], []
    for _ in range(iters):
        u = Smat @ p
        a = eta / (p @ u)
        x = x + a * p
        r = r - a * u
        z = Minv @ r
        e2 = r @ z
        p = z + (e2 / eta) * p
        eta = e2
        etas.append(float(eta))
        xs.append(x.clone())
    return etas, xs


def test_scaled_operators_and_pcg_equivalence():
    for seed in (0, 1):
        S, Phi, gam, K, nx = _system(seed)
        Sd, Pd = _dense(S, K, nx), _dense(Phi, K, nx)
        n = K * nx
        eye = torch.eye(n, dtype=torch.float64)
        L = torch.block_diag(*[torch.linalg.cholesky(-Sd[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx]) for t in range(K)])
        Li = torch.linalg.inv(L)
        Fh = -(Li @ Sd @ Li.T) - eye
        for t in range(K):
            assert float(Fh[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx].abs().max()) < 1e-12
        assert float((L.T @ Pd @ L - (eye - Fh)).abs().max()) < 1e-12
        e_ref, x_ref = _pcg(Sd, Pd, gam, 12)
        e_sc, x_sc = _pcg(-(eye + Fh), eye - Fh, Li @ gam, 12)
        for a, b in zip(e_ref, e_sc):
            assert abs(a - b) <= 1e-10 * abs(a)
        for a, b in zip(x_ref, x_sc):
            assert float((a - Li.T @ b).abs().max()) <= 1e-10 * float(a.abs().max())


def _fp64_finish(Sd, Pd, gam, lam, eps, max_iter):
    """The FP64 recurrence from lam (the kernels' fp64_finish, in the reference basis).
    Returns (lam, iterations, the recursion's final eta)."""
    r = gam - Sd @ lam
    z = Pd @ r
    p, e, it = z.copy(), float(r @ z), 0
    while (abs(e) > eps and it <= max_iter - 1) or it < 1:
        u = Sd @ p
        a = e / float(p @ u)
        lam, r = lam + a * p, r - a * u
        z = Pd @ r
        e2 = float(r @ z)
        p, e = z + (e2 / e) * p, e2
        it += 1
    return lam, it, e


STALL_MIN, STALL_GROWTH = 200, 2  # sqp_device.cuh: kStallMin, kStallGrowth


def _pcg_replacement(Fh, Li, Sd, gam, eps, upd_rel=1e-3, check_margin=0.1, max_iter=10000, Pd=None, max_ref=30,
                     stall=True, stats=None, stall_min=STALL_MIN, stall_growth=STALL_GROWTH):
    """Numpy restatement of the kernels' mixed recurrence (sqp_device.cuh: pcg_rows_scaled,
    pcg_mixed_scaled): FP32 vectors and FP32 F^, FP64 dot products, and the FP32 residual replaced
    by the FP64 one, r^ = r^_0 + (I + F^) lam^, each time the recursion's eta falls by `upd_rel`;
    convergence is decided on an exact residual gamma - S lam.  With `stall`, an FP32 segment is
    also cut after max(stall_growth x the previous segment, stall_min) iterations (stall_min for
    the first; the kernels' 4 and 200 by default).  With Pd
    given, the kernels' hand-over rules apply (a replacement triggered by the recursion's fall or
    its divergence whose true eta fell by less than 100x, or by the stall cut whose true eta fell
    by less than 1/upd_rel; half the budget or max_ref replacements spent) and the FP64 recurrence finishes; the replacement count is then
    returned negated and, with `stats` (a dict), the FP64 iteration count stored under "fp64".
    Returns (lam, iterations, replacements, eta64)."""
    f32, f64 = np.float32, np.float64
    F64 = Fh
    F32 = Fh.astype(f32)
    lam = np.zeros_like(gam)
    rh0 = Li @ (gam - Sd @ lam)
    eta64 = float(rh0 @ (rh0 - F64 @ rh0))
    scale = 1.0 / np.sqrt(eta64)
    s2 = scale * scale
    check_at = eps * s2 * check_margin
    r = (scale * rh0).astype(f32)
    p = (scale * (rh0 - F64 @ rh0)).astype(f32)
    d = np.zeros_like(r)
    acc = np.zeros_like(gam)
    eta = eta64 * s2
    trig = max(check_at, upd_rel * eta)
    hi = 1e4 * eta
    eta_upd, prev64 = eta, eta64
    it = nrep = seg0 = 0
    it_cap = max_iter // 2
    it_stop = min(it_cap, stall_min) if stall else it_cap
    while True:
        u = -(p + F32 @ p)
        vden = float(p.astype(f64) @ u.astype(f64))
        alpha = f32(eta / vden)
        d = d + alpha * p
        r = r - alpha * u
        z = r - F32 @ r
        etap = float(r.astype(f64) @ z.astype(f64))
        it += 1
        if trig < etap <= hi and it < it_stop:
            p = z + f32(etap / eta) * p
            eta = etap
            continue
        acc = acc + d.astype(f64) / scale
        d = np.zeros_like(r)
        at_check = etap <= check_at
        fell = etap <= upd_rel * eta_upd or etap > hi
        cut = not fell and it_stop <= it < it_cap  # ended by the stall detection
        progressed = fell or cut
        exact = at_check
        if not exact:
            rh = rh0 + acc + F64 @ acc
            eta64 = float(rh @ (rh - F64 @ rh))
            exact = not eta64 > eps
        if exact:
            lam = lam + Li.T @ acc
            acc = np.zeros_like(gam)
            rh0 = Li @ (gam - Sd @ lam)
            rh = rh0
            eta64 = float(rh @ (rh - F64 @ rh))
        nrep += 1
        if not abs(eta64) > eps:
            return lam + Li.T @ acc, it, nrep, eta64
        etas = eta64 * s2
        stalled = progressed and not at_check and eta64 > (upd_rel if cut else 1e-2) * prev64
        if Pd is not None and (it >= it_cap or nrep >= max_ref or stalled):
            lam, it64, e = _fp64_finish(Sd, Pd, gam, lam + Li.T @ acc, eps, max_iter)
            if stats is not None:
                stats["fp64"] = it64
            return lam, it + it64, -nrep, e
        assert it < it_cap, "FP32 share of the budget exhausted"
        eta_upd, prev64 = etas, eta64
        if stall:
            it_stop = min(it_cap, it + max(stall_growth * (it - seg0), stall_min))
        seg0 = it
        r = (scale * rh).astype(f32)
        z = (scale * (rh - F64 @ rh)).astype(f32)
        if etas > 10.0 * eta:
            p = np.zeros_like(p)
        p = z + f32(etas / eta) * p
        eta = etas
        trig = max(check_at, upd_rel * etas)
        hi = 1e4 * etas


def _pcg_restart(Fh, Li, Sd, gam, eps, inner_rel=1e-3, max_ref=30, stagnation=1e-4, Pd=None):
    """Restarting refinement, the alternative to residual replacement: FP64 iterative refinement
    around FP32 PCG solves that restart from the scaled FP64 residual and stop at inner_rel * eta
    (or 0.01 eps).  With Pd given, a refinement that cuts eta64 by less than 1/stagnation, or the
    max_ref-th refinement, hands the solve to the FP64 recurrence and the refinement count is
    returned negated.  Returns (lam, iterations, refinements, eta64)."""
    f32, f64 = np.float32, np.float64
    F32 = Fh.astype(f32)
    lam = np.zeros_like(gam)
    it = 0
    prev64 = None
    for ref in range(max_ref + 1):
        rh = Li @ (gam - Sd @ lam)
        eta64 = float(rh @ (rh - Fh @ rh))
        if not abs(eta64) > eps:
            return lam, it, ref, eta64
        if Pd is not None and (ref >= max_ref or (prev64 is not None and eta64 > stagnation * prev64)):
            lam, it64, e = _fp64_finish(Sd, Pd, gam, lam, eps, 10000)
            return lam, it + it64, -ref, e
        prev64 = eta64
        scale = 1.0 / np.sqrt(eta64)
        r = (scale * rh).astype(f32)
        d = np.zeros_like(r)
        z = r - F32 @ r
        p = z.copy()
        eta = float(r.astype(f64) @ z.astype(f64))
        target = max(inner_rel * eta, eps * scale * scale * 0.01)
        inner = 0
        while eta > target or inner < 1:
            u = -(p + F32 @ p)
            alpha = f32(eta / float(p.astype(f64) @ u.astype(f64)))
            d, r = d + alpha * p, r - alpha * u
            z = r - F32 @ r
            e2 = float(r.astype(f64) @ z.astype(f64))
            p, eta = z + f32(e2 / eta) * p, e2
            it += 1
            inner += 1
        lam = lam + Li.T @ (d.astype(f64) / scale)
    raise AssertionError("refinement did not converge")


def _scaled(seed, qspread=2.0):
    S, Phi, gam, K, nx = _system(seed, qspread=qspread)
    Sd, Pd = _dense(S, K, nx).numpy(), _dense(Phi, K, nx).numpy()
    n = K * nx
    L = np.zeros((n, n))
    for t in range(K):
        L[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx] = np.linalg.cholesky(-Sd[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx])
    Li = np.linalg.inv(L)
    Fh = -(Li @ Sd @ Li.T) - np.eye(n)
    return Sd, Pd, gam.numpy(), Li, Fh


def test_mixed_recurrences_reach_the_fp64_stopping_rule():
    """Both mixed recurrences stop only on an exact FP64 eta below eps and reach the solution
    of S lam = gamma to the accuracy that eps allows.  Keeping the search direction across the
    FP64 corrections (residual replacement, at the shipped defaults) takes fewer FP32 iterations
    than restarting at each refinement, even when the restarted inner solves run to 1e-8."""
    for seed in (0, 1, 2):
        Sd, Pd, g, Li, Fh = _scaled(seed)
        n = g.shape[0]
        exact = np.linalg.solve(Sd, g)
        eps = 1e-22 * float(g @ g)
        its = {}
        for name, solve in (("replace", _pcg_replacement),
                            ("restart", lambda *a: _pcg_restart(*a, inner_rel=1e-8))):
            lam, it, nfix, eta64 = solve(Fh, Li, Sd, g, eps)
            res = g - Sd @ lam
            assert float(res @ (Pd @ res)) <= eps, name
            assert abs(eta64 - float(res @ (Pd @ res))) <= 1e-6 * eps + 1e-12 * abs(eta64), name
            assert np.abs(lam - exact).max() <= 1e-8 * np.abs(exact).max(), name
            assert 0 < nfix <= 30, name
            its[name] = it
        _, it64, _ = _fp64_finish(Sd, Pd, g, np.zeros(n), eps, 10000)
        assert its["replace"] < its["restart"], (seed, its)
        assert its["replace"] <= 2.5 * it64, (seed, its, it64)


def test_restarting_refinement_at_the_shipped_tolerance_always_hands_over():
    """An FP32 inner solve stopped at the shipped relative tolerance (1e-3) cuts eta64 by about
    1e3, never by the 1e4 a restarting scheme's stagnation rule asks for, so restarting refinement
    with those settings would hand every solve to the FP64 recurrence after one refinement.
    Residual replacement at the same settings (a 100-fold true fall per 1e3-fold recursion fall)
    finishes these systems in FP32 with no hand-over."""
    for seed in (0, 1, 2):
        Sd, Pd, g, Li, Fh = _scaled(seed)
        eps = 1e-20 * float(g @ g)
        _, _, nref, eta = _pcg_restart(Fh, Li, Sd, g, eps, inner_rel=1e-3, stagnation=1e-4, Pd=Pd)
        assert nref == -1, (seed, nref)  # handed over after the first refinement
        assert abs(eta) <= eps
        _, _, nrep, eta = _pcg_replacement(Fh, Li, Sd, g, eps, upd_rel=1e-3, Pd=Pd)
        assert nrep > 0, (seed, nrep)
        assert abs(eta) <= eps


def test_ill_conditioned_systems_hand_over_to_fp64_and_match_the_reference_recurrence():
    """Diagonal cost weights over 1e-6..1e6 (cond(S) 1e10..1e11, the precision-stress shape):
    the FP32 recursion stalls, the stall detection cuts its segment and the stagnation rule sends
    the solve to the FP64 recurrence, which ends on the reference's stopping test; the solution is
    as accurate as that of the reference recurrence run alone to the same eps.  Without the stall
    detection the FP32 recursion runs to half the budget (5000 iterations) first.  (At this
    conditioning the recursively updated eta of either drifts above the true one, so the true eta
    is not compared.)"""
    for seed in (3, 4, 5):
        Sd, Pd, g, Li, Fh = _scaled(seed, qspread=6.0)
        n = g.shape[0]
        eps = 1e-20 * float(g @ g)
        exact = np.linalg.solve(Sd, g)
        ref, _, _ = _fp64_finish(Sd, Pd, g, np.zeros(n), eps, 10000)
        st = {}
        lam, it, nrep, eta = _pcg_replacement(Fh, Li, Sd, g, eps, Pd=Pd, stats=st)
        assert nrep < 0, (seed, nrep)
        assert abs(eta) <= eps, (seed, nrep, eta)
        err, rerr = np.abs(lam - exact).max(), np.abs(ref - exact).max()
        assert err <= 10.0 * rerr + 1e-9 * np.abs(exact).max(), (seed, err, rerr)
        fp32_its = it - st["fp64"]
        assert fp32_its <= 2 * STALL_MIN + 100, (seed, fp32_its)
        st_off = {}
        _, it_off, nrep_off, _ = _pcg_replacement(Fh, Li, Sd, g, eps, Pd=Pd, stall=False, stats=st_off)
        assert nrep_off < 0 and it_off - st_off["fp64"] >= 3000, (seed, it_off, st_off)


def test_stall_thresholds_leave_the_headline_qps_in_fp32():
    """The stall cut's thresholds against the QPs of the headline workload (quadrotor N=60, the
    first SQP iteration of four instances, the oracle's S and Phi^-1, eps 1e-20 relative): at the
    kernels' max(2 x previous, 200) no QP is handed to the FP64 recurrence; a tighter
    max(2 x previous, 50) hands some over although FP32 finishes them in fewer iteration-costs."""
    from diffmpc_b200 import workloads
    from tests.oracle_util import oracle_solver, tensor_params

    dyn, st, bt, sp = workloads.quadrotor(B=4, N=60, seed=1002)
    os_ = oracle_solver(dyn, st, sp)
    tp = tensor_params(bt)
    g0 = os_.initial_guess(tp)
    _, _, schur = os_.compute_qp_parameters(g0.states, g0.controls, tp)
    tight_handovers = 0
    for i in range(4):
        S, Phi = schur.S[i:i + 1], schur.preconditioner_Phiinv[i:i + 1]
        K, nx = S.shape[1], S.shape[2]
        Sd, Pd = _dense(S, K, nx).numpy(), _dense(Phi, K, nx).numpy()
        n = K * nx
        L = np.zeros((n, n))
        for t in range(K):
            L[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx] = np.linalg.cholesky(-Sd[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx])
        Li = np.linalg.inv(L)
        Fh = -(Li @ Sd @ Li.T) - np.eye(n)
        g = np.random.default_rng(i).standard_normal(n)
        eps = 1e-20 * float(g @ g)
        _, _, nrep, eta = _pcg_replacement(Fh, Li, Sd, g, eps, Pd=Pd)
        assert nrep > 0 and abs(eta) <= eps, (i, nrep)
        _, _, nrep_t, _ = _pcg_replacement(Fh, Li, Sd, g, eps, Pd=Pd, stall_min=50, stall_growth=2)
        tight_handovers += nrep_t < 0
    assert tight_handovers >= 1



def test_slowly_converging_fp32_recursions_hand_over_within_the_budget():
    """The ill-conditioned QPs of the GPU test (linear nx=5 and nx=6, N=40, state weights over
    1e-6..1e6, the first SQP iteration of three instances, eps 1e-20): on some the FP32 recursion
    does not stall but falls by 1e3 only every 400-1300 iterations, 8x slower than the FP64
    recurrence.  Segments allowed to grow 4-fold were never cut and ran the FP32 share of the budget
    (5000 iterations) before the FP64 finish; at the kernels' 2-fold growth the stall cut hands them
    to the FP64 recurrence after a few hundred FP32 iterations, at a total cost (FP64 iterations
    weighted 2.7x) within 10 % of the FP64 recurrence alone on every QP."""
    from diffmpc_b200 import workloads
    from tests.oracle_util import oracle_solver, tensor_params

    for nx in (5, 6):
        dyn, st, bt, sp = workloads.linear_lti(B=3, N=40, nx=nx, nu=3, seed=1003, log10_wx=6.0)
        os_ = oracle_solver(dyn, st, sp)
        tp = tensor_params(bt)
        g0 = os_.initial_guess(tp)
        qp, premult, schur = os_.compute_qp_parameters(g0.states, g0.controls, tp)
        gam = opcg.compute_gamma(premult, qp.dynamics.Cs, qp.cost.Qinv[:, 0], qp.cost.qvec, qp.cost.rvec)
        for i in range(3):
            S, Phi = schur.S[i:i + 1], schur.preconditioner_Phiinv[i:i + 1]
            K = S.shape[1]
            Sd, Pd = _dense(S, K, nx).numpy(), _dense(Phi, K, nx).numpy()
            n = K * nx
            L = np.zeros((n, n))
            for t in range(K):
                L[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx] = np.linalg.cholesky(-Sd[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx])
            Li = np.linalg.inv(L)
            Fh = -(Li @ Sd @ Li.T) - np.eye(n)
            g = gam[i].reshape(-1).numpy()
            eps = 1e-20
            _, it64, _ = _fp64_finish(Sd, Pd, g, np.zeros(n), eps, 10000)
            stats = {}
            _, it, nrep, eta = _pcg_replacement(Fh, Li, Sd, g, eps, Pd=Pd, stats=stats)
            assert abs(eta) <= eps, (nx, i, eta)
            fp32 = it - stats.get("fp64", 0)
            assert fp32 < 600, (nx, i, fp32)
            assert fp32 + 2.7 * stats.get("fp64", 0) <= 1.1 * 2.7 * it64 + 200, (nx, i, it, stats, it64)
