"""The FP32 iterations run PCG in the basis scaled by the Cholesky factors of the
diagonal Schur blocks.  This checks, in float64 on the CPU, the identities that basis
rests on, using the oracle's S and Phi^-1 (pcg.py:160-243):

* L^T Phi^-1 L = I - F^ and L^-1 S L^-T = -(I + F^), with F^ zero on the block diagonal;
* PCG on (S^, I - F^) from r^ = L^-1 r produces the reference recurrence's eta sequence
  and, mapped back by L^-T, its iterates;
* the two mixed-precision recurrences of the kernels, restated in numpy with FP32 vectors
  (residual replacement on the row-pair path, restarting refinement elsewhere), stop on the
  reference's FP64 test and reach the solution; replacement needs fewer FP32 iterations.
"""

import numpy as np
import torch

from oracle import pcg as opcg


def _system(seed, N=20, nx=6, nu=3):
    rng = np.random.default_rng(seed)
    K = N + 1
    A = torch.tensor(np.eye(nx) + 0.1 * rng.standard_normal((1, N, nx, nx)))
    Bm = torch.tensor(0.1 * rng.standard_normal((1, N, nx, nu)))
    An = -torch.eye(nx, dtype=torch.float64).expand(1, N, nx, nx).clone()
    Qinv = torch.diag_embed(torch.tensor(10 ** rng.uniform(-2, 2, (1, K, nx))))
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


def _pcg_replacement(Fh, Li, Sd, gam, eps, upd_rel=1e-3, check_margin=0.1, max_iter=10000):
    """Numpy restatement of the row-pair kernel's mixed recurrence (solver.cu, pcg_pair_scaled):
    FP32 vectors and FP32 F^, FP64 dot products, and the FP32 residual replaced by the FP64 one,
    r^ = r^_0 + (I + F^) lam^, each time the recursion's eta falls by `upd_rel`; convergence is
    decided on an exact residual gamma - S lam.  Returns (lam, iterations, replacements, eta64)."""
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
    it = nrep = 0
    while True:
        u = -(p + F32 @ p)
        vden = float(p.astype(f64) @ u.astype(f64))
        alpha = f32(eta / vden)
        d = d + alpha * p
        r = r - alpha * u
        z = r - F32 @ r
        etap = float(r.astype(f64) @ z.astype(f64))
        it += 1
        if etap > trig and it < max_iter // 2:
            p = z + f32(etap / eta) * p
            eta = etap
            continue
        acc = acc + d.astype(f64) / scale
        d = np.zeros_like(r)
        exact = etap <= check_at
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
        assert it < max_iter // 2, "FP32 share of the budget exhausted"
        etas = eta64 * s2
        r = (scale * rh).astype(f32)
        z = (scale * (rh - F64 @ rh)).astype(f32)
        if etas > 10.0 * eta:
            p = np.zeros_like(p)
        p = z + f32(etas / eta) * p
        eta = etas
        trig = max(check_at, upd_rel * etas)


def _pcg_restart(Fh, Li, Sd, gam, eps, inner_rel=1e-8, max_ref=30):
    """Numpy restatement of the generic mixed path (solver.cu, pcg_mixed_scaled): FP64
    iterative refinement around FP32 PCG solves that restart from the scaled FP64 residual
    and stop at inner_rel * eta (or 0.01 eps).  Returns (lam, iterations, refinements, eta64)."""
    f32, f64 = np.float32, np.float64
    F32 = Fh.astype(f32)
    lam = np.zeros_like(gam)
    it = 0
    for ref in range(max_ref):
        rh = Li @ (gam - Sd @ lam)
        eta64 = float(rh @ (rh - Fh @ rh))
        if not abs(eta64) > eps:
            return lam, it, ref, eta64
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


def test_mixed_recurrences_reach_the_fp64_stopping_rule():
    """Both mixed recurrences stop only on an exact FP64 eta below eps and reach the solution
    of S lam = gamma to the accuracy that eps allows.  Keeping the search direction across the
    FP64 corrections (residual replacement) takes fewer FP32 iterations than restarting at each
    refinement, as measured on the GPU (quadrotor QPs: 327 vs 424 per QP, FP64 PCG 256)."""
    for seed in (0, 1, 2):
        S, Phi, gam, K, nx = _system(seed)
        Sd, Pd = _dense(S, K, nx).numpy(), _dense(Phi, K, nx).numpy()
        g = gam.numpy()
        n = K * nx
        L = np.zeros((n, n))
        for t in range(K):
            L[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx] = np.linalg.cholesky(-Sd[t * nx:(t + 1) * nx, t * nx:(t + 1) * nx])
        Li = np.linalg.inv(L)
        Fh = -(Li @ Sd @ Li.T) - np.eye(n)
        exact = np.linalg.solve(Sd, g)
        eps = 1e-22 * float(g @ g)
        its = {}
        for name, solve in (("replace", _pcg_replacement), ("restart", _pcg_restart)):
            lam, it, nfix, eta64 = solve(Fh, Li, Sd, g, eps)
            res = g - Sd @ lam
            assert float(res @ (Pd @ res)) <= eps, name
            assert abs(eta64 - float(res @ (Pd @ res))) <= 1e-6 * eps + 1e-12 * abs(eta64), name
            assert np.abs(lam - exact).max() <= 1e-8 * np.abs(exact).max(), name
            assert nfix <= 30, name
            its[name] = it
        # the FP64 reference recurrence to the same eps
        x, rr = np.zeros(n), g.copy()
        zz = Pd @ rr
        pp, e = zz.copy(), float(rr @ zz)
        it64 = 0
        while abs(e) > eps or it64 < 1:
            uu = Sd @ pp
            a = e / float(pp @ uu)
            x, rr = x + a * pp, rr - a * uu
            zz = Pd @ rr
            e2 = float(rr @ zz)
            pp, e = zz + (e2 / e) * pp, e2
            it64 += 1
        assert its["replace"] < its["restart"], (seed, its)
        assert its["replace"] <= 2.5 * it64, (seed, its, it64)
