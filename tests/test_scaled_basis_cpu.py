"""The FP32 iterations run PCG in the basis scaled by the Cholesky factors of the
diagonal Schur blocks.  This checks, in float64 on the CPU, the identities that basis
rests on, using the oracle's S and Phi^-1 (pcg.py:160-243):

* L^T Phi^-1 L = I - F^ and L^-1 S L^-T = -(I + F^), with F^ zero on the block diagonal;
* PCG on (S^, I - F^) from r^ = L^-1 r produces the reference recurrence's eta sequence
  and, mapped back by L^-T, its iterates.
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
