"""CPU restatement of the two-CTA row PCG's register layout (sqp_device.cuh: pcg_rows_t).

TPK lanes share a knot; lane q owns rows 4q..4q+3 of W_t and keeps them with its column groups
permuted (register group g holds column group g ^ (TPK - 1 - q)).  The transposed product
W_t^T v_t is formed as per-lane column sums and a reduce-scatter of XOR shuffles (partner lane
q ^ 2, then q ^ 1 for TPK = 4) that always sends the first half of the registers and keeps the
second; afterwards lane q holds columns 4q..4q+3.  The lower product reads v_{t-1} in the same
permuted order.  This checks, lane by lane in numpy, that both products equal the dense ones for
every nx the layout serves.
"""

import numpy as np
import pytest


def tpk_of(nx):
    return 1 if nx <= 4 else (2 if nx <= 8 else 4)


def lanes_registers(W, q, tpk):
    """Lane q's register copy w[k][m] of rows 4q + k, columns in register-group order."""
    nx = W.shape[0]
    pd = 4 * tpk
    w = np.zeros((4, pd))
    for k in range(4):
        i = 4 * q + k
        for g in range(tpk):
            for kk in range(4):
                c = 4 * (g ^ (tpk - 1 - q)) + kk
                if i < nx and c < nx:
                    w[k, 4 * g + kk] = W[i, c]
    return w


def reduce_scatter(cs, tpk):
    """XOR-shuffle reduce-scatter of the lanes' column sums (list over lanes of pd-vectors)."""
    if tpk == 1:
        return [c[:4].copy() for c in cs]
    if tpk == 2:
        return [cs[q][4:8] + cs[q ^ 1][0:4] for q in range(2)]
    h = [cs[q][8:16] + cs[q ^ 2][0:8] for q in range(4)]
    return [h[q][4:8] + h[q ^ 1][0:4] for q in range(4)]


@pytest.mark.parametrize("nx", [3, 4, 6, 7, 8, 12, 13])
def test_register_layout_reproduces_both_products(nx):
    rng = np.random.default_rng(nx)
    tpk = tpk_of(nx)
    pd = 4 * tpk
    W = rng.standard_normal((nx, nx))
    v_prev = rng.standard_normal(nx)  # v_{t-1}
    v_own = rng.standard_normal(nx)   # v_t
    pad = lambda v: np.concatenate([v, np.zeros(pd - nx)])  # noqa: E731
    vp, vo = pad(v_prev), pad(v_own)
    lower = np.zeros(pd)
    cs = []
    for q in range(tpk):
        w = lanes_registers(W, q, tpk)
        # lower: rows 4q..4q+3 times v_{t-1} read in register-group order
        vperm = np.concatenate([vp[4 * (g ^ (tpk - 1 - q)): 4 * (g ^ (tpk - 1 - q)) + 4] for g in range(tpk)])
        lower[4 * q: 4 * q + 4] = w @ vperm
        # upper: the lane's column sums from its own rows of v_t
        cs.append(w.T @ vo[4 * q: 4 * q + 4])
    upper = np.concatenate(reduce_scatter(cs, tpk))
    assert np.allclose(lower[:nx], W @ v_prev, rtol=0, atol=1e-12)
    assert np.allclose(upper[:nx], W.T @ v_own, rtol=0, atol=1e-12)
    # padded rows and columns stay exactly zero
    assert not lower[nx:].any() and not upper[nx:].any()
