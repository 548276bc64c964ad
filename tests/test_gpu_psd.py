"""GPU parity of the PSD projection (dmpc_psd_project, FP64 Jacobi, one warp per matrix) with the
oracle's eigh-based restatement of jax_utils.py:75-95, through the C ABI's Python wrapper.
Bar: 1e-12 relative to the largest entry (the projection is unique, whatever the eigenvector
order, signs or basis within a repeated eigenvalue)."""

import numpy as np
import pytest
import torch

from diffmpc_b200.utils import project_matrix_onto_positive_semidefinite_cone as psd
from oracle.sqp import project_psd

pytestmark = pytest.mark.gpu


def _close(a, b):
    a, b = a.cpu(), b.cpu()
    return float((a - b).abs().max()) <= 1e-12 * max(1.0, float(b.abs().max()))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 8, 13, 24, 32])
def test_random_symmetric_indefinite_matrices(n):
    rng = np.random.default_rng(n)
    a = torch.tensor(rng.standard_normal((37, n, n)))
    a = a + a.mT
    for min_eig in (0.0, 1e-9, 0.5):
        assert _close(psd(a.cuda(), min_eig), project_psd(a, min_eig)), (n, min_eig)


def test_nonsymmetric_input_batched_leading_dims_and_in_place_layouts():
    rng = np.random.default_rng(7)
    a = torch.tensor(rng.standard_normal((3, 5, 6, 6)))
    out = psd(a.cuda(), 1e-9)
    assert out.shape == a.shape
    assert _close(out, project_psd(a, 1e-9))
    assert torch.equal(out, out.mT)


def test_repeated_and_clustered_eigenvalues():
    rng = np.random.default_rng(3)
    q, _ = np.linalg.qr(rng.standard_normal((10, 10)))
    lam = np.array([2.0, 2.0, 2.0, -1.0, -1.0, 1e-12, 0.0, 5.0, 5.0 + 1e-13, -3.0])
    m = torch.tensor(q @ np.diag(lam) @ q.T)[None]
    ref = torch.tensor(q @ np.diag(np.maximum(lam, 1e-9)) @ q.T)
    assert _close(psd(m.cuda(), 1e-9), ref[None])
    eye = torch.eye(13, dtype=torch.float64)[None].repeat(4, 1, 1)
    assert _close(psd(eye.cuda(), 1e-9), eye)


def test_diagonal_cost_hessians_of_a_workload():
    """The quadrotor cost Hessians 2 diag(w) (the fused solver's closed form max(2w, 1e-9))."""
    from diffmpc_b200 import workloads

    _, _, bt, _ = workloads.quadrotor(B=8, N=10, seed=5)
    w = bt["weights_penalization_reference_state_trajectory"].clone()
    w[:, ::3] = -w[:, ::3]  # indefinite entries exercise the clip
    h = torch.diag_embed(2.0 * w)
    assert _close(psd(h.cuda(), 1e-9), torch.diag_embed((2.0 * w).clamp_min(1e-9)))


def test_non_finite_input_gives_nan_and_leaves_the_other_matrices_alone():
    m = torch.eye(4, dtype=torch.float64)[None].repeat(3, 1, 1)
    m[0, 1, 2] = float("nan")
    m[1, 3, 3] = float("inf")
    out = psd(m.cuda(), 0.0).cpu()
    assert bool(torch.isnan(out[0]).all()) and bool(torch.isnan(out[1]).all())
    assert _close(out[2:], torch.eye(4, dtype=torch.float64)[None])
