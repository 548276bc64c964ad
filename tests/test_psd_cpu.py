"""The oracle's PSD projection (oracle.sqp.project_psd, restating jax_utils.py:75-95) against
closed forms, and the projection's C entry point and Python wrapper on a host without a GPU."""

import numpy as np
import pytest
import torch

from oracle.sqp import project_psd


def test_diagonal_matrices_clip_their_entries():
    d = torch.tensor([[3.0, -1.0, 0.0, 1e-12], [2.0, 2.0, -5.0, 4.0]], dtype=torch.float64)
    out = project_psd(torch.diag_embed(d), 1e-9)
    assert torch.allclose(out, torch.diag_embed(d.clamp_min(1e-9)), rtol=0, atol=1e-15)


def test_two_by_two_closed_form():
    # [[0, 1], [1, 0]] has eigenvalues +-1 with eigenvectors (1, 1)/sqrt2, (1, -1)/sqrt2
    m = torch.tensor([[0.0, 1.0], [1.0, 0.0]], dtype=torch.float64)
    assert torch.allclose(project_psd(m, 0.0), 0.5 * torch.ones(2, 2, dtype=torch.float64), atol=1e-15)


def test_projection_is_idempotent_symmetric_and_keeps_psd_matrices():
    rng = np.random.default_rng(0)
    for n in (1, 3, 7, 13):
        a = torch.tensor(rng.standard_normal((5, n, n)))
        p = project_psd(a, 1e-9)
        assert torch.equal(p, p.mT)
        assert float(torch.linalg.eigvalsh(p).min()) >= 1e-9 - 1e-12
        assert torch.allclose(project_psd(p, 1e-9), p, rtol=0, atol=1e-12 * float(p.abs().max()))
        spd = a @ a.mT + torch.eye(n, dtype=torch.float64)
        assert torch.allclose(project_psd(spd, 1e-9), spd, rtol=0, atol=1e-12 * float(spd.abs().max()))


def test_input_is_symmetrized_first():
    """jnp.linalg.eigh symmetrizes its input by default: only the symmetric part counts."""
    rng = np.random.default_rng(1)
    a = torch.tensor(rng.standard_normal((4, 6, 6)))
    skew = a - a.mT
    assert torch.allclose(project_psd(a, 0.0), project_psd(a + 3.0 * skew, 0.0), atol=1e-12)


def test_wrapper_refuses_host_tensors():
    from diffmpc_b200.utils import project_matrix_onto_positive_semidefinite_cone

    with pytest.raises(ValueError):
        project_matrix_onto_positive_semidefinite_cone(torch.eye(3, dtype=torch.float64))


def test_entry_point_validates_sizes_without_a_gpu():
    from diffmpc_b200 import _lib

    lib = _lib.load()
    assert lib.dmpc_psd_project(0, 3, None, 0.0, None, None) == _lib.DMPC_OK
    assert lib.dmpc_psd_project(1, 33, None, 0.0, None, None) == _lib.DMPC_ERR_INVALID
    assert lib.dmpc_psd_project(1, 0, None, 0.0, None, None) == _lib.DMPC_ERR_INVALID
    assert lib.dmpc_psd_project(-1, 3, None, 0.0, None, None) == _lib.DMPC_ERR_INVALID
    assert lib.dmpc_psd_project(2, 3, None, 0.0, None, None) == _lib.DMPC_ERR_INVALID
