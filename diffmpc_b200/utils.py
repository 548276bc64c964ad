"""GPU counterparts of the reference's matrix utilities (diffmpc/utils/jax_utils.py)."""

import torch

from . import _lib


def project_matrix_onto_positive_semidefinite_cone(matrix: torch.Tensor, minimum_eigenvalue: float = 0.0) -> torch.Tensor:
    """Projects symmetric matrices onto the positive semi-definite cone (jax_utils.py:75-95).

    ``matrix``: (..., n, n) float64 CUDA tensor, n <= 32; every leading index is one matrix.
    Returns V diag(max(S, minimum_eigenvalue)) V^T, symmetrized, where S, V is the eigen-
    decomposition of the symmetrized input (jnp.linalg.eigh symmetrizes by default).  The
    eigen-decomposition runs on the GPU (``dmpc_psd_project``: FP64 Jacobi, one warp per matrix);
    a CPU tensor is an error, as there is no host path.
    """
    if not isinstance(matrix, torch.Tensor) or not matrix.is_cuda:
        raise ValueError("project_matrix_onto_positive_semidefinite_cone needs a CUDA tensor")
    if matrix.dim() < 2 or matrix.shape[-1] != matrix.shape[-2]:
        raise ValueError(f"expected (..., n, n) matrices, got shape {tuple(matrix.shape)}")
    n = matrix.shape[-1]
    m = matrix.to(torch.float64).contiguous()
    out = torch.empty_like(m)
    batch = m.numel() // (n * n) if n > 0 else 0
    lib = _lib.load()
    with torch.cuda.device(m.device):
        _lib.check(lib.dmpc_psd_project(batch, n, m.data_ptr(), float(minimum_eigenvalue), out.data_ptr(),
                                        torch.cuda.current_stream(m.device).cuda_stream), "dmpc_psd_project")
    return out
