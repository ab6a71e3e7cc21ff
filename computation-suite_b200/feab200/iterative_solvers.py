"""preconditioned_cg / jacobi_preconditioner with the reference's signatures
(iterative_solvers.py:193-202, :362-481), running on the GPU through libfeab200."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib as L
from .device import Pattern, ReducedOperator, cuda_device, pcg_solve


class JacobiPreconditioner:
    """M^-1 r = r / diag(A); callable on host arrays, and carries d_inv for the GPU solve."""

    def __init__(self, d_inv):
        self.d_inv = np.asarray(d_inv, dtype=float)

    def __call__(self, r):
        return self.d_inv * r


def jacobi_preconditioner(A):
    if isinstance(A, ReducedOperator):
        return JacobiPreconditioner(A.dinv64.cpu().numpy())
    d = np.asarray(sp.csr_matrix(A).diagonal(), dtype=float)
    if np.any(d == 0):
        raise ValueError("jacobi_preconditioner: A has a zero diagonal entry.")
    return JacobiPreconditioner(1.0 / d)


def operator_from_scipy(A, device=None):
    """Upload a host CSR matrix to the device (every row its own group)."""
    dev = cuda_device(device)
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    if A.shape != (n, n):
        raise ValueError("preconditioned_cg: A must be square")
    d = np.asarray(A.diagonal(), dtype=float)
    with np.errstate(divide="ignore"):
        dinv = np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 0.0)
    row_ptr = torch.as_tensor(A.indptr.astype(np.int32)).to(dev)
    col_idx = torch.as_tensor(A.indices.astype(np.int32)).to(dev)
    vals = torch.as_tensor(A.data.astype(np.float64)).to(dev)
    group_ptr = torch.arange(n + 1, dtype=torch.int32, device=dev)
    pat = Pattern(n, int(A.nnz), n, row_ptr, col_idx, group_ptr, torch.empty(0, dtype=torch.int32, device=dev))
    dinv_t = torch.as_tensor(dinv).to(dev)
    return ReducedOperator(pat, vals, vals.float(), dinv_t, dinv_t.float())


def preconditioned_cg(A, b, M=None, x0=None, tol=1e-8, maxiter=None, callback=None, backend="scipy",
                      device="cpu", precision="fp64"):
    """Returns (x, n_iter); LinAlgError when p^T A p <= 0, RuntimeError after maxiter (10 n)."""
    if backend not in ("scipy", "torch"):
        raise ValueError(f"preconditioned_cg: unknown backend={backend!r} -- expected 'scipy' (default) or 'torch'.")
    if callback is not None:
        raise TypeError("preconditioned_cg: callback= is not supported on the GPU path")
    op = A if isinstance(A, ReducedOperator) else operator_from_scipy(A, device)
    use_dinv = M is not None
    if use_dinv:
        if not isinstance(M, JacobiPreconditioner):
            raise NotImplementedError("preconditioned_cg: only the Jacobi preconditioner runs on the GPU path")
        dinv = torch.as_tensor(M.d_inv).to(op.vals64.device)
        op = ReducedOperator(op.pattern, op.vals64, op.vals32, dinv, dinv.float())
    b_t = torch.as_tensor(np.asarray(b, dtype=float)).to(op.vals64.device)
    x, info = pcg_solve(op, b_t, x0=x0, tol=tol, maxiter=maxiter, precision=precision, use_dinv=use_dinv)
    if info.status == L.FEAB_NOT_SPD:
        raise np.linalg.LinAlgError(f"preconditioned_cg: p^T A p <= 0 at iteration {info.iters + 1} -- A is not SPD.")
    if info.status == L.FEAB_NOT_CONVERGED:
        raise RuntimeError(f"preconditioned_cg: did not converge in {info.iters} iterations "
                           f"(final relative residual {info.relres:.3e} >= tol={tol:.1e}).")
    L.raise_for(info.status, "preconditioned_cg")
    return x.cpu().numpy(), info.iters
