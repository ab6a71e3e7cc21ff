"""The torch-backend solve entry points of fea_engine, by name, on the GPU PCG.

``torch_sparse_cg_solve`` and ``fesystem_solve_static_torch`` keep the reference's signatures,
return conventions and errors (fea_engine/src/fea_engine/torch_sparse_solver.py:205-265,
:268-314); the Jacobi-CG loop of ``_cg_torch`` (:165-202) runs as libfeab200's PCG
(feab_pcg_solve) instead of one torch op per vector update.

Contract kept from the reference:
- ``torch_sparse_cg_solve(K, F, tol, max_iter, device, dtype)`` takes a SciPy sparse matrix or
  a dense array, raises ValueError when a diagonal entry is not positive, and returns
  ``(x numpy (n,), n_iter, converged)`` without raising on non-convergence.  A zero right-hand
  side returns x = 0 after 0 iterations, converged.  A direction with p^T K p <= 0 (K not SPD)
  also ends the solve with converged = False.
- ``fesystem_solve_static_torch(sysobj, method, device, tol, max_iter)`` solves
  K_ff u_f = F_f for the system's free DOFs and returns the full (n_dof,) numpy vector with
  zeros at every fixed DOF (as the reference, no Dirichlet correction), raising RuntimeError
  when CG does not converge and ValueError for an unknown method.

Differences: ``device`` may name any CUDA device ("cpu" selects the current CUDA device; the
library has no CPU compute path); ``dtype=torch.float32`` runs the FP32 operator with FP64
residual replacement (libfeab200's FEAB_PREC_FP32), which converges on the FP64 residual;
``method="dense"`` (the reference's dense LU) runs the FP64 PCG to a relative residual of 1e-12,
since there is no dense factorisation on this path.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib as L
from .device import pcg_solve
from .iterative_solvers import operator_from_scipy


def _precision_of(dtype):
    if dtype is None or dtype == torch.float64:
        return "fp64"
    if dtype == torch.float32:
        return "fp32"
    raise ValueError(f"torch_sparse_cg_solve: dtype must be torch.float64 or torch.float32, got {dtype}")


def torch_sparse_cg_solve(K, F, tol=1e-8, max_iter=None, device="cpu", dtype=None):
    """Jacobi-preconditioned CG for an SPD K (torch_sparse_solver.py:205-265).
    Returns (x (n,) numpy array, n_iter, converged)."""
    precision = _precision_of(dtype)
    K_csr = sp.csr_matrix(K)
    n = K_csr.shape[0]
    diag = K_csr.diagonal()
    if np.any(diag <= 0):
        raise ValueError(
            "torch_sparse_cg_solve: K's diagonal has a non-positive entry -- K cannot be SPD (a necessary "
            "condition fails), so Conjugate Gradient is not applicable here. Use torch_dense_solve() instead "
            "for a non-SPD system.")
    b = np.asarray(F, dtype=float).reshape(-1)
    if b.shape[0] != n:
        raise ValueError(f"torch_sparse_cg_solve: F has {b.shape[0]} entries, K is {n} x {n}")
    if not np.any(b):
        return np.zeros(n), 0, True
    op = operator_from_scipy(K_csr, device)
    x, info = pcg_solve(op, torch.as_tensor(b).to(op.vals64.device), tol=tol,
                        maxiter=10 * n if max_iter is None else int(max_iter), precision=precision, layout="csr")
    if info.status not in (L.FEAB_OK, L.FEAB_NOT_CONVERGED, L.FEAB_NOT_SPD):
        L.raise_for(info.status, "torch_sparse_cg_solve")
    return x.cpu().numpy(), int(info.iters), info.status == L.FEAB_OK


def fesystem_solve_static_torch(sysobj, method="cg", device="cpu", tol=1e-8, max_iter=None):
    """The free-DOF solve of an assembled FESystem through the torch-backend contract
    (torch_sparse_solver.py:268-314).  Returns the full (n_dof,) numpy vector, zero at every
    fixed DOF."""
    if method not in ("cg", "dense"):
        raise ValueError(f"fesystem_solve_static_torch: unknown method={method!r}, expected 'cg' or 'dense'")
    free = sysobj.free_dofs
    op = sysobj.reduced_operator(want32=False)
    Ff = np.asarray(sysobj.F, dtype=float)[free]
    U = np.zeros(sysobj.n_dof)
    if not np.any(Ff):
        return U
    b = torch.as_tensor(Ff).to(op.vals64.device)
    if method == "cg":
        x, info = pcg_solve(op, b, tol=tol, maxiter=max_iter, precision="fp64")
        if info.status in (L.FEAB_NOT_CONVERGED, L.FEAB_NOT_SPD):
            raise RuntimeError(
                f"fesystem_solve_static_torch: CG did not converge within {info.iters} iterations (tol={tol}) -- "
                "Kff may not be SPD, or needs a tighter tol/more iterations/a better preconditioner than the "
                "Jacobi one used here; try method='dense' as a fallback or diagnostic.")
    else:
        # a direct solve, as the reference's torch_dense_solve: the banded Cholesky of K_ff
        # (feab200.direct); a K_ff that is not SPD, or singular, goes to a tight PCG instead
        x = None
        try:
            fac = op.direct_factor(coords=getattr(sysobj.mesh, "nodes", None))
            if not fac.near_singular:
                x = fac.solve(b)
        except (MemoryError, np.linalg.LinAlgError):
            x = None
        if x is None:
            x, info = pcg_solve(op, b, tol=1e-12, maxiter=max_iter, precision="fp64")
            if info.status in (L.FEAB_NOT_CONVERGED, L.FEAB_NOT_SPD):
                raise RuntimeError("fesystem_solve_static_torch: method='dense' found K_ff not SPD or singular, "
                                   "and the tight PCG it falls back to did not converge")
            L.raise_for(info.status, "fesystem_solve_static_torch")
        U[free] = x.cpu().numpy()
        return U
    L.raise_for(info.status, "fesystem_solve_static_torch")
    U[free] = x.cpu().numpy()
    return U
