"""Natural frequencies and mode shapes on the GPU (FESystem.solve_modal, solver.py:2047-2114).

The reference calls scipy.sparse.linalg.eigsh(Kff, k=n_modes, M=Mff, sigma=0): shift-invert
Lanczos on a sparse LU factorisation.  feab200 finds the same lowest eigenpairs of
K phi = lambda M phi by block subspace iteration (inverse iteration on a block of p > n_modes
vectors) with a Rayleigh-Ritz step, every product on the GPU:

    Y  = K^-1 (M X)                 block-PCG over the block of vectors (feab_block_pcg_solve),
                                     M X by the block SpMM (feab_block_spmm)
    Kr = Y^T K Y,  Mr = Y^T M Y      block SpMMs and FP64 panel Grams (feab_panel_gram)
    Kr v = lambda Mr v               Mr = Q L Q^T, then the eigenpairs of L^-1/2 Q^T Kr Q L^-1/2
                                     (feab_symeig_jacobi, one CTA, k <= 64; p x p products only)
    X  = Y V                         M-orthonormal Ritz vectors, lambda ascending (feab_panel_small)

until the n_modes lowest Ritz values change by less than ``tol`` (relative), or stop decreasing
once the change is below ``1e3 * tol`` (round-off, not convergence, then sets it).  Ritz values converge
like (lambda_i / lambda_{p+1})^(2j), so the block is wider than the number of modes asked for.
"""
from __future__ import annotations

import numpy as np
import torch

from .batched import block_pcg, panel_width
from .device import ReducedOperator
from .panel import block_spmm, panel_gram, panel_small
from .pod import symeig


def _generalized_eig(Kr, Mr):
    """Eigenpairs of Kr v = lambda Mr v (Kr, Mr symmetric, Mr positive definite), lambda ascending
    and V^T Mr V = I."""
    lm, Q = symeig(Mr)
    if not bool((lm > 0).all()):
        raise np.linalg.LinAlgError("solve_modal: the subspace lost rank (M-Gram matrix not positive definite)")
    S = Q * lm.rsqrt()[None, :]
    A = S.t() @ Kr @ S
    A = 0.5 * (A + A.t())
    w, W = symeig(A)
    order = torch.argsort(w)
    return w[order], S @ W[:, order]


def subspace_iteration(Kop: ReducedOperator, Mop: ReducedOperator, n_modes, subspace=None, tol=1e-12, maxiter=300,
                       pcg_tol=1e-10, seed=0):
    """The n_modes lowest eigenpairs of Kff phi = lambda Mff phi.  Returns (lambda (n_modes,)
    device, Phi (n, n_modes) device, M-orthonormal, iterations)."""
    n = Kop.n
    if not (1 <= n_modes < n):
        raise ValueError(f"solve_modal: n_modes must be in [1, {n - 1}] for {n} free DOFs, got {n_modes}")
    p = int(subspace) if subspace else max(2 * n_modes, n_modes + 8)
    p = max(n_modes, min(p, n, 64))
    K = panel_width(p)
    dev = Kop.vals64.device
    g = torch.Generator(device=dev).manual_seed(int(seed))
    X = torch.zeros((n, K), dtype=torch.float64, device=dev)      # panel of width K, columns >= p zero
    X[:, :p] = torch.randn((n, p), generator=g, dtype=torch.float64, device=dev)
    B = torch.empty((n, K), dtype=torch.float64, device=dev)
    KY = torch.empty_like(B)
    MY = torch.empty_like(B)
    lam_old = None
    change_old = None
    for it in range(1, maxiter + 1):
        block_spmm(Mop, X, out=B)
        Y, res = block_pcg(Kop, np.array([0, n]), B, [p], tol=pcg_tol)
        if not (res.status == 0).all():
            raise RuntimeError(f"solve_modal: the inner block-PCG did not converge (status {res.status.tolist()})")
        block_spmm(Kop, Y, out=KY)
        block_spmm(Mop, Y, out=MY)
        Kr = panel_gram(Y[:, :p], KY[:, :p])
        Mr = panel_gram(Y[:, :p], MY[:, :p])
        lam, V = _generalized_eig(0.5 * (Kr + Kr.t()), 0.5 * (Mr + Mr.t()))
        X[:, :p] = panel_small(Y[:, :p], V)
        low = lam[:n_modes]
        if lam_old is not None:
            change = float(((low - lam_old).abs() / low.abs().clamp_min(1e-300)).max())
            if change < tol or (change_old is not None and change >= change_old and change < 1e3 * tol):
                break
            change_old = change
        lam_old = low.clone()
    return lam[:n_modes], X[:, :n_modes].contiguous(), it
