"""Panel products on the device through libfeab200 (no cuBLAS on n-length panels).

- ``block_spmm(op, X)``: K X for a row-major n x k panel (feab_block_spmm, the block-PCG's SpMM);
- ``panel_gram(X, Y)``: X^T Y for n x k panels (feab_panel_gram, FP64, deterministic);
- ``panel_small(Y, V)``: Y V for an n x k panel and a small k x m matrix (feab_panel_small).
They carry the modal subspace iteration's Rayleigh-Ritz steps and the POD mode formation."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .device import ReducedOperator

WIDTHS = (1, 2, 4, 8, 16, 32, 64)


def _f64_panel(X, what):
    if not isinstance(X, torch.Tensor) or X.dtype != torch.float64 or X.ndim != 2 or not X.is_cuda:
        raise ValueError(f"{what} must be a 2-D float64 CUDA tensor")
    if X.stride(1) != 1:
        X = X.contiguous()
    return X


def block_spmm(op: ReducedOperator, X, out=None, node_tiles=False):
    """K X for an (n, k) device panel, k a power of two <= 64: one warp per node row group at
    four resident CTAs per SM (the faster form at every size measured), or, with node_tiles,
    through the operator's node tiles (``ReducedOperator.tile_operator``)."""
    X = _f64_panel(X, "X").contiguous()
    n, k = X.shape
    if n != op.n or k not in WIDTHS:
        raise ValueError(f"block_spmm: X must be ({op.n}, k) with k in {WIDTHS}, got {tuple(X.shape)}")
    Y = out if out is not None else torch.empty_like(X)
    csr = op.csr_struct()
    tiles = C.byref(op.tile_operator("fp64")) if node_tiles else None
    rc = L.lib.feab_block_spmm(C.byref(csr), tiles, L.dptr(X), L.dptr(Y), k, L.stream_ptr(X.device))
    L.raise_for(rc, "block_spmm")
    return Y


def panel_gram(X, Y):
    """X^T Y (k x k) for (n, k) device panels (row stride may exceed k), k <= 64."""
    X, Y = _f64_panel(X, "X"), _f64_panel(Y, "Y")
    if X.shape != Y.shape or X.shape[1] > 64:
        raise ValueError("panel_gram: X and Y must have the same shape (n, k <= 64)")
    n, k = X.shape
    ws = torch.empty(int(L.lib.feab_panel_gram_workspace_bytes(n)), dtype=torch.uint8, device=X.device)
    G = torch.empty((k, k), dtype=torch.float64, device=X.device)
    rc = L.lib.feab_panel_gram(L.dptr(X), X.stride(0), L.dptr(Y), Y.stride(0), n, k, L.dptr(G), L.dptr(ws),
                               ws.numel(), L.stream_ptr(X.device))
    L.raise_for(rc, "panel_gram")
    return G


def panel_small(Y, V):
    """Y V for an (n, k) device panel and a (k, m) device matrix, k, m <= 64."""
    Y = _f64_panel(Y, "Y")
    V = _f64_panel(V, "V").contiguous()
    n, k = Y.shape
    if V.shape[0] != k or V.shape[1] > 64 or k > 64:
        raise ValueError(f"panel_small: V must be ({k}, m <= 64), got {tuple(V.shape)}")
    m = V.shape[1]
    Z = torch.empty((n, m), dtype=torch.float64, device=Y.device)
    rc = L.lib.feab_panel_small(L.dptr(Y), Y.stride(0), n, k, L.dptr(V), m, L.dptr(Z), m, L.stream_ptr(Y.device))
    L.raise_for(rc, "panel_small")
    return Z
