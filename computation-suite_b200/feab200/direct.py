"""Direct solve of the reduced system on the GPU: a banded tile Cholesky factorisation.

The reference's default static solve (FESystem.solve_static with method=None on a sparse
system) is FESystem._sparse_lu_solve (fea_engine/src/fea_engine/solver.py:1681-1724): SuperLU's
splu of K_ff, a singularity test on its pivots (min |U_ii| < tol max |U_ii|, tol 1e-10), then
lu.solve.  K_ff is SPD, so its LU factorisation without pivoting is the Cholesky factorisation
K_ff = L L^T with U_ii = L_ii^2; the same pivot test is made on the Cholesky pivots.

The free DOFs are renumbered node by node in reverse Cuthill-McKee order of the node graph (the
ordering is host-side preprocessing, as SuperLU's column ordering is in the reference), so that
the band of the renumbered K_ff is narrow; the band is factored and solved on the GPU with the
feab_band_* kernels (64 x 64 tiles).  The factor of an operator is computed once and reused for
every right-hand side.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L

PIVOT_TOL = 1e-10        # the reference's _sparse_lu_solve default
TILE = 64


def node_order(op):
    """Reverse Cuthill-McKee order of the node row groups of op (int64 array of group ids).
    The node graph is formed on the device from each group's column list; its edges go to the
    host for SciPy's reverse_cuthill_mckee."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    p = op.pattern
    dev = op.vals64.device
    gp = p.group_ptr.to(torch.int64)
    G = gp.numel() - 1
    sizes = gp[1:] - gp[:-1]
    row_group = torch.repeat_interleave(torch.arange(G, device=dev), sizes)
    rp = p.row_ptr.to(torch.int64)
    starts, lens = rp[gp[:-1]], rp[gp[:-1] + 1] - rp[gp[:-1]]
    src = torch.repeat_interleave(torch.arange(G, device=dev), lens)
    off = torch.arange(int(lens.sum()), device=dev) - torch.repeat_interleave(torch.cumsum(lens, 0) - lens, lens)
    nbr = row_group[p.col_idx.to(torch.int64)[torch.repeat_interleave(starts, lens) + off]]
    keep = torch.ones_like(nbr, dtype=torch.bool)
    keep[1:] = (nbr[1:] != nbr[:-1]) | (src[1:] != src[:-1])   # the DOFs of one neighbour are adjacent
    src, nbr = src[keep].cpu().numpy(), nbr[keep].cpu().numpy()
    g = sp.csr_matrix((np.ones(src.size, np.int8), (src, nbr)), shape=(G, G))
    return np.asarray(reverse_cuthill_mckee(g, symmetric_mode=True), dtype=np.int64)


def coordinate_order(op, coords):
    """Node row groups sorted by their node's coordinate along the mesh's longest extent (then
    the other two): on an elongated mesh the band is about one cross-section of nodes wide."""
    X = np.asarray(coords, dtype=float)
    fm = op.pattern.free_map
    dof_of_row = torch.nonzero(fm >= 0).flatten().cpu().numpy()
    gp = op.pattern.group_ptr.cpu().numpy().astype(np.int64)
    key = X[dof_of_row[gp[:-1]] // 3]
    ax = np.argsort(np.ptp(key, axis=0))          # ascending extent: the longest axis is last
    return np.lexsort((key[:, ax[0]], key[:, ax[1]], key[:, ax[2]])).astype(np.int64)


def dof_permutation(op, order):
    """iperm (old reduced row -> new row, int32 device tensor) for the node order `order`."""
    gp = op.pattern.group_ptr.cpu().numpy().astype(np.int64)
    sz = (gp[1:] - gp[:-1])[order]
    old = np.repeat(gp[order], sz) + (np.arange(int(sz.sum())) - np.repeat(np.cumsum(sz) - sz, sz))
    iperm = np.empty(op.n, np.int32)
    iperm[old] = np.arange(op.n, dtype=np.int32)
    return torch.as_tensor(iperm).to(op.vals64.device)


class BandCholesky:
    """K_ff = L L^T on the device, in the renumbered order.  Raises MemoryError when the band
    would take more than `max_fraction` of the device's free memory."""

    def __init__(self, op, coords=None, max_fraction=0.6):
        """coords: the mesh's node coordinates (N, 3), if known: the ordering along the longest
        axis is then tried beside reverse Cuthill-McKee, and the narrower band is kept."""
        self.op = op
        dev = op.vals64.device
        if op.pattern.group_ptr is None:
            raise ValueError("the direct solve needs node row groups (an assembled K_ff)")
        csr = op.csr_struct()
        scratch = torch.zeros(2, dtype=torch.int32, device=dev)
        orders = {"rcm": node_order(op)}
        if coords is not None:
            orders["axis"] = coordinate_order(op, coords)
        best = None
        for name, order in orders.items():
            iperm = dof_permutation(op, order)
            bw = C.c_int32(0)
            rc = L.lib.feab_band_width(C.byref(csr), L.dptr(iperm), L.dptr(scratch), C.byref(bw), L.stream_ptr(dev))
            L.raise_for(rc, "band width")
            if best is None or bw.value < best[1]:
                best = (iperm, int(bw.value), name)
        self.iperm, self.bandwidth, self.ordering = best
        nbytes = int(L.lib.feab_band_bytes(op.n, self.bandwidth))
        free, _ = torch.cuda.mem_get_info(dev)
        if nbytes > max_fraction * free:
            raise MemoryError(f"banded Cholesky of n={op.n} (bandwidth {self.bandwidth}) needs {nbytes / 1e9:.1f} GB, "
                              f"more than {max_fraction:.0%} of the {free / 1e9:.1f} GB free on the device")
        self.storage = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.band = L.Band(0, 0, 0, 0, self.storage.data_ptr())
        rc = L.lib.feab_band_assemble(C.byref(csr), L.dptr(self.iperm), self.bandwidth, C.byref(self.band),
                                      L.stream_ptr(dev))
        L.raise_for(rc, "band assembly")
        piv = (C.c_double * 2)()
        rc = L.lib.feab_band_cholesky(C.byref(self.band), piv, L.stream_ptr(dev))
        self.pivots = (float(piv[0]), float(piv[1]))
        if rc == L.FEAB_NOT_SPD:
            raise np.linalg.LinAlgError("banded Cholesky: a pivot <= 0 -- K_ff is not SPD")
        L.raise_for(rc, "banded Cholesky")
        self.padded = int(self.band.n_tiles) * TILE

    @property
    def near_singular(self):
        """The reference's test on the factor's pivots: min < 1e-10 max."""
        lo, hi = self.pivots
        return not (lo >= PIVOT_TOL * hi)

    def solve(self, b):
        """x = K_ff^{-1} b (b: (n,) host or device array; returns an FP64 device tensor)."""
        op = self.op
        dev = op.vals64.device
        b = torch.as_tensor(b, dtype=torch.float64).to(dev).reshape(-1)
        if b.numel() != op.n:
            raise ValueError(f"b must have {op.n} entries, got {b.numel()}")
        bp = torch.zeros(self.padded, dtype=torch.float64, device=dev)
        bp[self.iperm.long()] = b
        xp = torch.empty_like(bp)
        work = torch.empty_like(bp)
        rc = L.lib.feab_band_solve(C.byref(self.band), L.dptr(bp), L.dptr(xp), L.dptr(work), L.stream_ptr(dev))
        L.raise_for(rc, "banded Cholesky solve")
        return xp[self.iperm.long()]
