"""NumPy model of the arithmetic of feab200's mixed-precision PCG (test helper, not a test).

It restates what the CUDA kernels compute for ``precision="mixed"``:
- the off-node entries of each row are stored with 36 mantissa bits (the double's bit pattern
  + 0x8000, low 16 bits cleared, as in k_sell_fill / k_build_diff);
- the own-node term is T x_a with T = S - (sum of the rounded off-node entries) in FP64,
  S being the exact row-block sums, so y = sum_{b != a} w~ x_b + T x_a;
- vectors and scalars are FP64; the recursive residual is replaced by the FP64 b - K x when it
  has dropped by `delta` since the last replacement or passed the tolerance, and convergence
  is declared only on that FP64 residual (the k_step_b rule).
The FP64 branch is the reference recurrence (iterative_solvers.py:434-481).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def round_mantissa(v, bits=36):
    """Round doubles to `bits` explicit mantissa bits (half up on the bit pattern)."""
    sh = 52 - bits
    u = np.ascontiguousarray(v, dtype=np.float64).view(np.uint64)
    u = (u + np.uint64(1 << (sh - 1))) & np.uint64((0xFFFFFFFFFFFFFFFF >> sh) << sh)
    return u.view(np.float64)


def difference_operator(Kff, free, bits=36):
    """y = K~ x for the reduced K (CSR over the free DOFs, `free` = their global DOF ids)."""
    node, comp = free // 3, free % 3
    K = Kff.tocoo()
    i, j, v = K.row, K.col, K.data
    w = np.where(node[i] == node[j], 0.0, round_mantissa(v, bits))
    S = np.zeros((len(free), 3))
    np.add.at(S, (i, comp[j]), v)
    W = np.zeros((len(free), 3))
    np.add.at(W, (i, comp[j]), w)
    T = S - W
    Wm = sp.csr_matrix((w, (i, j)), shape=Kff.shape)
    row_of = -np.ones(3 * (int(free.max()) + 1) + 3, np.int64)
    row_of[free] = np.arange(len(free))
    own = row_of[3 * node[:, None] + np.arange(3)[None, :]]

    def apply(x):
        xs = np.where(own >= 0, x[np.maximum(own, 0)], 0.0)
        return Wm @ x + (T * xs).sum(1)
    return apply


def pcg_iterations(Kff, b, dinv, tol, apply=None, delta=0.1, maxiter=100000):
    """(x, iterations, residual replacements).  apply=None: the FP64 recurrence; otherwise the
    mixed recurrence with `apply` as the stored operator."""
    mixed = apply is not None
    apply = apply or (lambda v: Kff @ v)
    x = np.zeros_like(b)
    r = b.copy()
    bn = np.linalg.norm(b) or 1.0
    z = dinv * r
    p = z.copy()
    rz = r @ z
    rmax = np.linalg.norm(r)
    k = reps = 0
    while k < maxiter:
        Ap = apply(p)
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        k += 1
        rn = np.linalg.norm(r)
        if mixed and (rn / bn < tol or rn < delta * rmax):
            r = b - Kff @ x
            rn = rmax = np.linalg.norm(r)
            reps += 1
            if rn / bn < tol:
                return x, k, reps
        elif not mixed and rn / bn < tol:
            return x, k, reps
        z = dinv * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    raise RuntimeError("no convergence")


def tip_loaded_cantilever(nx, ny, nz, E=210e9, nu=0.3):
    """2.0 x 0.4 x 0.4 box, x = 0 clamped, unit z load on every node of x = 2.0:
    (Kff CSR, b, dinv, free)."""
    import oracle as O
    X, el = O.box_mesh(2.0, 0.4, 0.4, nx, ny, nz)
    fixed = O.fixed_dofs_on_plane(X, 0, 0.0)
    free = O.free_dofs(3 * len(X), fixed)
    ke = O.hex8_element_stiffness(X[el], O.D_solid3d(E, nu))
    Kff = O.reduce_free(O.structural_csr(ke, el, 3 * len(X)), free).tocsr()
    F = np.zeros(3 * len(X))
    F[O.fixed_dofs_on_plane(X, 0, 2.0, dofs=(2,))] = 1.0
    return Kff, F[free], O.jacobi_inverse_diagonal(Kff), free
