"""NumPy/SciPy restatement of the reference's hex8 static path (test infrastructure).

Citations are ``file:line`` inside abhi2k16/computation-suite.  The restatement
follows the reference's algorithm and operation order where it matters for
parity (quadrature order, signed det J, CSR built by COO duplicate summation,
the PCG recurrence and its stopping rule); it is vectorised over elements so
that it stays usable at the large mesh sizes.

Only tests, the smoke check and the CPU-baseline leg of the benchmark use this
module.
"""
from __future__ import annotations

import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

__all__ = [
    "gauss_legendre", "box_mesh", "perturb_interior", "D_solid3d", "hex8_shape_and_derivs",
    "hex8_element_stiffness", "hex8_bbar_element_stiffness", "hex8_element_mass", "modal", "global_dofs", "structural_csr", "structural_pattern", "reduce_free", "fixed_dofs_on_plane",
    "free_dofs", "quad4_shape_and_derivs", "HEX8_FACES", "facet_load_shares", "facet_mass",
    "jacobi_inverse_diagonal", "preconditioned_cg", "simp_scale", "simp_scale_grad",
    "compliance_sensitivity_closed_form", "pod_singular_values", "element_strain_energy_density",
    "recover", "von_mises", "reactions", "build_filter_weights", "apply_sensitivity_filter", "oc_update",
    "topology_optimize_compliance",
]


# ----------------------------------------------------------------------------- quadrature
def gauss_legendre(n):
    """n-point Gauss-Legendre rule on [-1, 1] (fea_engine/src/fea_engine/elements/base.py:73-78)."""
    return np.polynomial.legendre.leggauss(n)


def _gauss_product_3d(n):
    """Tensor-product rule, xi outer, eta middle, zeta inner (elements/base.py:81-95)."""
    p, w = gauss_legendre(n)
    pts = [(a, b, c) for a in p for b in p for c in p]
    wts = [wa * wb * wc for wa in w for wb in w for wc in w]
    return pts, wts


# ----------------------------------------------------------------------------- mesh
def box_mesh(Lx, Ly, Lz, nx, ny, nz):
    """Structured hex8 box.

    rectangle_mesh (fea_engine/src/fea_engine/mesh.py:716-733): node (i, j) has id
    i*(ny+1)+j at (i*dx, j*dy); quad (i, j) = [(i,j), (i+1,j), (i+1,j+1), (i,j+1)],
    i outer.  extrude_mesh (mesh.py:1270-1285): layer k holds the 2-D nodes at
    z = linspace(0, Lz, nz+1)[k]; element = [quad + k*n2d, quad + (k+1)*n2d], k outer.
    box_mesh = extrude(rectangle) (mesh.py:1288-1289).
    """
    dx, dy = Lx / nx, Ly / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    nodes2d = np.zeros(((nx + 1) * (ny + 1), 2))
    nodes2d[(ii * (ny + 1) + jj).ravel(), 0] = (0.0 + ii * dx).ravel()
    nodes2d[(ii * (ny + 1) + jj).ravel(), 1] = (0.0 + jj * dy).ravel()
    qi, qj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    qi, qj = qi.ravel(), qj.ravel()
    nid = lambda i, j: i * (ny + 1) + j  # noqa: E731
    quads = np.stack([nid(qi, qj), nid(qi + 1, qj), nid(qi + 1, qj + 1), nid(qi, qj + 1)], axis=1)
    n2d = nodes2d.shape[0]
    z = 0.0 + np.linspace(0.0, Lz, nz + 1)
    nodes = np.zeros((n2d * (nz + 1), 3))
    for k in range(nz + 1):
        nodes[k * n2d:(k + 1) * n2d, 0:2] = nodes2d
        nodes[k * n2d:(k + 1) * n2d, 2] = z[k]
    elems = np.concatenate([np.concatenate([quads + k * n2d, quads + (k + 1) * n2d], axis=1)
                            for k in range(nz)], axis=0)
    return nodes, elems.astype(np.int64)


def perturb_interior(nodes, h, amp, seed):
    """Interior-node jitter in the style of fea_engine/tests/test_benchmarks_convergence.py:65-72:
    X[inner] += amp * h * (U[0,1) - 0.5), inner = strictly inside the bounding box, with a
    per-axis element size h (the configs quote the noise as a fraction of the element size)."""
    rng = np.random.default_rng(seed)
    X = np.array(nodes, dtype=float, copy=True)
    lo, hi = X.min(0), X.max(0)
    inner = np.all((X > lo + 1e-9) & (X < hi - 1e-9), axis=1)
    X[inner] += amp * np.asarray(h, dtype=float) * (rng.random((int(inner.sum()), X.shape[1])) - 0.5)
    return X


# ----------------------------------------------------------------------------- material
def D_solid3d(E, nu):
    """Isotropic 6x6 D, Voigt order xx,yy,zz,xy,yz,zx with engineering shear
    (fea_engine/src/fea_engine/material.py:650-660)."""
    c = E / ((1 + nu) * (1 - 2 * nu))
    g = (1 - 2 * nu) / 2
    return c * np.array([
        [1 - nu, nu, nu, 0, 0, 0],
        [nu, 1 - nu, nu, 0, 0, 0],
        [nu, nu, 1 - nu, 0, 0, 0],
        [0, 0, 0, g, 0, 0],
        [0, 0, 0, 0, g, 0],
        [0, 0, 0, 0, 0, g]])


# ----------------------------------------------------------------------------- element
_XI = np.array([-1, 1, 1, -1, -1, 1, 1, -1], dtype=float)
_ETA = np.array([-1, -1, 1, 1, -1, -1, 1, 1], dtype=float)
_ZETA = np.array([-1, -1, -1, -1, 1, 1, 1, 1], dtype=float)


def hex8_shape_and_derivs(xi, eta, zeta):
    """Trilinear shape functions and natural derivatives
    (fea_engine/src/fea_engine/elements/solids.py:133-142).  Returns N (8,), dN (3, 8)."""
    N = 0.125 * (1 + xi * _XI) * (1 + eta * _ETA) * (1 + zeta * _ZETA)
    dxi = 0.125 * _XI * (1 + eta * _ETA) * (1 + zeta * _ZETA)
    deta = 0.125 * _ETA * (1 + xi * _XI) * (1 + zeta * _ZETA)
    dzeta = 0.125 * _ZETA * (1 + xi * _XI) * (1 + eta * _ETA)
    return N, np.vstack([dxi, deta, dzeta])


def _b_matrices(dN_g):
    """B (E, 6, 24) from physical gradients dN_g (E, 3, 8); row order as
    elements/solids.py:150-162 (xx, yy, zz, xy, yz, zx)."""
    E = dN_g.shape[0]
    B = np.zeros((E, 6, 24))
    dx, dy, dz = dN_g[:, 0, :], dN_g[:, 1, :], dN_g[:, 2, :]
    c = 3 * np.arange(8)
    B[:, 0, c] = dx
    B[:, 1, c + 1] = dy
    B[:, 2, c + 2] = dz
    B[:, 3, c] = dy
    B[:, 3, c + 1] = dx
    B[:, 4, c + 1] = dz
    B[:, 4, c + 2] = dy
    B[:, 5, c] = dz
    B[:, 5, c + 2] = dx
    return B


def _gauss_geometry(coords):
    """Yield (w, detJ (E,), dN_g (E,3,8)) per Gauss point, following
    Hex8Solid3D.B_matrix + jacobian (elements/solids.py:144-149, elements/base.py:268-277):
    J = dN @ X, detJ = det(J), dN_g = solve(J, dN).  Degenerate |detJ| < 1e-300 raises
    ValueError like MeshTransformation (fea_engine/src/fea_engine/mesh_transform.py:327-332)."""
    coords = np.asarray(coords, dtype=float)
    pts, wts = _gauss_product_3d(2)
    for p, w in zip(pts, wts):
        _, dN = hex8_shape_and_derivs(*p)
        J = np.einsum("in,enj->eij", dN, coords)
        detJ = np.linalg.det(J)
        if np.any(np.abs(detJ) < 1e-300):
            raise ValueError("degenerate element(s) found (near-zero detJ)")
        dN_g = np.linalg.solve(J, np.broadcast_to(dN, (coords.shape[0], 3, 8)))
        yield w, detJ, dN_g


def hex8_element_stiffness(coords, D, thickness=1.0):
    """All element stiffness matrices ke (E, 24, 24) = sum_gp B^T D B detJ w thickness
    (Element.stiffness, fea_engine/src/fea_engine/elements/base.py:494-514; signed detJ)."""
    coords = np.asarray(coords, dtype=float)
    D = np.asarray(D, dtype=float)
    ke = np.zeros((coords.shape[0], 24, 24))
    for w, detJ, dN_g in _gauss_geometry(coords):
        B = _b_matrices(dN_g)
        ke += np.matmul(np.transpose(B, (0, 2, 1)), np.matmul(D, B)) * (detJ * w * thickness)[:, None, None]
    return ke


def hex8_element_mass(coords, R, thickness=1.0):
    """Consistent element mass me = sum_gp Nm^T R Nm |detJ| w thickness (Element.mass,
    fea_engine/src/fea_engine/elements/base.py:711-731; Nm the 3 x 24 block expansion of N, N_matrix
    :475-487).  coords (E, 8, 3), R the 3x3 density matrix.  Returns (E, 24, 24)."""
    coords = np.asarray(coords, dtype=float)
    R = np.asarray(R, dtype=float)
    me = np.zeros((coords.shape[0], 24, 24))
    pts, _ = _gauss_product_3d(2)
    for (w, detJ, _), p in zip(_gauss_geometry(coords), pts):
        N, _ = hex8_shape_and_derivs(*p)
        Nm = np.zeros((3, 24))
        for a in range(8):
            Nm[:, 3 * a:3 * a + 3] = N[a] * np.eye(3)
        me += (Nm.T @ R @ Nm)[None, :, :] * (np.abs(detJ) * w * thickness)[:, None, None]
    return me


def modal(Kff, Mff, n_modes):
    """Lowest eigenpairs of Kff phi = w^2 Mff phi by shift-invert Lanczos, as FESystem.solve_modal
    (solver.py:2047-2114): scipy.sparse.linalg.eigsh(Kff, k, M=Mff, sigma=0).  Returns
    (freq_hz (n_modes,), modes (n_free, n_modes), M-orthonormal)."""
    w2, vecs = spla.eigsh(sp.csc_matrix(Kff), k=n_modes, M=sp.csc_matrix(Mff), sigma=0, which="LM")
    order = np.argsort(w2)
    w2, vecs = np.clip(w2[order], 0, None), vecs[:, order]
    return np.sqrt(w2) / (2 * np.pi), vecs


def hex8_bbar_element_stiffness(coords, D, thickness=1.0):
    """Element stiffness of Hex8SolidBbar (fea_engine/src/fea_engine/elements/solids.py:228-257):
    at each Gauss point B-bar = B - P B + P Bavg, P = m m^T / 3 (m = [1 1 1 0 0 0]),
    Bavg = sum_q B detJ w / sum_q detJ w (signed detJ); ke = sum_q B-bar^T D B-bar detJ w."""
    coords = np.asarray(coords, dtype=float)
    D = np.asarray(D, dtype=float)
    m = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    P = np.outer(m, m) / 3.0
    geo = [(w, detJ, _b_matrices(dN_g)) for w, detJ, dN_g in _gauss_geometry(coords)]
    vol = sum(detJ * w for w, detJ, _ in geo)
    Bavg = sum(np.matmul(P, B) * (detJ * w)[:, None, None] for w, detJ, B in geo) / vol[:, None, None]
    ke = np.zeros((coords.shape[0], 24, 24))
    for w, detJ, B in geo:
        Bb = B - np.matmul(P, B) + Bavg
        ke += np.matmul(np.transpose(Bb, (0, 2, 1)), np.matmul(D, Bb)) * (detJ * w * thickness)[:, None, None]
    return ke


def element_strain_energy_density(coords, D, u_e, v_e=None):
    """sum_gp eps(v)^T D eps(u) detJ w per element, which equals v_e^T ke_e u_e
    (the quadratic form inside topopt.py:161-177's einsum('ei,eij,ej->e'))."""
    v_e = u_e if v_e is None else v_e
    out = np.zeros(np.asarray(coords).shape[0])
    for w, detJ, dN_g in _gauss_geometry(coords):
        B = _b_matrices(dN_g)
        eu = np.einsum("esm,em->es", B, u_e)
        ev = np.einsum("esm,em->es", B, v_e)
        out += np.einsum("es,st,et->e", ev, D, eu) * detJ * w
    return out


# ----------------------------------------------------------------------------- assembly
def global_dofs(conn, dofs_per_node=3):
    """g[e] = dofs_per_node*node + local dof (vectorized_assembly.py:249-251,
    FESystem._global_dofs solver.py:275-280)."""
    conn = np.asarray(conn)
    E, nb = conn.shape
    return (dofs_per_node * conn[:, :, None] + np.arange(dofs_per_node)[None, None, :]).reshape(E, nb * dofs_per_node)


def structural_csr(ke, conn, n_dof, dofs_per_node=3):
    """COO (row = repeat(g), col = tile(g), data = ke) -> CSR with duplicates summed
    (scatter_global_stiffness, fea_engine/src/fea_engine/vectorized_assembly.py:217-262).
    Keeps the full structural pattern, exact zeros included."""
    g = global_dofs(conn, dofs_per_node)
    E, m = g.shape
    row = np.repeat(g, m, axis=1).reshape(-1)
    col = np.tile(g, (1, m)).reshape(-1)
    K = sp.coo_matrix((np.asarray(ke).reshape(-1), (row, col)), shape=(n_dof, n_dof))
    return K.tocsr()


def structural_pattern(conn, n_dof, free, dofs_per_node=3):
    """(indptr, indices) of the free x free structural pattern alone: the COO of
    scatter_global_stiffness (vectorized_assembly.py:217-262, row = repeat(g), col = tile(g))
    with a one-byte placeholder value, summed by SciPy's COO -> CSR, then
    K[np.ix_(free, free)] (solver.py:1977-1978).  It is the pattern of
    reduce_free(structural_csr(...)) without forming the element matrices, for meshes whose
    FP64 COO would not fit in host memory."""
    g = global_dofs(conn, dofs_per_node).astype(np.int32)
    E, m = g.shape
    row = np.repeat(g, m, axis=1).reshape(-1)
    col = np.tile(g, (1, m)).reshape(-1)
    K = sp.coo_matrix((np.ones(row.shape[0], dtype=np.int8), (row, col)), shape=(n_dof, n_dof)).tocsr()
    del row, col
    Kff = K[np.ix_(free, free)]
    Kff.sort_indices()
    return Kff.indptr, Kff.indices


def reduce_free(K, free):
    """Kff = K.tocsr()[np.ix_(free, free)] (solver.py:1977-1978, form_linear_system :1434-1435)."""
    return sp.csr_matrix(K)[np.ix_(free, free)]


def fixed_dofs_on_plane(nodes, axis=0, value=0.0, dofs=(0, 1, 2), dofs_per_node=3, tol=1e-9):
    """Sorted fixed DOFs for every node on a coordinate plane: Mesh.nodes_on_plane
    (mesh.py:330-332) + FESystem.fix_dofs (solver.py:1163-1176) + fixed_dofs_array (:1482-1487)."""
    ids = np.where(np.abs(np.asarray(nodes)[:, axis] - value) < tol)[0]
    return np.array(sorted(dofs_per_node * int(n) + int(k) for n in ids for k in dofs), dtype=np.int64)


def free_dofs(n_dof, fixed):
    """Sorted complement of the fixed set (FESystem.free_dofs, solver.py:1400-1401)."""
    mask = np.ones(n_dof, dtype=bool)
    mask[np.asarray(fixed, dtype=np.int64)] = False
    return np.flatnonzero(mask)


# ----------------------------------------------------------------------------- facet loads
# Hex8 face table (fea_engine/src/fea_engine/facet_loads.py:172-179): local node ids per face.
HEX8_FACES = ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7))


def quad4_shape_and_derivs(xi, eta):
    """Bilinear facet shape functions (Quad4PlaneStress.shape_and_derivs,
    fea_engine/src/fea_engine/elements/solids.py:20-26)."""
    N = 0.25 * np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
    dxi = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
    deta = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
    return N, np.vstack([dxi, deta])


def _facet_points(quad_order):
    n = max(1, int(np.ceil((quad_order + 1) / 2)))
    p, w = gauss_legendre(n)
    return [(a, b) for a in p for b in p], [wa * wb for wa in w for wb in w]


def _facet_measure(dN, fc):
    """Gram determinant sqrt(det(J J^T)) for a 2-D facet in 3-D (elements/base.py:308-311)."""
    J = np.einsum("in,fnj->fij", dN, fc)
    G = np.einsum("fij,fkj->fik", J, J)
    return np.sqrt(np.maximum(np.linalg.det(G), 0.0))


def facet_load_shares(facet_coords, traction, quad_order=2):
    """Consistent nodal shares of a uniform traction on quad4 faces, (F, 4)
    (consistent_facet_load_shares, fea_engine/src/fea_engine/facet_loads.py:283-325)."""
    fc = np.asarray(facet_coords, dtype=float)
    share = np.zeros((fc.shape[0], 4))
    pts, wts = _facet_points(quad_order)
    for p, w in zip(pts, wts):
        N, dN = quad4_shape_and_derivs(*p)
        share += N[None, :] * traction * (_facet_measure(dN, fc) * w)[:, None]
    return share


def facet_mass(facet_coords, coefficient=1.0, quad_order=2):
    """Consistent facet 'mass' integral c N_a N_b over quad4 faces, (F, 4, 4)
    (consistent_facet_mass, fea_engine/src/fea_engine/facet_loads.py:263-280)."""
    fc = np.asarray(facet_coords, dtype=float)
    out = np.zeros((fc.shape[0], 4, 4))
    pts, wts = _facet_points(quad_order)
    for p, w in zip(pts, wts):
        N, dN = quad4_shape_and_derivs(*p)
        out += (coefficient * _facet_measure(dN, fc) * w)[:, None, None] * np.outer(N, N)[None]
    return out


# ----------------------------------------------------------------------------- solve
def jacobi_inverse_diagonal(A):
    """d_inv = 1/diag(A); ValueError on a zero diagonal
    (jacobi_preconditioner, fea_engine/src/fea_engine/iterative_solvers.py:193-202)."""
    d = np.asarray(sp.csr_matrix(A).diagonal(), dtype=float)
    if np.any(d == 0):
        raise ValueError("jacobi_preconditioner: A has a zero diagonal entry.")
    return 1.0 / d


def preconditioned_cg(A, b, d_inv=None, x0=None, tol=1e-8, maxiter=None, history=None):
    """Hestenes-Stiefel PCG with the reference's exact control flow
    (preconditioned_cg, fea_engine/src/fea_engine/iterative_solvers.py:362-481, SciPy branch
    :434-481): x0 = 0, bnorm = ||b|| (1 if zero), early exit when ||r0||/bnorm < tol,
    LinAlgError when p^T A p <= 0, convergence tested right after the r update, RuntimeError
    after maxiter = 10 n.  Returns (x, n_iter, final relative residual).  ``history``, if a
    list, receives (time.perf_counter(), relative residual) after every iteration, so that one
    tight solve also gives the time and iterate at any looser tolerance."""
    A = sp.csr_matrix(A)
    b = np.asarray(b, dtype=float)
    n = b.shape[0]
    if maxiter is None:
        maxiter = 10 * n
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=float)
    bnorm = np.linalg.norm(b)
    if bnorm == 0.0:
        bnorm = 1.0
    r = b - A @ x
    rel = np.linalg.norm(r) / bnorm
    if rel < tol:
        return x, 0, rel
    Minv = (lambda v: v) if d_inv is None else (lambda v: d_inv * v)  # noqa: E731
    z = Minv(r)
    p = z.copy()
    rz_old = float(r @ z)
    for k in range(1, maxiter + 1):
        Ap = A @ p
        pAp = float(p @ Ap)
        if pAp <= 0.0:
            raise np.linalg.LinAlgError(f"preconditioned_cg: p^T A p = {pAp:.3e} <= 0 at iteration {k}")
        alpha = rz_old / pAp
        x = x + alpha * p
        r = r - alpha * Ap
        rel = np.linalg.norm(r) / bnorm
        if history is not None:
            history.append((time.perf_counter(), rel))
        if rel < tol:
            return x, k, rel
        z = Minv(r)
        rz_new = float(r @ z)
        beta = rz_new / rz_old
        p = z + beta * p
        rz_old = rz_new
    raise RuntimeError(f"preconditioned_cg: did not converge in {maxiter} iterations (rel {rel:.3e})")


# ----------------------------------------------------------------------------- SIMP
def simp_scale(rho, p=3.0, rho_min=1e-3):
    """s = rho_min + (1 - rho_min) rho^p (fea_engine/src/fea_engine/topopt.py:74-82)."""
    rho = np.asarray(rho, dtype=float)
    return rho_min + (1.0 - rho_min) * rho ** p


def simp_scale_grad(rho, p=3.0, rho_min=1e-3):
    """ds/drho = p (1 - rho_min) rho^(p-1) (topopt.py:85-93)."""
    rho = np.asarray(rho, dtype=float)
    return p * (1.0 - rho_min) * rho ** (p - 1.0)


def compliance_sensitivity_closed_form(ke_unit, conn, u_full, rho, p, rho_min, dofs_per_node=3):
    """dC/drho_e = -s'(rho_e) u_e^T ke_unit_e u_e (topopt.py:161-177)."""
    g = global_dofs(conn, dofs_per_node)
    u_e = np.asarray(u_full)[g]
    quad = np.einsum("ei,eij,ej->e", u_e, ke_unit, u_e)
    return -simp_scale_grad(rho, p, rho_min) * quad


# ----------------------------------------------------------------------------- SIMP OC loop
def build_filter_weights(centroids, radius):
    """Dense H[e, j] = max(0, radius - |c_e - c_j|) (topopt.py:235-243)."""
    c = np.asarray(centroids, dtype=float)
    d = np.sqrt(np.sum((c[:, None, :] - c[None, :, :]) ** 2, axis=-1))
    return np.maximum(0.0, radius - d)


def apply_sensitivity_filter(H, rho, dc, eps=1e-9):
    """H (rho dc) / max(max(rho, eps) H 1, eps) (topopt.py:246-253)."""
    rho, dc = np.asarray(rho, dtype=float), np.asarray(dc, dtype=float)
    return (H @ (rho * dc)) / np.maximum(np.maximum(rho, eps) * H.sum(axis=1), eps)


def oc_update(rho, dc, volume_fraction, move=0.2, rho_min_bound=1e-3, rho_max_bound=1.0, bisection_tol=1e-4,
              max_bisection_iter=100):
    """Optimality-criteria update with an expanding bracket, then bisection, on the volume
    multiplier (topopt.py:259-295)."""
    rho = np.asarray(rho, dtype=float)
    dc = np.minimum(np.asarray(dc, dtype=float), -1e-12)

    def trial(lam):
        t = np.clip(rho * np.sqrt(-dc / lam), rho - move, rho + move)
        return np.clip(t, rho_min_bound, rho_max_bound)

    lo, hi = 1e-12, 1.0
    for _ in range(60):
        if trial(hi).mean() <= volume_fraction:
            break
        hi *= 2.0
    new = None
    for _ in range(max_bisection_iter):
        mid = 0.5 * (lo + hi)
        new = trial(mid)
        if new.mean() > volume_fraction:
            lo = mid
        else:
            hi = mid
        if hi - lo < bisection_tol * max(hi, 1.0):
            break
    return new


def topology_optimize_compliance(nodes, conn, D, fixed, F_ext, volume_fraction, p=3.0, rho_min=1e-3, move=0.2,
                                 n_iter=50, filter_radius=None, tol=1e-3):
    """SIMP loop with the closed-form sensitivity (topopt.py:298-379); K(rho) u = F by a sparse
    direct solve.  Returns (rho, compliance history, u)."""
    nodes, conn = np.asarray(nodes, dtype=float), np.asarray(conn)
    n_dof = 3 * len(nodes)
    free = free_dofs(n_dof, fixed)
    ke = hex8_element_stiffness(nodes[conn], D)
    F_ext = np.asarray(F_ext, dtype=float)
    rho = np.full(len(conn), float(volume_fraction))
    H = None
    if filter_radius is not None and filter_radius > 0:
        H = build_filter_weights(nodes[conn].mean(axis=1), filter_radius)
    hist, u = [], None
    for _ in range(n_iter):
        s = simp_scale(rho, p, rho_min)
        Kff = reduce_free(structural_csr(ke * s[:, None, None], conn, n_dof), free).tocsc()
        u = np.zeros(n_dof)
        u[free] = spla.spsolve(Kff, F_ext[free])
        hist.append(float(F_ext @ u))
        dc = compliance_sensitivity_closed_form(ke, conn, u, rho, p, rho_min)
        if H is not None:
            dc = apply_sensitivity_filter(H, rho, dc)
        new = oc_update(rho, dc, volume_fraction, move=move, rho_min_bound=rho_min)
        change = float(np.max(np.abs(new - rho)))
        rho = new
        if change < tol:
            break
    return rho, hist, u


# ----------------------------------------------------------------------------- recovery
def recover(nodes, conn, U, D=None):
    """Strain (D is None) or stress (D given) of hex8 elements, as recovery._recover for one
    Hex8 block (fea_engine/src/fea_engine/recovery.py:196-227 and :258-334): at each Gauss point
    val = [D] B u_e; numE[e, a] += |detJ| w N_a val, denE[e, a] += |detJ| w N_a; nodal =
    sum over elements (np.add.at over the connectivity) of numE / denE (0 where denE is 0);
    elem = sum_q |detJ| w val / sum_q |detJ| w.  Returns (nodal (N, 6), elem (E, 6))."""
    nodes = np.asarray(nodes, dtype=float)
    conn = np.asarray(conn)
    U = np.asarray(U, dtype=float)
    X = nodes[conn]
    ue = U[global_dofs(conn)]
    E = len(conn)
    numE, denE = np.zeros((E, 8, 6)), np.zeros((E, 8))
    acc, vol = np.zeros((E, 6)), np.zeros(E)
    pts, _ = _gauss_product_3d(2)
    for (w, detJ, dN_g), p in zip(_gauss_geometry(X), pts):
        N, _ = hex8_shape_and_derivs(*p)
        val = np.einsum("esm,em->es", _b_matrices(dN_g), ue)
        if D is not None:
            val = np.einsum("st,et->es", np.asarray(D, dtype=float), val)
        wt = np.abs(detJ) * w
        numE += np.einsum("e,c,es->ecs", wt, N, val)
        denE += np.einsum("e,c->ec", wt, N)
        acc += wt[:, None] * val
        vol += wt
    num, den = np.zeros((len(nodes), 6)), np.zeros(len(nodes))
    np.add.at(num, conn, numE)
    np.add.at(den, conn, denE)
    nodal = np.divide(num, den[:, None], out=np.zeros_like(num), where=den[:, None] > 0)
    return nodal, acc / vol[:, None]


def von_mises(s):
    """3-D von Mises stress of Voigt rows [xx, yy, zz, xy, yz, xz] (recovery.py:386-394)."""
    s = np.asarray(s, dtype=float)
    sxx, syy, szz, sxy, syz, sxz = (s[..., j] for j in range(6))
    return np.sqrt(0.5 * ((sxx - syy) ** 2 + (syy - szz) ** 2 + (szz - sxx) ** 2)
                   + 3.0 * (sxy ** 2 + syz ** 2 + sxz ** 2))


def reactions(K, U, F, fixed):
    """R = K U - F at the constrained DOFs, zero elsewhere (recovery.py:422-440)."""
    r = np.asarray(K @ np.asarray(U, dtype=float)).ravel() - np.asarray(F, dtype=float).ravel()
    out = np.zeros_like(r)
    out[np.asarray(fixed)] = r[np.asarray(fixed)]
    return out


# ----------------------------------------------------------------------------- POD
def pod_singular_values(X):
    """Singular values of the snapshot matrix by economy SVD
    (PodBasis._fit_standard, rom_engine/src/rom_engine/pod.py:140-147)."""
    return np.linalg.svd(np.asarray(X, dtype=float), full_matrices=False, compute_uv=False)
