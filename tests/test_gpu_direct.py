"""The direct solve of solve_static(method=None): banded Cholesky on the GPU.

The reference's default sparse solve is SuperLU (FESystem._sparse_lu_solve,
fea_engine/src/fea_engine/solver.py:1681-1724).  The golden fixture's U_lu is the reference's own
direct solution; SciPy's spsolve on the oracle's K_ff is the independent check on other meshes.
Bars: 1e-10 relative (2-norm) against a direct solve of the same K_ff.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import oracle as O

pytestmark = pytest.mark.gpu

DTOL = 1e-10


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _op(nodes, elements, D, fixed):
    from feab200.device import DeviceMesh
    dm = DeviceMesh(nodes, elements)
    return dm.assemble(dm.element_stiffness(D), dm.pattern(fixed), want32=False)


def test_solve_static_default_is_the_direct_solve(golden):
    """The reference's call sequence with method=None against its own SuperLU solution."""
    import feab200 as feab
    g = golden("cantilever_20x4x4")
    mesh = feab.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab.FESystem(mesh, feab.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(g["D"])
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    fs.add_consistent_facet_load(feab.Hex8Solid3D(), [tuple(f) for f in g["facets"]], 2, -1.0e6)
    U = fs.solve_static()
    assert fs.last_solve_info.precision == "direct" and fs.last_solve_info.iters == 0
    assert _rel(U, g["U_lu"]) < DTOL
    assert fs.last_solve_info.relres < 1e-11     # SuperLU's own: 3.0e-12 on this system
    fac = fs.reduced_operator(want32=False).direct_factor()
    assert fac.bandwidth > 0 and not fac.near_singular
    # the factor is reused: a second load case through the same operator
    U2 = fs.solve_static()
    assert _rel(U2, U) == 0.0


@pytest.mark.parametrize("shape,dofs", [((24, 8, 8), (0, 1, 2)), ((9, 5, 3), (0,)), ((7, 3, 2), (1, 2))])
def test_band_cholesky_matches_scipy_direct_solve(shape, dofs):
    """Ragged sizes (n not a multiple of 64), partially fixed nodes (only some components of the
    x = 0 face fixed, plus three pinned face nodes so K_ff stays SPD) and two right-hand sides."""
    from feab200.direct import BandCholesky
    nx, ny, nz = shape
    X, el = O.box_mesh(2.0, 0.4, 0.4, nx, ny, nz)
    face = np.flatnonzero(np.isclose(X[:, 0], 0.0))
    fixed = (3 * face[:, None] + np.asarray(dofs)[None, :]).reshape(-1)
    pins = face[[0, len(face) // 2, len(face) - 1]]           # all components of three face nodes
    fixed = np.unique(np.concatenate([fixed, (3 * pins[:, None] + np.arange(3)[None, :]).reshape(-1)]))
    D = O.D_solid3d(210e9, 0.3)
    free = O.free_dofs(3 * len(X), fixed)
    ke = O.hex8_element_stiffness(X[el], D)
    Kff = O.reduce_free(O.structural_csr(ke, el, 3 * len(X)), free).tocsc()
    op = _op(X, el, D, fixed)
    assert op.n == Kff.shape[0]
    fac = BandCholesky(op)
    assert not fac.near_singular
    rng = np.random.default_rng(3)
    for _ in range(2):
        b = rng.standard_normal(op.n)
        x = fac.solve(b).cpu().numpy()
        assert _rel(x, spla.spsolve(Kff, b)) < DTOL


def test_band_cholesky_rejects_a_matrix_that_is_not_spd():
    from feab200.direct import BandCholesky
    X, el = O.box_mesh(1.0, 0.5, 0.5, 4, 2, 2)
    op = _op(X, el, O.D_solid3d(1.0, 0.3), O.fixed_dofs_on_plane(X, 0, 0.0))
    op.vals64.neg_()
    with pytest.raises(np.linalg.LinAlgError):
        BandCholesky(op)


@pytest.mark.parametrize("pinned", [False, True])
def test_singular_system_gives_the_minimum_norm_solution(pinned):
    """K_ff singular: a floating body (six rigid-body modes) or one pinned node (three rotations
    left).  The reference detects it on its LU pivots and solves by eigenvalues for the
    minimum-norm least-squares answer (_eigen_solve, solver.py:1584-1679); feab200 detects it on
    its Cholesky pivots, warns, and must return the same pinv(K_ff) F -- here for a load with a
    net force and moment, so the system is also inconsistent."""
    import feab200 as feab
    X, el = O.box_mesh(1.0, 0.5, 0.5, 4, 2, 2)
    D = O.D_solid3d(1.0, 0.3)
    mesh = feab.Mesh(nodes=X, elements=el)
    fs = feab.FESystem(mesh, feab.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(D)
    if pinned:
        fs.fix_dofs([7], [0, 1, 2])
    F = np.random.default_rng(0).standard_normal(fs.n_dof)
    fs.F[:] = F
    with pytest.warns(UserWarning, match="singular"):
        U = np.asarray(fs.solve_static(tol=1e-13, maxiter=20000))
    free = fs.free_dofs
    K = O.structural_csr(O.hex8_element_stiffness(X[el], D), el, 3 * len(X)).toarray()[np.ix_(free, free)]
    assert _rel(U[free], np.linalg.pinv(K, rcond=1e-10) @ F[free]) < 1e-7


def test_band_entry_points_check_their_arguments():
    from feab200 import _lib as L
    X, el = O.box_mesh(1.0, 0.5, 0.5, 4, 2, 2)
    op = _op(X, el, O.D_solid3d(1.0, 0.3), O.fixed_dofs_on_plane(X, 0, 0.0))
    dev = op.vals64.device
    csr = op.csr_struct()
    bad = torch.arange(op.n, dtype=torch.int32, device=dev)
    bad[3] = op.n + 7                                        # not a row number
    scratch = torch.zeros(2, dtype=torch.int32, device=dev)
    bw = C.c_int32(0)
    rc = L.lib.feab_band_width(C.byref(csr), L.dptr(bad), L.dptr(scratch), C.byref(bw), L.stream_ptr(dev))
    assert rc == L.FEAB_BAD_ARG
    # an assembly with a band narrower than the matrix's reports the entries it cannot hold
    ident = torch.arange(op.n, dtype=torch.int32, device=dev)
    rc = L.lib.feab_band_width(C.byref(csr), L.dptr(ident), L.dptr(scratch), C.byref(bw), L.stream_ptr(dev))
    assert rc == L.FEAB_OK and bw.value > 0
    storage = torch.empty(int(L.lib.feab_band_bytes(op.n, 0)), dtype=torch.uint8, device=dev)
    band = L.Band(0, 0, 0, 0, storage.data_ptr())
    rc = L.lib.feab_band_assemble(C.byref(csr), L.dptr(ident), 0, C.byref(band), L.stream_ptr(dev))
    assert rc == L.FEAB_BAD_ARG


def test_torch_backend_dense_method_is_the_direct_solve(golden):
    """fesystem_solve_static_torch(method="dense") (torch_sparse_solver.py:268-314, a dense LU in
    the reference) runs the banded Cholesky: the reference's SuperLU solution to 1e-10, and the
    same answer as the CG method to its tolerance."""
    import feab200 as feab
    from feab200.torch_sparse_solver import fesystem_solve_static_torch
    g = golden("cantilever_20x4x4")
    mesh = feab.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab.FESystem(mesh, feab.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(g["D"])
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    fs.add_consistent_facet_load(feab.Hex8Solid3D(), [tuple(f) for f in g["facets"]], 2, -1.0e6)
    Ud = fesystem_solve_static_torch(fs, method="dense")
    assert _rel(Ud, g["U_lu"]) < DTOL
    Uc = fesystem_solve_static_torch(fs, method="cg", tol=1e-10)
    assert _rel(Uc, Ud) < 1e-8
