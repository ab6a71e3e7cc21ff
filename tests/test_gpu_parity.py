"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's golden vectors.

Bars: CSR row_ptr/col_idx bit-exact; K values within 1e-12 (normwise, max|dK|/max|K|);
displacements within 1e-8 relative (2-norm) of the FP64 reference solution; SIMP sensitivities
within 1e-10 of the closed form evaluated on the same u.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle as O

pytestmark = pytest.mark.gpu

KTOL = 1e-12      # K values, normwise relative
UTOL = 1e-8       # displacements, relative 2-norm


def _feab():
    import feab200
    return feab200


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _device_mesh(nodes, elements):
    from feab200.device import DeviceMesh
    return DeviceMesh(nodes, elements)


def _reduced(nodes, elements, D, fixed, want32=True):
    dm = _device_mesh(nodes, elements)
    pat = dm.pattern(fixed)
    ke = dm.element_stiffness(D)
    return dm, dm.assemble(ke, pat, want32=want32)


# ----------------------------------------------------------------------------- pattern + values
def test_csr_pattern_bit_exact_and_values_20x4x4(golden):
    g = golden("cantilever_20x4x4")
    dm, op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    p = op.pattern
    assert p.nnz == g["col_idx"].size
    assert np.array_equal(p.row_ptr.cpu().numpy(), g["row_ptr"])
    assert np.array_equal(p.col_idx.cpu().numpy(), g["col_idx"])
    v = op.vals64.cpu().numpy()
    assert np.abs(v - g["vals"]).max() / np.abs(g["vals"]).max() < KTOL
    # FP32 copy and Jacobi diagonals
    assert np.array_equal(op.vals32.cpu().numpy(), g["vals"].astype(np.float32))
    Kff = sp.csr_matrix((g["vals"], g["col_idx"], g["row_ptr"]))
    dinv = 1.0 / Kff.diagonal()
    assert np.abs(op.dinv64.cpu().numpy() - dinv).max() / np.abs(dinv).max() < KTOL


def test_csr_pattern_full_and_partially_fixed(golden):
    g = golden("pattern_4x3x2")
    dm = _device_mesh(g["nodes"], g["elements"])
    ke = dm.element_stiffness(g["D"])
    for fixed, rp, ci, vals in ((np.array([], dtype=int), g["K_row_ptr"], g["K_col_idx"], g["K_vals"]),
                                (g["fixed"], g["Kff_row_ptr"], g["Kff_col_idx"], g["Kff_vals"])):
        op = dm.assemble(ke, dm.pattern(fixed))
        assert np.array_equal(op.pattern.row_ptr.cpu().numpy(), rp)
        assert np.array_equal(op.pattern.col_idx.cpu().numpy(), ci)
        assert np.abs(op.vals64.cpu().numpy() - vals).max() / np.abs(vals).max() < KTOL


@pytest.mark.parametrize("shape", [(9, 5, 3), (16, 6, 6)])
def test_pattern_and_values_vs_oracle_jittered(shape):
    feab = _feab()
    c = feab.cantilever.plain_cantilever(*shape, seed=11)
    X, el = c.mesh.nodes, c.mesh.elements
    fixed = np.union1d(c.fixed, 3 * c.mesh.nodes_on_plane(1, 0.0) + 1)   # add a partial (uy) support
    dm, op = _reduced(X, el, c.D, fixed)
    K = O.structural_csr(O.hex8_element_stiffness(X[el], c.D), el, 3 * len(X))
    Kff = O.reduce_free(K, O.free_dofs(3 * len(X), fixed))
    assert np.array_equal(op.pattern.row_ptr.cpu().numpy(), Kff.indptr)
    assert np.array_equal(op.pattern.col_idx.cpu().numpy(), Kff.indices)
    assert np.abs(op.vals64.cpu().numpy() - Kff.data).max() / np.abs(Kff.data).max() < KTOL


def test_element_stiffness_vs_reference(golden):
    g = golden("ke_distorted")
    from feab200 import _lib as L
    el = np.arange(48).reshape(6, 8)
    dm = _device_mesh(g["coords"].reshape(-1, 3), el)
    for D, ref in ((g["D"], g["ke"]), (g["D_aniso"], g["ke_aniso"])):
        ke = dm.element_stiffness(D, layout=L.KE_FULL).cpu().numpy()
        assert np.abs(ke - ref).max() / np.abs(ref).max() < 1e-13
        assert np.array_equal(ke, np.transpose(ke, (0, 2, 1)))        # exactly symmetric


def test_assembly_is_deterministic(golden):
    g = golden("cantilever_20x4x4")
    _, a = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    _, b = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    assert torch.equal(a.vals64, b.vals64) and torch.equal(a.dinv64, b.dinv64)


def test_element_by_element_apply_matches_csr(golden):
    g = golden("pattern_4x3x2")
    dm = _device_mesh(g["nodes"], g["elements"])
    ke = dm.element_stiffness(g["D"])
    K = sp.csr_matrix((g["K_vals"], g["K_col_idx"], g["K_row_ptr"]))
    v = np.random.default_rng(0).standard_normal(K.shape[0])
    y = dm.apply(ke, v).cpu().numpy()
    assert np.abs(y - K @ v).max() / np.abs(K @ v).max() < 1e-13


# ----------------------------------------------------------------------------- PCG
def test_pcg_fp64_reproduces_reference_solve(golden):
    g = golden("cantilever_20x4x4")
    from feab200.device import pcg_solve
    _, op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    x, info = pcg_solve(op, g["Ff"], tol=1e-10, precision="fp64")
    assert info.status == 0
    assert abs(info.iters - int(g["pcg_iters"])) <= 2
    assert _rel(x.cpu().numpy(), g["uf_pcg"]) < 1e-11
    assert _rel(x.cpu().numpy(), g["U_lu"][g["free"]]) < UTOL


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_pcg_reduced_precision_reaches_fp64_accuracy(golden, precision):
    g = golden("cantilever_20x4x4")
    from feab200.device import pcg_solve
    _, op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    x, info = pcg_solve(op, g["Ff"], tol=1e-10, precision=precision)
    assert info.status == 0 and info.reliable_updates >= 1
    assert info.relres < 1e-10                               # the FP64 residual, not the recurrence one
    assert _rel(x.cpu().numpy(), g["U_lu"][g["free"]]) < UTOL
    if precision == "mixed":
        # 36-bit values in difference form keep the FP64 recurrence's iteration count
        assert info.iters <= int(g["pcg_iters"]) + 5


def test_difference_form_spmv_matches_fp64(golden):
    g = golden("cantilever_20x4x4")
    from feab200.device import spmv
    _, op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    Kff = sp.csr_matrix((g["vals"], g["col_idx"], g["row_ptr"]))
    rng = np.random.default_rng(4)
    absK = abs(Kff)
    for x in (rng.standard_normal(op.n), g["U_lu"][g["free"]]):
        ref = Kff @ x
        scale = np.linalg.norm(absK @ np.abs(x))           # size of the terms that cancel in K x
        y64 = spmv(op, x, "fp64").cpu().numpy()
        ymx = spmv(op, x, "mixed").cpu().numpy()
        y32 = spmv(op, x.astype(np.float32), "fp32").cpu().numpy()
        assert np.linalg.norm(y64 - ref) / scale < 1e-14
        assert np.linalg.norm(ymx - ref) / scale < 1e-10
        assert np.linalg.norm(y32 - ref) / scale < 1e-5


def test_pcg_is_deterministic(golden):
    g = golden("cantilever_20x4x4")
    from feab200.device import pcg_solve
    _, op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    for prec in ("fp64", "mixed", "fp32"):
        a, ia = pcg_solve(op, g["Ff"], tol=1e-10, precision=prec)
        b, ib = pcg_solve(op, g["Ff"], tol=1e-10, precision=prec)
        assert torch.equal(a, b) and ia.iters == ib.iters


def test_pcg_on_host_csr_and_plain_cg(golden):
    """preconditioned_cg(A, b, M) with a host SciPy matrix, like the reference call."""
    g = golden("cantilever_20x4x4")
    feab = _feab()
    Kff = sp.csr_matrix((g["vals"], g["col_idx"], g["row_ptr"]))
    x, it = feab.preconditioned_cg(Kff, g["Ff"], M=feab.jacobi_preconditioner(Kff), tol=1e-10)
    assert abs(it - int(g["pcg_iters"])) <= 2 and _rel(x, g["uf_pcg"]) < 1e-11
    ref, ref_it, _ = O.preconditioned_cg(Kff, g["Ff"], None, tol=1e-9)
    x2, it2 = feab.preconditioned_cg(Kff, g["Ff"], M=None, tol=1e-9)
    assert abs(it2 - ref_it) <= max(3, ref_it // 100) and _rel(x2, ref) < 1e-7


def test_fesystem_drop_in_flow(golden):
    """The reference's own call sequence, with feab200 names."""
    g = golden("cantilever_20x4x4")
    feab = _feab()
    mesh = feab.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab.FESystem(mesh, feab.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(feab.D_solid3d(feab.Material(E=210e9, nu=0.3)), vectorized=True)
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    fs.add_consistent_facet_load(feab.Hex8Solid3D(), [tuple(f) for f in g["facets"]], 2, -1.0e6)
    U = fs.solve_static(method="pcg", tol=1e-10)
    assert isinstance(U, feab.FEField) and U.shape == (fs.n_dof,)
    assert _rel(U, g["U_pcg"]) < 1e-11
    Um = fs.solve_static(method="pcg", tol=1e-10, precision="mixed")
    assert _rel(Um, g["U_lu"]) < UTOL
    Ud = fs.solve_static()             # the reference's direct solve: banded Cholesky here
    assert _rel(Ud, g["U_lu"]) < 1e-10
    rs = fs.form_linear_system()
    assert np.array_equal(rs.K.indptr, g["row_ptr"]) and np.array_equal(rs.K.indices, g["col_idx"])
    assert np.abs(rs.F - g["Ff"]).max() <= 1e-12 * np.abs(g["Ff"]).max()
    assert fs.K.nnz == int(g["nnz_full"])


def test_patch_test_with_prescribed_displacements():
    """Affine displacement prescribed on the boundary of a distorted mesh is reproduced inside
    (the hex8 patch test of the reference's test_benchmarks_convergence.py:155-175)."""
    feab = _feab()
    m = feab.box_mesh(1.0, 1.0, 1.0, 4, 4, 4)
    from feab200.mesh import jitter_interior
    m = jitter_interior(m, 0.4, 3, h=(0.25, 0.25, 0.25))
    X = m.nodes
    Gm = np.array([[1e-3, 2e-4, -3e-4], [5e-4, -1e-3, 1e-4], [2e-4, 3e-4, 2e-3]])
    b = np.array([1e-4, -2e-4, 3e-4])
    exact = X @ Gm.T + b
    fs = feab.FESystem(m, feab.Hex8Solid3D())
    fs.assemble_stiffness(feab.D_solid3d(feab.Material(E=200e9, nu=0.3)))
    lo, hi = X.min(0), X.max(0)
    bnd = np.where(np.any((np.abs(X - lo) < 1e-9) | (np.abs(X - hi) < 1e-9), axis=1))[0]
    for n in bnd:
        for d in range(3):
            fs.fix_dofs([int(n)], [d], value=float(exact[n, d]))
    U = fs.solve_static(method="pcg", tol=1e-14, maxiter=20000)
    err = np.abs(np.asarray(U).reshape(-1, 3) - exact).max() / np.abs(exact).max()
    assert err < 1e-10


# ----------------------------------------------------------------------------- errors
def test_error_paths_raise_reference_exceptions(golden):
    g = golden("cantilever_20x4x4")
    feab = _feab()
    Kff = sp.csr_matrix((g["vals"], g["col_idx"], g["row_ptr"]))
    with pytest.raises(np.linalg.LinAlgError):
        feab.preconditioned_cg(-Kff, g["Ff"], M=None, tol=1e-10)
    with pytest.raises(RuntimeError):
        feab.preconditioned_cg(Kff, g["Ff"], M=feab.jacobi_preconditioner(Kff), tol=1e-10, maxiter=3)
    with pytest.raises(ValueError):
        feab.jacobi_preconditioner(sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 2.0]])))
    # a collapsed element (all nodes in one plane): near-zero det J
    nodes = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]] * 2, dtype=float)
    with pytest.raises(ValueError, match="degenerate"):
        _device_mesh(nodes, np.arange(8)[None, :]).element_stiffness(np.eye(6))
    # a repeated node id in one element
    nodes = np.random.default_rng(0).random((8, 3))
    with pytest.raises(ValueError):
        _device_mesh(nodes, np.array([[0, 1, 2, 3, 4, 5, 6, 6]])).topology()


# ----------------------------------------------------------------------------- SIMP adjoint
def test_simp_closed_form_and_autograd(golden):
    g = golden("simp_6x3x3")
    feab = _feab()
    from feab200 import topopt
    mesh = feab.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab.FESystem(mesh, feab.Hex8Solid3D())
    ke_unit, conn = topopt.unit_stiffness_stack(fs, g["D"])
    p, rmin = float(g["p"]), float(g["rho_min"])
    # kernel on the reference's own u
    dc = topopt.compliance_sensitivity_closed_form(ke_unit, conn, 3, g["u"], g["rho"], p, rmin)
    assert np.abs(dc - g["dc"]).max() / np.abs(g["dc"]).max() < 1e-10
    # GPU forward solve
    u, Kff, Ff = topopt.solve_simp_equilibrium(ke_unit, conn, 3, fs.n_dof, g["free"], g["F"], g["rho"], p, rmin)
    assert _rel(u, g["u"]) < UTOL
    dc_adj = topopt.compliance_sensitivity_via_adjoint(ke_unit, conn, 3, fs.n_dof, g["free"], u, Kff, Ff,
                                                       g["rho"], p, rmin)
    assert np.abs(dc_adj - g["dc_adjoint"]).max() / np.abs(g["dc_adjoint"]).max() < 1e-7
    # autograd Function: C = f.u ; dC/drho and the finite differences of the reference
    prob = topopt.SimpProblem(fs.device_mesh, g["D"], g["free"], penal=p, rho_min=rmin)
    dev = fs.device
    f = torch.as_tensor(g["F"][g["free"]], device=dev)
    for recompute in (False, True):
        rho = torch.as_tensor(g["rho"], device=dev).requires_grad_(True)
        uf = prob(rho, f, recompute=recompute)
        C = torch.dot(f, uf)
        C.backward()
        gr = rho.grad.cpu().numpy()
        assert np.abs(gr - g["dc"]).max() / np.abs(g["dc"]).max() < 1e-7
        assert np.allclose(gr[g["fd_elems"]], g["dc_fd"], rtol=1e-5)


def test_simp_vjp_against_torch_autograd_reference():
    """VJP of u(rho) with a random cotangent against plain torch autograd through a dense
    solve (small mesh, FP64)."""
    feab = _feab()
    from feab200 import topopt
    c = feab.cantilever.simp_cantilever(4, 2, 2, seed=1)
    fs = feab.FESystem(c.mesh, feab.Hex8Solid3D())
    prob = topopt.SimpProblem(fs.device_mesh, c.D, c.free, penal=3.0, rho_min=1e-9)
    dev = fs.device
    rho0 = torch.as_tensor(c.meta["rho"], device=dev)
    f = torch.as_tensor(c.F[c.free], device=dev)
    w = torch.as_tensor(np.random.default_rng(2).standard_normal(len(c.free)), device=dev)
    rho = rho0.clone().requires_grad_(True)
    (prob(rho, f) * w).sum().backward()
    # torch reference: K(rho) dense from the unit element matrices
    ke = topopt.unit_stiffness_stack(fs, c.D)[0].ke.to(dev)
    gidx = torch.as_tensor(O.global_dofs(c.mesh.elements), device=dev)
    free = torch.as_tensor(c.free, device=dev)
    rho_t = rho0.clone().requires_grad_(True)
    s = 1e-9 + (1 - 1e-9) * rho_t ** 3
    Kd = torch.zeros(fs.n_dof, fs.n_dof, dtype=torch.float64, device=dev)
    Kd = Kd.index_put((gidx[:, :, None].expand(-1, -1, 24).reshape(-1), gidx[:, None, :].expand(-1, 24, -1).reshape(-1)),
                      (s[:, None, None] * ke).reshape(-1), accumulate=True)
    u_ref = torch.linalg.solve(Kd[free][:, free], f)
    (u_ref * w).sum().backward()
    a, b = rho.grad.cpu().numpy(), rho_t.grad.cpu().numpy()
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-8


# ----------------------------------------------------------------------------- mid-size vs oracle
@pytest.mark.slow
def test_random_tip_mid_size_vs_oracle():
    feab = _feab()
    c = feab.cantilever.random_tip_cantilever(32, 8, 8, seed=7)
    X, el = c.mesh.nodes, c.mesh.elements
    K = O.structural_csr(O.hex8_element_stiffness(X[el], c.D), el, 3 * len(X))
    free = O.free_dofs(3 * len(X), c.fixed)
    Kff = O.reduce_free(K, free)
    u_ref, _, _ = O.preconditioned_cg(Kff, c.F[free], O.jacobi_inverse_diagonal(Kff), tol=1e-13)
    from feab200.device import pcg_solve
    dm, op = _reduced(X, el, c.D, c.fixed)
    assert np.array_equal(op.pattern.col_idx.cpu().numpy(), Kff.indices)
    for prec in ("fp64", "mixed", "fp32"):
        x, info = pcg_solve(op, c.F[free], tol=1e-9, precision=prec)
        assert info.status == 0
        assert _rel(x.cpu().numpy(), u_ref) < UTOL, (prec, info)
