"""Generate the golden fixtures in this folder by running the REFERENCE implementation.

Run from the repository root, in a checkout where the reference is available:

    python tests/golden/make_golden.py --reference <reference checkout>

It imports abhi2k16/computation-suite's ``fea_engine`` and ``rom_engine`` from
``<reference>/fea_engine/src`` and ``<reference>/rom_engine/src`` and calls the
reference's own public functions on small seeded inputs, then writes
``*.npz`` files next to this script.  The tests only read the ``.npz`` files, so
the reference is not needed where the tests run.

Fixtures
--------
cantilever_20x4x4.npz  config "plain method, CPU-runnable": 20x4x4 hex8 cantilever over
                       2.0x0.4x0.4 m, interior nodes jittered by +-5 % of the element size
                       (seed 1234), x=0 clamped, uniform -1e6 Pa z traction on x=L through
                       FESystem.add_consistent_facet_load.  Holds the mesh, the reduced CSR
                       (FESystem(sparse=True) vectorized assembly), Ff, the SuperLU solution
                       and the reference PCG (rtol 1e-10) solution with its iteration count.
pattern_4x3x2.npz      undistorted 4x3x2 box: the structural CSR pattern of K and Kff
                       (scatter_global_stiffness COO->CSR) and the FESystem LIL pattern
                       (which drops exact-zero cancellations).
ke_distorted.npz       element stiffness of 6 distorted hexes from Hex8Solid3D.stiffness.
facets.npz             consistent facet load shares / facet mass of 5 distorted quad faces.
simp_6x3x3.npz         SIMP compliance: densities, forward solution, closed-form dc, the
                       torch-adjoint dc and central finite differences at 4 elements.
pod_small.npz          singular values of a 400x12 snapshot matrix from PodBasis.fit.
recovery_20x4x4.npz    the cantilever_20x4x4 system at its SuperLU displacement: FESystem.stress /
                       strain / von_mises at the nodes and per element, and reactions.
modal_20x4x4.npz       Hex8Solid3D.mass of distorted hexes, and the cantilever_20x4x4 system's
                       assemble_mass(7850 I) + solve_modal(n_modes=6).  The frequencies reproduce
                       run to run; the mode vectors' signs and their rotation inside the two
                       near-degenerate bending pairs follow ARPACK's random start vector, so the
                       tests compare the spanned subspace, not the vectors.
bbar_hex8.npz          Hex8SolidBbar element stiffness of distorted hexes (nu 0.3, 0.4999) and the
                       near-incompressible cantilever deflection with Hex8SolidBbar and Hex8Solid3D.
topopt_8x4x4.npz       SIMP on an 8x4x4 cantilever: build_filter_weights, apply_sensitivity_filter,
                       oc_update on seeded inputs, and 12 iterations of
                       topology_optimize_compliance (final densities, compliance history, u).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference(root):
    sys.path.insert(0, os.path.join(root, "fea_engine", "src"))
    sys.path.insert(0, os.path.join(root, "rom_engine", "src"))
    import fea_engine  # noqa: F401
    import rom_engine  # noqa: F401


def jitter(nodes, h, amp, seed):
    rng = np.random.default_rng(seed)
    X = nodes.copy()
    lo, hi = X.min(0), X.max(0)
    inner = np.all((X > lo + 1e-9) & (X < hi - 1e-9), axis=1)
    X[inner] += amp * np.asarray(h) * (rng.random((int(inner.sum()), 3)) - 0.5)
    return X


def _cantilever_20x4x4_system():
    """The jittered 20x4x4 FESystem, clamped and loaded: (fs, mesh, D, facets)."""
    from fea_engine.mesh import box_mesh, Mesh
    from fea_engine.elements.solids import Hex8Solid3D
    from fea_engine.material import Material, D_solid3d
    from fea_engine.solver import FESystem
    from fea_engine import facet_loads

    Lx, Ly, Lz, nx, ny, nz = 2.0, 0.4, 0.4, 20, 4, 4
    base = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    nodes = jitter(base.nodes, (Lx / nx, Ly / ny, Lz / nz), 0.1, 1234)
    mesh = Mesh(nodes=nodes, elements=base.elements, dim=3)
    elem = Hex8Solid3D()
    D = D_solid3d(Material(E=210e9, nu=0.3))
    fs = FESystem(mesh, elem, sparse=True)
    fs.assemble_stiffness(D, vectorized=True)
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    tip = set(mesh.nodes_on_plane(0, Lx).tolist())
    facets = []
    for conn in mesh.elements:
        for idx, _, _ in facet_loads.list_facets(elem):
            f = tuple(int(conn[i]) for i in idx)
            if all(n in tip for n in f):
                facets.append(f)
    fs.add_consistent_facet_load(elem, facets, 2, -1.0e6)
    return fs, mesh, D, facets


def cantilever_20x4x4():
    from fea_engine.elements.solids import Hex8Solid3D
    from fea_engine import iterative_solvers
    from fea_engine.vectorized_assembly import scatter_global_stiffness, tensorized_element_stiffness
    from fea_engine.mesh_transform import MeshTransformation

    fs, mesh, D, facets = _cantilever_20x4x4_system()
    nodes, elem = mesh.nodes, Hex8Solid3D()
    rs = fs.form_linear_system()
    Kff = rs.K.tocsr()
    U_lu = np.asarray(fs.solve_static())
    M = iterative_solvers.jacobi_preconditioner(Kff)
    uf_pcg, n_iter = iterative_solvers.preconditioned_cg(Kff, rs.F, M=M, tol=1e-10)
    U_pcg = np.asarray(fs.solve_static(method="pcg", tol=1e-10))
    # the structural pattern (COO->CSR, exact zeros kept) must agree on this jittered mesh
    ke = tensorized_element_stiffness(MeshTransformation(mesh, elem), D)
    Ks = scatter_global_stiffness(ke, mesh.elements, 3, fs.n_dof, sparse=True).tocsr()
    Ks_ff = Ks[np.ix_(rs.free, rs.free)]
    assert np.array_equal(Ks_ff.indptr, Kff.indptr) and np.array_equal(Ks_ff.indices, Kff.indices)
    return dict(nodes=nodes, elements=np.asarray(mesh.elements, dtype=np.int64), D=D,
                fixed=rs.fixed, free=rs.free, F=np.asarray(fs.F), Ff=np.asarray(rs.F),
                row_ptr=Kff.indptr, col_idx=Kff.indices, vals=Kff.data,
                nnz_full=np.int64(Ks.nnz), U_lu=U_lu, U_pcg=U_pcg, uf_pcg=uf_pcg,
                pcg_iters=np.int64(n_iter), facets=np.array(facets, dtype=np.int64))


def pattern_4x3x2():
    from fea_engine.mesh import box_mesh
    from fea_engine.elements.solids import Hex8Solid3D
    from fea_engine.material import Material, D_solid3d
    from fea_engine.solver import FESystem
    from fea_engine.vectorized_assembly import scatter_global_stiffness, tensorized_element_stiffness
    from fea_engine.mesh_transform import MeshTransformation

    mesh = box_mesh(1.0, 0.6, 0.4, 4, 3, 2)
    elem = Hex8Solid3D()
    D = D_solid3d(Material(E=1.0e3, nu=0.25))
    ke = tensorized_element_stiffness(MeshTransformation(mesh, elem), D)
    n_dof = 3 * len(mesh.nodes)
    K = scatter_global_stiffness(ke, mesh.elements, 3, n_dof, sparse=True).tocsr()
    fixed = np.array(sorted(3 * int(n) + k for n in mesh.nodes_on_plane(0, 0.0) for k in (0, 1, 2)))
    fixed = np.union1d(fixed, [3 * int(n) + 1 for n in mesh.nodes_on_plane(1, 0.0)])  # a partial (uy only) set too
    free = np.setdiff1d(np.arange(n_dof), fixed)
    Kff = K[np.ix_(free, free)]
    fs = FESystem(mesh, elem, sparse=True)
    fs.assemble_stiffness(D)
    Kl = fs.K.tocsr()
    return dict(nodes=mesh.nodes, elements=np.asarray(mesh.elements, dtype=np.int64), D=D,
                fixed=fixed, free=free, K_row_ptr=K.indptr, K_col_idx=K.indices, K_vals=K.data,
                Kff_row_ptr=Kff.indptr, Kff_col_idx=Kff.indices, Kff_vals=Kff.data,
                lil_row_ptr=Kl.indptr, lil_col_idx=Kl.indices)


def ke_distorted():
    from fea_engine.elements.solids import Hex8Solid3D
    from fea_engine.material import Material, D_solid3d
    rng = np.random.default_rng(7)
    ref = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=float)
    coords = np.stack([ref * rng.uniform(0.3, 2.0, 3) + 0.15 * rng.standard_normal((8, 3)) for _ in range(6)])
    D = D_solid3d(Material(E=70e9, nu=0.33))
    elem = Hex8Solid3D()
    ke = np.stack([elem.stiffness(c, D) for c in coords])
    # an anisotropic (still symmetric) D exercises the general B^T D B path
    A = rng.standard_normal((6, 6))
    D_aniso = D + 1e9 * (A @ A.T)
    ke_aniso = np.stack([elem.stiffness(c, D_aniso) for c in coords])
    return dict(coords=coords, D=D, ke=ke, D_aniso=D_aniso, ke_aniso=ke_aniso)


def facets():
    from fea_engine import facet_loads
    rng = np.random.default_rng(11)
    sq = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], dtype=float)
    fc = np.stack([sq @ np.diag([rng.uniform(0.2, 1.5), rng.uniform(0.2, 1.5), 1.0])
                   + 0.05 * rng.standard_normal((4, 3)) for _ in range(5)])
    fc = fc[:, :, [2, 0, 1]]  # faces of constant-ish x, like the cantilever end face
    shares = np.stack([facet_loads.consistent_facet_load_shares(3, c, -2.5e5) for c in fc])
    mass = np.stack([facet_loads.consistent_facet_mass(3, c, 1.0) for c in fc])
    return dict(coords=fc, traction=np.float64(-2.5e5), shares=shares, mass=mass)


def simp_6x3x3():
    import torch  # noqa: F401  (the adjoint path needs torch; CPU is fine)
    from fea_engine.mesh import box_mesh
    from fea_engine.elements.solids import Hex8Solid3D
    from fea_engine.material import Material, D_solid3d
    from fea_engine.solver import FESystem
    from fea_engine import topopt

    mesh = box_mesh(1.2, 0.4, 0.4, 6, 3, 3)
    fs = FESystem(mesh, Hex8Solid3D())
    D = D_solid3d(Material(E=1.0, nu=0.3))
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    tip = mesh.nodes_on_plane(0, 1.2)
    target = np.array([1.2, 0.2, 0.2])
    node = int(tip[np.argmin(np.linalg.norm(mesh.nodes[tip] - target, axis=1))])
    F = np.zeros(fs.n_dof)
    F[3 * node + 2] = -1.0
    ke_unit, conn = topopt.unit_stiffness_stack(fs, D)
    rng = np.random.default_rng(5)
    rho = rng.uniform(0.3, 1.0, len(conn))
    p, rho_min = 3.0, 1e-9
    free = fs.free_dofs
    u, Kff, Ff = topopt.solve_simp_equilibrium(ke_unit, conn, 3, fs.n_dof, free, F, rho, p, rho_min)
    dc = topopt.compliance_sensitivity_closed_form(ke_unit, conn, 3, u, rho, p, rho_min)
    dc_adj = topopt.compliance_sensitivity_via_adjoint(ke_unit, conn, 3, fs.n_dof, free, u, Kff, Ff, rho, p, rho_min)
    h = 1e-6
    fd_elems = np.array([0, 5, 17, 40])
    fd = []
    for e in fd_elems:
        rp, rm = rho.copy(), rho.copy()
        rp[e] += h
        rm[e] -= h
        up, _, _ = topopt.solve_simp_equilibrium(ke_unit, conn, 3, fs.n_dof, free, F, rp, p, rho_min)
        um, _, _ = topopt.solve_simp_equilibrium(ke_unit, conn, 3, fs.n_dof, free, F, rm, p, rho_min)
        fd.append((topopt.compliance(F, up) - topopt.compliance(F, um)) / (2 * h))
    return dict(nodes=mesh.nodes, elements=np.asarray(conn, dtype=np.int64), D=D, F=F, rho=rho,
                p=np.float64(p), rho_min=np.float64(rho_min), free=free, u=u, dc=dc,
                dc_adjoint=np.asarray(dc_adj), fd_elems=fd_elems, dc_fd=np.array(fd),
                compliance=np.float64(topopt.compliance(F, u)))


def recovery_20x4x4():
    """FESystem.stress / strain / von_mises (nodes and elements) and reactions of the jittered
    20x4x4 cantilever at its SuperLU displacement (recovery.py through solver.py:413-445)."""
    fs, mesh, D, _ = _cantilever_20x4x4_system()
    U = np.asarray(fs.solve_static())
    n = len(mesh.nodes)
    return dict(nodes=np.asarray(mesh.nodes), elements=np.asarray(mesh.elements, dtype=np.int64), D=D, U=U,
                F=np.asarray(fs.F), fixed=np.asarray(fs.fixed_dofs_array),
                stress_nodes=np.asarray(fs.stress(U)).reshape(n, 6), stress_elements=np.asarray(fs.stress(U, at="elements")),
                strain_nodes=np.asarray(fs.strain(U)).reshape(n, 6), strain_elements=np.asarray(fs.strain(U, at="elements")),
                von_mises_nodes=np.asarray(fs.von_mises(U)), von_mises_elements=np.asarray(fs.von_mises(U, at="elements")),
                reactions=np.asarray(fs.reactions(U)))


def topopt_8x4x4():
    """The reference's SIMP loop on a small hex8 cantilever (2.0 x 1.0 x 1.0, 8x4x4, E = 1,
    nu = 0.3, x = 0 clamped, unit -z load at the tip node nearest (2, 0.5, 0)): filter weights,
    one filtered sensitivity, one OC update on seeded inputs, and topology_optimize_compliance
    (vf 0.4, p 3, rho_min 1e-2, move 0.2, filter radius 0.375, 12 iterations)."""
    from fea_engine.mesh import box_mesh
    from fea_engine.elements.solids import Hex8Solid3D
    from fea_engine.material import Material, D_solid3d
    from fea_engine.solver import FESystem
    from fea_engine import topopt

    mesh = box_mesh(2.0, 1.0, 1.0, 8, 4, 4)
    fs = FESystem(mesh, Hex8Solid3D())
    D = D_solid3d(Material(E=1.0, nu=0.3))
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    tip = mesh.nodes_on_plane(0, 2.0)
    node = int(tip[np.argmin(np.linalg.norm(mesh.nodes[tip] - np.array([2.0, 0.5, 0.0]), axis=1))])
    F = np.zeros(fs.n_dof)
    F[3 * node + 2] = -1.0
    conn = np.asarray(mesh.elements)
    centroids = mesh.nodes[conn].mean(axis=1)
    radius = 0.375
    H = topopt.build_filter_weights(centroids, radius)
    rng = np.random.default_rng(9)
    rho_s = rng.uniform(0.05, 1.0, len(conn))
    dc_s = -rng.uniform(0.1, 5.0, len(conn))
    dc_s[::17] = rng.uniform(0.0, 1e-3, dc_s[::17].shape)        # a few non-negative entries
    dc_filtered = topopt.apply_sensitivity_filter(H, rho_s, dc_s)
    rho_oc = topopt.oc_update(rho_s, dc_s, 0.4, move=0.2, rho_min_bound=1e-2)
    res = topopt.topology_optimize_compliance(fs, D, F, 0.4, p=3.0, rho_min=1e-2, move=0.2, n_iter=12,
                                             filter_radius=radius, tol=1e-3)
    return dict(nodes=np.asarray(mesh.nodes), elements=conn.astype(np.int64), D=D, F=F,
                fixed=np.asarray(fs.fixed_dofs_array), radius=np.float64(radius), H=H, rho_s=rho_s, dc_s=dc_s,
                dc_filtered=dc_filtered, rho_oc=rho_oc, rho_final=res["rho"],
                compliance_history=np.asarray(res["compliance_history"]), u_final=res["u_final"])


def bbar_hex8():
    """Hex8SolidBbar: element stiffness of 6 distorted hexes at nu = 0.3 and 0.4999, and the tip
    deflection of the reference's locking benchmark (fea_engine/tests/test_hex8_bbar.py:122-143:
    1.0 x 0.05 x 0.05 cantilever, 20x4x4, -1000 N on the tip face) with Hex8SolidBbar and
    Hex8Solid3D at nu = 0.4999, solved by FESystem.solve_static."""
    from fea_engine.elements.solids import Hex8Solid3D, Hex8SolidBbar
    from fea_engine.material import Material, D_solid3d
    from fea_engine.mesh import box_mesh
    from fea_engine.solver import FESystem

    rng = np.random.default_rng(17)
    cube = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    coords = np.stack([cube * rng.uniform(0.3, 2.0, 3) + 0.12 * rng.standard_normal((8, 3)) for _ in range(6)])
    out = dict(coords=coords)
    for tag, nu in (("03", 0.3), ("04999", 0.4999)):
        D = D_solid3d(Material(E=2.1e11, nu=nu))
        out["D_" + tag] = D
        out["ke_" + tag] = np.stack([Hex8SolidBbar().stiffness(c, D) for c in coords])
    mesh = box_mesh(1.0, 0.05, 0.05, 20, 4, 4)
    D = out["D_04999"]
    tip = mesh.nodes_on_plane(0, 1.0)
    for name, cls in (("bbar", Hex8SolidBbar), ("plain", Hex8Solid3D)):
        fs = FESystem(mesh, cls())
        fs.assemble_stiffness(D)
        fs.add_nodal_force(tip, dof_index=2, total_force=-1000.0)
        fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
        out["U_" + name] = np.asarray(fs.solve_static())
    out["nodes"] = np.asarray(mesh.nodes)
    out["elements"] = np.asarray(mesh.elements, dtype=np.int64)
    out["F"] = np.asarray(fs.F)
    return out


def modal_20x4x4():
    """Consistent mass and the modal solve of the jittered 20x4x4 cantilever: Hex8Solid3D.mass of
    6 distorted hexes (rho = 7850 I), and FESystem(sparse=True).assemble_mass(7850 I) +
    solve_modal(n_modes=6) (shift-invert eigsh)."""
    from fea_engine.elements.solids import Hex8Solid3D
    fs, mesh, D, _ = _cantilever_20x4x4_system()
    R = 7850.0 * np.eye(3)
    rng = np.random.default_rng(23)
    cube = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    coords = np.stack([cube * rng.uniform(0.3, 2.0, 3) + 0.1 * rng.standard_normal((8, 3)) for _ in range(6)])
    me = np.stack([Hex8Solid3D().mass(c, R) for c in coords])
    fs.assemble_mass(R)
    freq, modes = fs.solve_modal(n_modes=6)
    return dict(coords=coords, R=R, me=me, nodes=np.asarray(mesh.nodes), elements=np.asarray(mesh.elements, np.int64),
                D=D, fixed=np.asarray(fs.fixed_dofs_array), freq=np.asarray(freq), modes=np.asarray(modes),
                M_nnz=np.int64(fs.M.tocsr().nnz if hasattr(fs.M, "tocsr") else np.count_nonzero(fs.M)))


def pod_small():
    from rom_engine.pod import PodBasis
    rng = np.random.default_rng(3)
    t = np.linspace(0, 1, 400)[:, None]
    modes = np.cos(np.pi * np.arange(1, 13)[None, :] * t)
    X = (modes * (10.0 ** -np.arange(12) * 0.5)[None, :]) @ rng.standard_normal((12, 12))
    basis = PodBasis().fit(X, n_modes=10)
    return dict(X=X, singular_values=np.asarray(basis.singular_values))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    ap.add_argument("--only", nargs="*", default=None, help="fixture names to write (default: all)")
    args = ap.parse_args()
    _import_reference(args.reference)
    for name, fn in [("cantilever_20x4x4", cantilever_20x4x4), ("pattern_4x3x2", pattern_4x3x2),
                     ("ke_distorted", ke_distorted), ("facets", facets), ("simp_6x3x3", simp_6x3x3),
                     ("pod_small", pod_small), ("recovery_20x4x4", recovery_20x4x4),
                     ("topopt_8x4x4", topopt_8x4x4), ("bbar_hex8", bbar_hex8), ("modal_20x4x4", modal_20x4x4)]:
        if args.only and name not in args.only:
            continue
        data = fn()
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
