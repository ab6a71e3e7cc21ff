"""Seeded cantilever workloads built from the oracle's own pieces (TEST INFRASTRUCTURE ONLY).

The benchmark's CPU arms and the large-size parity tests use these so that building their
inputs never loads the CUDA library.  Each builder follows the same recipe as the product's
workload generator (``feab200.cantilever``), and ``tests/test_host.py`` checks that both give
identical inputs:

- mesh: ``box_mesh`` over Lx x Ly x Lz (mesh.py:716-733, :1270-1289), x = 0 clamped in all
  three DOFs (Mesh.nodes_on_plane + FESystem.fix_dofs, mesh.py:330-332, solver.py:1163-1176);
- tip load from a per-node z traction field t: F = sum over the x = L faces of M_face t, with
  M_face = consistent_facet_mass(3, face_coords, 1.0) (facet_loads.py:263-280), the pattern of
  fea_engine/tests/test_benchmarks_convergence.py:193-196, faces in the reference's facet order
  (element order, then the Hex8 face table, facet_loads.py:172-179).
"""
from __future__ import annotations

import numpy as np

from .fea_oracle import D_solid3d, HEX8_FACES, box_mesh, facet_mass, fixed_dofs_on_plane, free_dofs

__all__ = ["tip_faces", "nodal_tip_load", "random_tip_cantilever", "simp_cantilever"]


def tip_faces(nodes, conn, Lx, tol=1e-9):
    """(F, 4) global node ids of every element face on the plane x = Lx."""
    on = np.abs(np.asarray(nodes)[:, 0] - Lx) < tol
    conn = np.asarray(conn)
    faces = np.stack([conn[:, list(f)] for f in HEX8_FACES], axis=1)        # (E, 6, 4)
    return faces[np.all(on[faces], axis=2)]


def nodal_tip_load(nodes, conn, Lx, t_nodes, dof=2):
    """F (3N,) or (3N, k) = sum over tip faces of M_face t (t per node, (N,) or (N, k))."""
    faces = tip_faces(nodes, conn, Lx)
    M = facet_mass(np.asarray(nodes)[faces], 1.0)                            # (F, 4, 4)
    t = np.asarray(t_nodes, dtype=float)
    tk = t.reshape(len(nodes), -1)
    contrib = np.einsum("fab,fbk->fak", M, tk[faces])                        # (F, 4, k)
    F = np.zeros((3 * len(nodes), tk.shape[1]))
    np.add.at(F, 3 * faces.reshape(-1) + dof, contrib.reshape(-1, tk.shape[1]))
    return F[:, 0] if t.ndim == 1 else F


def _problem(nodes, conn, D, F, **meta):
    fixed = fixed_dofs_on_plane(nodes, 0, 0.0)
    return dict(nodes=nodes, elements=conn, D=D, fixed=fixed, free=free_dofs(3 * len(nodes), fixed), F=F,
                n_dof=3 * len(nodes), **meta)


def random_tip_cantilever(nx=128, ny=32, nz=32, Lx=2.0, Ly=0.4, Lz=0.4, E=210e9, nu=0.3, seed=2, scale=1.0e6):
    """Per-node tip z traction N(0, 1) * scale (seeded), consistent load; E, nu isotropic."""
    nodes, conn = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    rng = np.random.default_rng(seed)
    t = np.zeros(len(nodes))
    tip = np.where(np.abs(nodes[:, 0] - Lx) < 1e-9)[0]
    t[tip] = scale * rng.standard_normal(len(tip))
    return _problem(nodes, conn, D_solid3d(E, nu), nodal_tip_load(nodes, conn, Lx, t), shape=(nx, ny, nz))


def simp_cantilever(nx=96, ny=32, nz=32, Lx=2.0, Ly=0.4, Lz=0.4, nu=0.3, seed=4, rho_lo=0.3, rho_hi=1.0):
    """E0 = 1, unit -z point load at the tip node nearest (Lx, Ly/2, Lz/2), densities
    U[rho_lo, rho_hi] per element (seeded)."""
    nodes, conn = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    tip = np.where(np.abs(nodes[:, 0] - Lx) < 1e-9)[0]
    node = int(tip[np.argmin(np.linalg.norm(nodes[tip] - np.array([Lx, Ly / 2, Lz / 2]), axis=1))])
    F = np.zeros(3 * len(nodes))
    F[3 * node + 2] = -1.0
    rho = np.random.default_rng(seed).uniform(rho_lo, rho_hi, len(conn))
    return _problem(nodes, conn, D_solid3d(1.0, nu), F, shape=(nx, ny, nz), rho=rho, load_node=node)
