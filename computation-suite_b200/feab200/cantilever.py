"""Synthetic cantilever problems (seeded) for the benchmark and the tests.

Every problem is a hex8 box over Lx x Ly x Lz (default 2.0 x 0.4 x 0.4 m) built by
``box_mesh``, clamped on x = 0 (all three DOFs), and loaded on the x = L face with
consistent facet loads (facet_loads.py of the reference):
- ``uniform_tip``: uniform z traction (add_consistent_facet_load);
- ``nodal_tip``: per-node z traction field t, F = sum_faces M_face t (consistent_facet_mass);
- ``point``: a point z load at the tip node nearest (L, Ly/2, Lz/2).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .facet_loads import boundary_faces_on_plane, facet_load_shares_batch, facet_mass_batch
from .material import D_solid3d, Material
from .mesh import Mesh, box_mesh, jitter_interior


@dataclass
class Cantilever:
    mesh: Mesh
    D: np.ndarray
    fixed: np.ndarray            # sorted fixed DOFs
    F: np.ndarray                # (n_dof,) or (n_dof, k)
    meta: dict = field(default_factory=dict)

    @property
    def n_dof(self):
        return 3 * len(self.mesh.nodes)

    @property
    def free(self):
        mask = np.ones(self.n_dof, dtype=bool)
        mask[self.fixed] = False
        return np.flatnonzero(mask)


def clamped_dofs(mesh, axis=0, value=0.0):
    ids = mesh.nodes_on_plane(axis, value)
    return np.sort((3 * ids[:, None] + np.arange(3)[None, :]).reshape(-1))


def tip_faces(mesh, Lx):
    return boundary_faces_on_plane(mesh.nodes, mesh.elements, 0, Lx)


def uniform_tip_load(mesh, Lx, traction, dof=2):
    faces = tip_faces(mesh, Lx)
    F = np.zeros(3 * len(mesh.nodes))
    sh = facet_load_shares_batch(mesh.nodes[faces], traction)
    np.add.at(F, 3 * faces.reshape(-1) + dof, sh.reshape(-1))
    return F


def nodal_tip_load(mesh, Lx, t_nodes, dof=2):
    """F = sum over tip faces of M_face @ t (t per node, (n_nodes,) or (n_nodes, k))."""
    faces = tip_faces(mesh, Lx)
    M = facet_mass_batch(mesh.nodes[faces])                 # (F, 4, 4)
    t = np.asarray(t_nodes, dtype=float)
    k = 1 if t.ndim == 1 else t.shape[1]
    tf = t[faces].reshape(faces.shape[0], 4, k)              # (F, 4, k)
    contrib = np.einsum("fab,fbk->fak", M, tf)               # (F, 4, k)
    F = np.zeros((3 * len(mesh.nodes), k))
    np.add.at(F, 3 * faces.reshape(-1) + dof, contrib.reshape(-1, k))
    return F[:, 0] if t.ndim == 1 else F


def plain_cantilever(nx=20, ny=4, nz=4, Lx=2.0, Ly=0.4, Lz=0.4, E=210e9, nu=0.3, jitter=0.1, seed=1234,
                     traction=-1.0e6):
    """The CPU-runnable case: jittered interior nodes (+-5 % of the element size), uniform tip
    traction.  Same recipe as tests/golden/make_golden.py's 20x4x4 fixture."""
    mesh = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    if jitter:
        mesh = jitter_interior(mesh, jitter, seed, h=(Lx / nx, Ly / ny, Lz / nz))
    F = uniform_tip_load(mesh, Lx, traction)
    return Cantilever(mesh, D_solid3d(Material(E=E, nu=nu)), clamped_dofs(mesh), F,
                      dict(kind="plain", shape=(nx, ny, nz)))


def random_tip_cantilever(nx=128, ny=32, nz=32, Lx=2.0, Ly=0.4, Lz=0.4, E=210e9, nu=0.3, seed=2, scale=1.0e6):
    """Plain-vs-mixed case: per-node tip z traction N(0,1)*1e6 Pa (seeded), consistent load."""
    mesh = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    rng = np.random.default_rng(seed)
    t = np.zeros(len(mesh.nodes))
    tip = mesh.nodes_on_plane(0, Lx)
    t[tip] = scale * rng.standard_normal(len(tip))
    F = nodal_tip_load(mesh, Lx, t)
    return Cantilever(mesh, D_solid3d(Material(E=E, nu=nu)), clamped_dofs(mesh), F,
                      dict(kind="random_tip", shape=(nx, ny, nz)))


def simp_cantilever(nx=96, ny=32, nz=32, Lx=2.0, Ly=0.4, Lz=0.4, nu=0.3, seed=4, rho_lo=0.3, rho_hi=1.0):
    """SIMP case: E0 = 1, unit -z point load at the tip node nearest (L, Ly/2, Lz/2),
    element densities U[0.3, 1] (seeded)."""
    mesh = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    tip = mesh.nodes_on_plane(0, Lx)
    node = int(tip[np.argmin(np.linalg.norm(mesh.nodes[tip] - np.array([Lx, Ly / 2, Lz / 2]), axis=1))])
    F = np.zeros(3 * len(mesh.nodes))
    F[3 * node + 2] = -1.0
    rng = np.random.default_rng(seed)
    rho = rng.uniform(rho_lo, rho_hi, len(mesh.elements))
    return Cantilever(mesh, D_solid3d(Material(E=1.0, nu=nu)), clamped_dofs(mesh), F,
                      dict(kind="simp", shape=(nx, ny, nz), rho=rho, load_node=node))


def batch_cantilevers(n_problems=256, seed=3, nx_range=(8, 48), nyz_range=(4, 16), rhs_range=(4, 16),
                      Lx=2.0, Ly=0.4, Lz=0.4, nu=0.3):
    """Uneven batch: nx ~ U{8..48}, ny = nz ~ U{4..16}, E ~ lognormal(ln 210e9, 0.3), 4-16 load
    cases each with a uniform tip z traction ~ N(0, 1e6) Pa."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_problems):
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        nyz = int(rng.integers(nyz_range[0], nyz_range[1] + 1))
        E = float(np.exp(rng.normal(np.log(210e9), 0.3)))
        k = int(rng.integers(rhs_range[0], rhs_range[1] + 1))
        tr = rng.normal(0.0, 1.0e6, k)
        mesh = box_mesh(Lx, Ly, Lz, nx, nyz, nyz)
        unit = uniform_tip_load(mesh, Lx, 1.0)
        F = unit[:, None] * tr[None, :]
        out.append(Cantilever(mesh, D_solid3d(Material(E=E, nu=nu)), clamped_dofs(mesh), F,
                              dict(kind="batch", shape=(nx, nyz, nyz), E=E, tractions=tr)))
    return out


def fourier_snapshot_cantilever(nx=192, ny=48, nz=48, Lx=2.0, Ly=0.4, Lz=0.4, E=210e9, nu=0.3, n_rhs=64,
                                n_modes=8, seed=5, amplitude=1.0e6):
    """Snapshot case: n_rhs tip z tractions, each sum_m a_m cos(2 pi (ky y/Ly + kz z/Lz) + phi_m)
    with seeded integer wavenumbers, phases and amplitudes, scaled to max |t| = amplitude."""
    mesh = box_mesh(Lx, Ly, Lz, nx, ny, nz)
    rng = np.random.default_rng(seed)
    tip = mesh.nodes_on_plane(0, Lx)
    y, z = mesh.nodes[tip, 1], mesh.nodes[tip, 2]
    T = np.zeros((len(mesh.nodes), n_rhs))
    for c in range(n_rhs):
        ky = rng.integers(0, 4, n_modes)
        kz = rng.integers(0, 4, n_modes)
        ph = rng.uniform(0, 2 * np.pi, n_modes)
        a = rng.standard_normal(n_modes)
        t = (a[None, :] * np.cos(2 * np.pi * (ky[None, :] * y[:, None] / Ly + kz[None, :] * z[:, None] / Lz)
                                 + ph[None, :])).sum(1)
        T[tip, c] = amplitude * t / np.abs(t).max()
    F = nodal_tip_load(mesh, Lx, T)
    return Cantilever(mesh, D_solid3d(Material(E=E, nu=nu)), clamped_dofs(mesh), F,
                      dict(kind="snapshot", shape=(nx, ny, nz)))
