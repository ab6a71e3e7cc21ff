"""Hex8 mesh container and structured box generator (host side).

Mirrors the parts of ``fea_engine.mesh`` the hex8 static path uses: ``Mesh`` with
``nodes``/``elements``/``dim`` and node selection (mesh.py:268-332), and ``box_mesh``
(mesh.py:1288-1289 = ``extrude_mesh(rectangle_mesh(...))``, :716-733, :1270-1285) with the
same node and element numbering, so meshes built here or by the reference are interchangeable.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Mesh:
    nodes: np.ndarray       # (n_nodes, 3)
    elements: np.ndarray    # (n_elements, 8) int
    dim: int = 3
    node_sets: dict = field(default_factory=dict)

    def nodes_on_plane(self, axis, value, tol=1e-9):
        """Node ids with coordinate ``axis`` within tol of value (mesh.py:330-332)."""
        return np.where(np.abs(np.asarray(self.nodes)[:, axis] - value) < tol)[0]

    def add_node_set(self, name, ids):
        self.node_sets[name] = np.unique(np.asarray(ids, dtype=int))
        return self.node_sets[name]

    def select_nodes(self, x=None, y=None, z=None, tol=1e-9, name=None):
        """Nodes matching every given coordinate value (a subset of the reference's selector)."""
        X = np.asarray(self.nodes)
        mask = np.ones(len(X), dtype=bool)
        for axis, v in enumerate((x, y, z)):
            if v is not None:
                mask &= np.abs(X[:, axis] - v) < tol
        ids = np.where(mask)[0]
        if name is not None:
            self.add_node_set(name, ids)
        return ids


def box_mesh(Lx, Ly, Lz, nx, ny, nz):
    """Structured nx x ny x nz hex8 box over [0,Lx]x[0,Ly]x[0,Lz].

    Numbering: 2-D node (i, j) -> i*(ny+1)+j at (i*Lx/nx, j*Ly/ny); layer k of the extrusion
    holds those nodes at z = linspace(0, Lz, nz+1)[k] with offset k*(nx+1)*(ny+1); element
    (k, i, j) = [quad(i,j) + k*n2d, quad(i,j) + (k+1)*n2d] with quad(i,j) =
    [(i,j), (i+1,j), (i+1,j+1), (i,j+1)], ordered k, i, j (outer to inner)."""
    nx, ny, nz = int(nx), int(ny), int(nz)
    if min(nx, ny, nz) < 1:
        raise ValueError("box_mesh needs at least one element per direction")
    n2d = (nx + 1) * (ny + 1)
    i2, j2 = np.divmod(np.arange(n2d), ny + 1)
    xy = np.stack([0.0 + i2 * (Lx / nx), 0.0 + j2 * (Ly / ny)], axis=1)
    z = 0.0 + np.linspace(0.0, Lz, nz + 1)
    nodes = np.empty((n2d * (nz + 1), 3))
    nodes[:, 0:2] = np.tile(xy, (nz + 1, 1))
    nodes[:, 2] = np.repeat(z, n2d)
    qi, qj = np.divmod(np.arange(nx * ny), ny)
    base = qi * (ny + 1) + qj
    quad = np.stack([base, base + (ny + 1), base + (ny + 1) + 1, base + 1], axis=1)
    k = np.arange(nz)[:, None, None] * n2d
    elements = np.concatenate([quad[None] + k, quad[None] + k + n2d], axis=2).reshape(-1, 8)
    return Mesh(nodes=nodes, elements=elements.astype(np.int64), dim=3)


def jitter_interior(mesh, fraction, seed, h=None):
    """Copy of ``mesh`` whose strictly-interior nodes are moved by U(-fraction/2, fraction/2)*h
    per axis (h = element size per axis for a box; the style of the reference's distorted-mesh
    tests).  A seeded numpy Generator draws the offsets in node order."""
    X = np.array(mesh.nodes, dtype=float, copy=True)
    lo, hi = X.min(0), X.max(0)
    if h is None:
        raise ValueError("jitter_interior needs the element size h per axis")
    inner = np.all((X > lo + 1e-9) & (X < hi - 1e-9), axis=1)
    rng = np.random.default_rng(seed)
    X[inner] += fraction * np.asarray(h, dtype=float) * (rng.random((int(inner.sum()), 3)) - 0.5)
    return Mesh(nodes=X, elements=np.asarray(mesh.elements), dim=3)
