"""Consistent facet loads on hex8 faces (host side, small).

Follows fea_engine/src/fea_engine/facet_loads.py: the Hex8 face table (:172-179), facet
quadrature = 2x2 Gauss on the bilinear face (:218-260), the Gram-determinant measure
(elements/base.py:308-311), consistent_facet_mass (:263-280) and
consistent_facet_load_shares (:283-325).  The *_batch helpers do the same integrals for many
faces at once with numpy."""
from __future__ import annotations

import math

import numpy as np

from .elements import is_hex8

# local node ids of each hex8 face, as the reference's table (needed for identical facet order)
HEX8_FACES = (
    ((0, 3, 2, 1), "quad4"),
    ((4, 5, 6, 7), "quad4"),
    ((0, 1, 5, 4), "quad4"),
    ((1, 2, 6, 5), "quad4"),
    ((2, 3, 7, 6), "quad4"),
    ((3, 0, 4, 7), "quad4"),
)


def list_facets(formulation):
    """(local_node_indices, family, None) per face of a hex8 element."""
    if not is_hex8(formulation):
        raise ValueError(f"facet_loads: no facet table for {type(formulation).__name__} (hex8 only)")
    return [(idx, fam, None) for idx, fam in HEX8_FACES]


def _quad4(xi, eta):
    N = 0.25 * np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
    dN = 0.25 * np.array([[-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)],
                          [-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)]])
    return N, dN


def _rule(quad_order):
    n = max(1, math.ceil((quad_order + 1) / 2))
    p, w = np.polynomial.legendre.leggauss(n)
    return [(a, b) for a in p for b in p], [wa * wb for wa in w for wb in w]


def _measure(dN, fc):
    J = np.einsum("in,fnj->fij", dN, fc)
    return np.sqrt(np.maximum(np.linalg.det(np.einsum("fij,fkj->fik", J, J)), 0.0))


def _as_faces(facet_coords):
    fc = np.asarray(facet_coords, dtype=float)
    if fc.ndim == 2:
        fc = fc[None]
    if fc.shape[1:] != (4, 3):
        raise ValueError("hex8 facets are 4-node quads in 3-D: coordinates must be (4, 3) per face")
    return fc


def facet_load_shares_batch(facet_coords, traction, quad_order=2):
    """(F, 4) consistent shares of a uniform scalar traction on F quad faces."""
    fc = _as_faces(facet_coords)
    out = np.zeros((fc.shape[0], 4))
    for p, w in zip(*_rule(quad_order)):
        N, dN = _quad4(*p)
        out += N[None, :] * traction * (_measure(dN, fc) * w)[:, None]
    return out


def facet_mass_batch(facet_coords, coefficient=1.0, quad_order=2):
    """(F, 4, 4) integral of c N_a N_b over F quad faces."""
    fc = _as_faces(facet_coords)
    out = np.zeros((fc.shape[0], 4, 4))
    for p, w in zip(*_rule(quad_order)):
        N, dN = _quad4(*p)
        out += (coefficient * _measure(dN, fc) * w)[:, None, None] * np.outer(N, N)[None]
    return out


def consistent_facet_load_shares(parent_dim, facet_coords, traction, quad_order=2):
    if parent_dim != 3 or np.asarray(facet_coords).shape != (4, 3):
        raise ValueError("consistent_facet_load_shares: hex8 faces (parent_dim=3, 4 nodes) only")
    return facet_load_shares_batch(facet_coords, traction, quad_order)[0]


def consistent_facet_mass(parent_dim, facet_coords, coefficient=1.0, quad_order=2):
    if parent_dim != 3 or np.asarray(facet_coords).shape != (4, 3):
        raise ValueError("consistent_facet_mass: hex8 faces (parent_dim=3, 4 nodes) only")
    if callable(coefficient):
        raise NotImplementedError("consistent_facet_mass: a callable coefficient is not supported")
    return facet_mass_batch(facet_coords, coefficient, quad_order)[0]


def boundary_faces_on_plane(nodes, elements, axis, value, tol=1e-9):
    """Global node tuples (F, 4) of every element face lying on a coordinate plane, in the
    reference's facet order: element order, then face-table order."""
    X = np.asarray(nodes)
    conn = np.asarray(elements)
    on = np.abs(X[:, axis] - value) < tol
    allf = np.stack([conn[:, list(idx)] for idx, _ in HEX8_FACES], axis=1)   # (E, 6, 4)
    return allf[np.all(on[allf], axis=2)]
