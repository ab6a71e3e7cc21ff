"""The hex8 solid element formulations: Hex8Solid3D (elements/solids.py:130-163) and the
mean-dilatation Hex8SolidBbar (elements/solids.py:225-270).

The element matrices themselves are computed on the GPU (libfeab200); this class carries the
formulation's identity and constants, and host-side shape functions for load integration."""
from __future__ import annotations

import numpy as np

_XI = np.array([-1, 1, 1, -1, -1, 1, 1, -1], dtype=float)
_ETA = np.array([-1, -1, 1, 1, -1, -1, 1, 1], dtype=float)
_ZETA = np.array([-1, -1, -1, -1, 1, 1, 1, 1], dtype=float)


class Hex8Solid3D:
    n_nodes, dofs_per_node, dim, gauss_order = 8, 3, 3, 2
    dof_names = ("ux", "uy", "uz")
    translational_dof_mask = (True, True, True)

    def shape_and_derivs(self, natural_coords):
        xi, eta, zeta = natural_coords
        N = 0.125 * (1 + xi * _XI) * (1 + eta * _ETA) * (1 + zeta * _ZETA)
        dxi = 0.125 * _XI * (1 + eta * _ETA) * (1 + zeta * _ZETA)
        deta = 0.125 * _ETA * (1 + xi * _XI) * (1 + zeta * _ZETA)
        dzeta = 0.125 * _ZETA * (1 + xi * _XI) * (1 + eta * _ETA)
        return N, np.vstack([dxi, deta, dzeta])

    def stiffness(self, elem_coords, D, thickness=1.0, gauss_order=None, device=None):
        """24x24 element stiffness of one element (computed by the GPU element kernel)."""
        if gauss_order not in (None, 2):
            raise NotImplementedError("Hex8Solid3D.stiffness: only the full 2x2x2 rule is implemented")
        from .device import DeviceMesh
        coords = np.asarray(elem_coords, dtype=float).reshape(8, 3)
        dm = DeviceMesh(coords, np.arange(8)[None, :], device=device)
        from . import _lib as L
        return dm.element_stiffness(D, thickness=thickness, layout=L.KE_FULL, bbar=is_bbar(self))[0].cpu().numpy()

    def full_stiffness(self, elem_coords, D, thickness=1.0):
        return self.stiffness(elem_coords, D, thickness)


class Hex8SolidBbar(Hex8Solid3D):
    """Hex8 with the mean-dilatation B-bar: at each of the 8 Gauss points the volumetric part of
    B is replaced by its volume average (elements/solids.py:225-257), which relieves volumetric
    locking as nu -> 0.5.  Its element matrices come from feab_hex8_bbar_element_stiffness."""

    def stiffness(self, elem_coords, D, thickness=1.0, gauss_order=None, device=None):
        """B-bar is only defined at the full 8-point rule; gauss_order is ignored, as in the
        reference (elements/solids.py:250-262)."""
        return super().stiffness(elem_coords, D, thickness=thickness, gauss_order=None, device=device)

    def reduced_stiffness(self, elem_coords, D, thickness=1.0):
        raise NotImplementedError(
            "Hex8SolidBbar has no reduced-integration variant -- B-bar's mean-dilatation correction is only "
            "meaningful at the full 8-point rule. Use Hex8Solid3D for a reduced-integration Hex8.")


def is_hex8(formulation):
    """Accept this package's Hex8Solid3D / Hex8SolidBbar or the reference's classes of those names."""
    return (type(formulation).__name__ in ("Hex8Solid3D", "Hex8SolidBbar")
            and getattr(formulation, "n_nodes", 8) == 8)


def is_bbar(formulation):
    return type(formulation).__name__ == "Hex8SolidBbar"
