"""Isotropic linear-elastic material (material.py:26-38) and the 3-D solid D matrix
(material.py:650-660): Voigt order xx, yy, zz, xy, yz, zx with engineering shear."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Material:
    E: float
    nu: float
    rho: float = 0.0

    @property
    def G(self):
        return self.E / (2.0 * (1.0 + self.nu))


def D_solid3d(mat) -> np.ndarray:
    E, nu = mat.E, mat.nu
    c = E / ((1 + nu) * (1 - 2 * nu))
    g = (1 - 2 * nu) / 2
    return c * np.array([[1 - nu, nu, nu, 0, 0, 0],
                         [nu, 1 - nu, nu, 0, 0, 0],
                         [nu, nu, 1 - nu, 0, 0, 0],
                         [0, 0, 0, g, 0, 0],
                         [0, 0, 0, 0, g, 0],
                         [0, 0, 0, 0, 0, g]], dtype=float)
