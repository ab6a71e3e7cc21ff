"""ReducedSystem: the constrained system K_ff u_f = F_f - K_fc u_c (linear_system.py:26-162),
with K_ff resident on the GPU."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from .device import ReducedOperator, pcg_solve


@dataclass
class ReducedSystem:
    operator: ReducedOperator
    F_device: torch.Tensor
    free: np.ndarray
    fixed: np.ndarray
    u_fixed: np.ndarray
    n_dof: int
    _system: object = field(default=None, repr=False, compare=False)
    _K_host: object = field(default=None, repr=False, compare=False)

    @property
    def K(self):
        """Host scipy CSR copy of K_ff (built on first access)."""
        if self._K_host is None:
            self._K_host = self.operator.to_scipy()
        return self._K_host

    @property
    def F(self):
        return self.F_device.cpu().numpy()

    @property
    def n_free(self):
        return len(self.free)

    def restrict(self, v):
        return np.asarray(v)[self.free]

    def expand(self, u_free, include_prescribed=True):
        u_free = u_free.detach().cpu().numpy() if torch.is_tensor(u_free) else np.asarray(u_free)
        if u_free.shape[0] != self.n_free:
            raise ValueError(f"expected {self.n_free} free-DOF rows, got {u_free.shape[0]}")
        full = np.zeros((self.n_dof,) + u_free.shape[1:])
        full[self.free] = u_free
        if include_prescribed and u_free.ndim == 1:
            full[self.fixed] = self.u_fixed
        return full

    def recover(self, u_free, label="displacement", include_prescribed=True):
        full = self.expand(u_free, include_prescribed=include_prescribed)
        return self._system.field(full, label=label) if self._system is not None else full

    def solve(self, label="displacement", tol=1e-12, max_iter=None, precision="fp64", **_ignored):
        x, info = pcg_solve(self.operator, self.F_device, tol=tol, maxiter=max_iter, precision=precision)
        if info.status == L.FEAB_NOT_SPD:
            raise np.linalg.LinAlgError("ReducedSystem.solve: K is not SPD")
        if info.status == L.FEAB_NOT_CONVERGED:
            raise RuntimeError(f"ReducedSystem.solve: CG did not converge in {info.iters} iterations (tol={tol})")
        L.raise_for(info.status, "ReducedSystem.solve")
        return self.recover(x, label=label)

    def residual(self, u_free):
        return self.K @ np.asarray(u_free) - self.F
