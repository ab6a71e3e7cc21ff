"""SIMP compliance sensitivities on the GPU (topopt.py:74-232 of the reference).

- ``compliance_sensitivity_closed_form``: dC/drho_e = -s'(rho_e) u_e^T K0_e u_e, one GPU
  kernel that recomputes K0_e's quadratic form from the coordinates at the Gauss points
  (topopt.py:161-177).
- ``compliance_sensitivity_via_adjoint``: adjoint solve K lam = -dC/du with the GPU PCG, then
  the VJP of rho -> K(rho) u with the same kernel (topopt.py:180-232, differentiable.py:478-512).
- ``SimpSolve``: torch.autograd.Function u = K(rho)^-1 f with a hand-written backward that
  reuses the PCG for the adjoint system; u can be recomputed instead of stored.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from .device import DeviceMesh, DeviceStatus, pcg_solve


def simp_scale(rho, p=3.0, rho_min=1e-3):
    """s = rho_min + (1 - rho_min) rho^p (topopt.py:74-82)."""
    if torch.is_tensor(rho):
        return rho_min + (1.0 - rho_min) * rho ** p
    rho = np.asarray(rho, dtype=float)
    return rho_min + (1.0 - rho_min) * rho ** p


def simp_scale_grad(rho, p=3.0, rho_min=1e-3):
    """ds/drho = p (1 - rho_min) rho^(p-1) (topopt.py:85-93)."""
    if torch.is_tensor(rho):
        return p * (1.0 - rho_min) * rho ** (p - 1.0)
    rho = np.asarray(rho, dtype=float)
    return p * (1.0 - rho_min) * rho ** (p - 1.0)


class UnitStiffnessStack:
    """Stand-in for the reference's (E, 24, 24) ke_unit array: the mesh and D at rho = 1.
    The GPU kernels recompute what they need from it; ``.ke`` / ``np.asarray`` materialise
    the full stack on request."""

    def __init__(self, dmesh: DeviceMesh, D):
        self.dmesh = dmesh
        self.D = np.asarray(D, dtype=float)
        self._ke = None

    @property
    def shape(self):
        return (self.dmesh.n_elem, 24, 24)

    @property
    def ke(self):
        if self._ke is None:
            self._ke = self.dmesh.element_stiffness(self.D, layout=L.KE_FULL)
        return self._ke

    def __array__(self, dtype=None, copy=None):
        a = self.ke.cpu().numpy()
        return a.astype(dtype) if dtype is not None else a

    def __len__(self):
        return self.dmesh.n_elem


def unit_stiffness_stack(fesystem, D, gauss_order=None):
    """(ke_unit, connectivity) at rho = 1 (topopt.py:96-105)."""
    if gauss_order not in (None, 2):
        raise NotImplementedError("unit_stiffness_stack: only the full 2x2x2 rule is implemented")
    return UnitStiffnessStack(fesystem.device_mesh, D), np.asarray(fesystem.mesh.elements)


def _dmesh_of(ke_unit):
    if not isinstance(ke_unit, UnitStiffnessStack):
        raise TypeError("ke_unit must come from feab200.topopt.unit_stiffness_stack (the GPU path recomputes "
                        "element matrices from the mesh instead of reading a stored stack)")
    return ke_unit.dmesh


def compliance(F_ext, u_full):
    """C = F . u (topopt.py:150-158)."""
    if torch.is_tensor(F_ext) or torch.is_tensor(u_full):
        return float(torch.dot(torch.as_tensor(F_ext, dtype=torch.float64).flatten(),
                               torch.as_tensor(u_full, dtype=torch.float64).to(
                                   torch.as_tensor(F_ext).device).flatten()))
    return float(np.dot(F_ext, u_full))


def compliance_sensitivity_closed_form(ke_unit, connectivity, dofs_per_node, u_full, rho, p, rho_min):
    """dC/drho_e = -simp_scale_grad(rho_e) u_e^T ke_unit_e u_e, computed by the GPU kernel."""
    dm = _dmesh_of(ke_unit)
    out = dm.simp_vjp(ke_unit.D, rho, p, rho_min, u_full)
    return out.cpu().numpy() if not torch.is_tensor(u_full) else out


def _operator_for_scale(dm: DeviceMesh, D, scale, free_dofs, want32=False):
    free = np.asarray(free_dofs, dtype=np.int64)
    mask = np.ones(3 * dm.n_nodes, dtype=bool)
    mask[free] = False
    fixed = np.flatnonzero(mask)
    pat = dm.pattern(fixed)
    ke = dm.element_stiffness(D, scale=scale)
    return dm.assemble(ke, pat, want32=want32)


def _solve(op, rhs, tol, precision):
    x, info = pcg_solve(op, rhs, tol=tol, precision=precision)
    if info.status == L.FEAB_NOT_SPD:
        raise np.linalg.LinAlgError("SIMP equilibrium: K(rho) is not SPD")
    if info.status == L.FEAB_NOT_CONVERGED:
        raise RuntimeError(f"SIMP equilibrium: PCG did not converge in {info.iters} iterations")
    L.raise_for(info.status, "SIMP equilibrium")
    return x, info


def solve_simp_equilibrium(ke_unit, connectivity, dofs_per_node, n_dof, free_dofs, F_ext, rho, p, rho_min,
                           tol=1e-12, precision="fp64"):
    """K(rho) u = F_ext on the free DOFs (topopt.py:125-147) with the sparse GPU PCG.
    Returns (u_full, Kff operator, Ff)."""
    dm = _dmesh_of(ke_unit)
    scale = simp_scale(np.asarray(rho, dtype=float), p, rho_min)
    op = _operator_for_scale(dm, ke_unit.D, scale, free_dofs, want32=(precision == "fp32"))
    free = np.asarray(free_dofs, dtype=np.int64)
    Ff = torch.as_tensor(np.asarray(F_ext, dtype=float)[free]).to(dm.device)
    uf, _ = _solve(op, Ff, tol, precision)
    u = torch.zeros(n_dof, dtype=torch.float64, device=dm.device)
    u[torch.as_tensor(free).to(dm.device)] = uf
    return u.cpu().numpy(), op, Ff.cpu().numpy()


def compliance_sensitivity_via_adjoint(ke_unit, connectivity, dofs_per_node, n_dof, free_dofs, u_full, Kff, Ff, rho,
                                       p, rho_min, tol=1e-12):
    """lam = solve(Kff, -Ff) on the GPU, then lam^T d(K(rho) u)/drho (topopt.py:180-232)."""
    dm = _dmesh_of(ke_unit)
    free = np.asarray(free_dofs, dtype=np.int64)
    rhs = -torch.as_tensor(np.asarray(Ff, dtype=float)).to(dm.device)
    lam_f, _ = _solve(Kff, rhs, tol, "fp64")
    lam = torch.zeros(n_dof, dtype=torch.float64, device=dm.device)
    lam[torch.as_tensor(free).to(dm.device)] = lam_f
    # kernel: -s' lam_e^T K0_e u_e ; the VJP is +s' lam_e^T K0_e u_e
    return (-dm.simp_vjp(ke_unit.D, rho, p, rho_min, u_full, lam=lam)).cpu().numpy()


class SimpSolve(torch.autograd.Function):
    """u_free = K(rho)^-1 f_free on the GPU; backward: lam = K^-1 g (same PCG, K symmetric),
    df = lam, drho_e = -s'(rho_e) lam_e^T K0_e u_e.  With recompute=True only (rho, f) are saved
    and u is solved again in backward."""

    @staticmethod
    def forward(ctx, rho, f_free, problem, recompute):
        u = problem.solve_free(rho, f_free)
        ctx.problem = problem
        ctx.recompute = bool(recompute)
        if ctx.recompute:
            ctx.save_for_backward(rho, f_free)
        else:
            ctx.save_for_backward(rho, f_free, u)
        return u

    @staticmethod
    def backward(ctx, g):
        problem = ctx.problem
        if ctx.recompute:
            rho, f_free = ctx.saved_tensors
            u = problem.solve_free(rho, f_free)
        else:
            rho, f_free, u = ctx.saved_tensors
        lam = problem.solve_free(rho, g.contiguous())
        drho = problem.vjp_rho(rho, u, lam)
        return drho, lam, None, None


class SimpProblem:
    """A SIMP-scaled hex8 problem on the GPU: mesh, unit-modulus D, penalty, fixed DOFs."""

    def __init__(self, dmesh: DeviceMesh, D_unit, free_dofs, penal=3.0, rho_min=1e-9, tol=1e-12, precision="fp64"):
        self.dm = dmesh
        self.D = np.asarray(D_unit, dtype=float)
        self.free = torch.as_tensor(np.asarray(free_dofs, dtype=np.int64)).to(dmesh.device)
        mask = np.ones(3 * dmesh.n_nodes, dtype=bool)
        mask[np.asarray(free_dofs, dtype=np.int64)] = False
        self.fixed = np.flatnonzero(mask)
        self.penal = float(penal)
        self.rho_min = float(rho_min)
        self.tol = tol
        self.precision = precision
        self.last_info = None

    def operator(self, rho):
        scale = simp_scale(rho.detach(), self.penal, self.rho_min)
        pat = self.dm.pattern(self.fixed)
        ke = self.dm.element_stiffness(self.D, scale=scale)
        return self.dm.assemble(ke, pat, want32=(self.precision == "fp32"))

    def solve_free(self, rho, rhs):
        op = self.operator(rho)
        x, self.last_info = _solve(op, rhs.detach().to(torch.float64), self.tol, self.precision)
        return x

    def full(self, v_free):
        out = torch.zeros(3 * self.dm.n_nodes, dtype=torch.float64, device=self.dm.device)
        out[self.free] = v_free
        return out

    def vjp_rho(self, rho, u_free, lam_free):
        return self.dm.simp_vjp(self.D, rho.detach(), self.penal, self.rho_min, self.full(u_free.detach()),
                                lam=self.full(lam_free.detach()))

    def __call__(self, rho, f_free, recompute=False):
        return SimpSolve.apply(rho, f_free, self, recompute)
