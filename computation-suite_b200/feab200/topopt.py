"""SIMP compliance sensitivities on the GPU (topopt.py:74-232 of the reference).

- ``compliance_sensitivity_closed_form``: dC/drho_e = -s'(rho_e) u_e^T K0_e u_e, one GPU
  kernel that recomputes K0_e's quadratic form from the coordinates at the Gauss points
  (topopt.py:161-177).
- ``compliance_sensitivity_via_adjoint``: adjoint solve K lam = -dC/du with the GPU PCG, then
  the VJP of rho -> K(rho) u with the same kernel (topopt.py:180-232, differentiable.py:478-512).
- ``SimpSolve``: torch.autograd.Function u = K(rho)^-1 f with a hand-written backward that
  reuses the PCG for the adjoint system; u can be recomputed instead of stored.
- ``topology_optimize_compliance``: the SIMP optimality-criteria loop (topopt.py:235-379) with
  the filter weights, the sensitivity filter and the OC bisection on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .device import DeviceMesh, DeviceStatus, cuda_device, pcg_solve
from .elements import is_bbar


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
    if is_bbar(fesystem.elem):
        # the reference builds the stack with MeshTransformation, which refuses elements that
        # override Element.stiffness (mesh_transform.py:155-170)
        raise ValueError("unit_stiffness_stack: Hex8SolidBbar overrides the element stiffness; the SIMP "
                         "path supports Hex8Solid3D")
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


# ---------------------------------------------------------------------------- SIMP OC loop
class FilterWeights:
    """The sensitivity-filter weights H of build_filter_weights (topopt.py:235-243) on the device,
    as a CSR over elements holding the positive entries (columns ascending) and the row sums."""

    def __init__(self, ptr, idx, w, rowsum):
        self.ptr, self.idx, self.w, self.rowsum = ptr, idx, w, rowsum
        self.n = int(rowsum.shape[0])
        self.nnz = int(w.shape[0])

    @property
    def shape(self):
        return (self.n, self.n)

    @property
    def device(self):
        return self.rowsum.device

    def toarray(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.w.cpu().numpy(), self.idx.cpu().numpy(), self.ptr.cpu().numpy()),
                             shape=self.shape).toarray()

    @classmethod
    def from_dense(cls, H, device=None):
        import scipy.sparse as sp
        dev = cuda_device(device)
        A = sp.csr_matrix(np.asarray(H, dtype=float))
        A.eliminate_zeros()
        A.sort_indices()
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt)).to(dev)  # noqa: E731
        return cls(t(A.indptr, np.int32), t(A.indices, np.int32), t(A.data, np.float64),
                   t(np.asarray(A.sum(axis=1)).ravel(), np.float64))


def element_centroids(dmesh: DeviceMesh):
    """(n_elem, 3) device tensor: mean of each element's 8 corner coordinates."""
    out = torch.empty((dmesh.n_elem, 3), dtype=torch.float64, device=dmesh.device)
    rc = L.lib.feab_element_centroids(L.dptr(dmesh.coords), L.dptr(dmesh.conn), dmesh.n_elem, L.dptr(out),
                                      dmesh.stream)
    L.raise_for(rc, "element centroids")
    return out


def build_filter_weights(centroids, radius, device=None):
    """H[e, j] = max(0, radius - |c_e - c_j|) for every pair (topopt.py:235-243), built on the GPU
    and kept sparse (a FilterWeights; ``.toarray()`` gives the reference's dense array).  2-D
    centroids are taken as z = 0."""
    if torch.is_tensor(centroids):
        dev = centroids.device
        c = centroids.to(torch.float64)
    else:
        dev = cuda_device(device)
        c = torch.as_tensor(np.asarray(centroids, dtype=float)).to(dev)
    if c.ndim != 2 or c.shape[1] not in (2, 3):
        raise ValueError(f"centroids must be (n, 2) or (n, 3), got {tuple(c.shape)}")
    if c.shape[1] == 2:
        c = torch.cat([c, torch.zeros((c.shape[0], 1), dtype=torch.float64, device=dev)], dim=1)
    c = c.contiguous()
    n = int(c.shape[0])
    if not (float(radius) > 0.0):
        raise ValueError("build_filter_weights: radius must be positive")
    stream = L.stream_ptr(dev)
    ptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    sbytes = int(L.lib.feab_filter_scratch_bytes(n))
    scratch = torch.empty(max(sbytes, 1), dtype=torch.uint8, device=dev)
    nnz = C.c_int64(0)
    rc = L.lib.feab_filter_build(L.dptr(c), n, float(radius), L.dptr(ptr), None, None, None, C.byref(nnz),
                                 L.dptr(scratch), sbytes, stream)
    L.raise_for(rc, "filter weights")
    idx = torch.empty(max(int(nnz.value), 1), dtype=torch.int32, device=dev)
    w = torch.empty(max(int(nnz.value), 1), dtype=torch.float64, device=dev)
    rowsum = torch.empty(n, dtype=torch.float64, device=dev)
    rc = L.lib.feab_filter_build(L.dptr(c), n, float(radius), L.dptr(ptr), L.dptr(idx), L.dptr(w), L.dptr(rowsum),
                                 None, None, 0, stream)
    L.raise_for(rc, "filter weights")
    return FilterWeights(ptr, idx[: int(nnz.value)], w[: int(nnz.value)], rowsum)


def _as_device(x, dev):
    return torch.as_tensor(x, dtype=torch.float64).to(dev).contiguous()


def apply_sensitivity_filter(H, rho, dc, eps=1e-9):
    """dc~_e = sum_j H_ej rho_j dc_j / max(max(rho_e, eps) sum_j H_ej, eps) (topopt.py:246-253) on
    the GPU.  H: a FilterWeights (or a dense array, uploaded as one).  Returns the type of dc."""
    if not isinstance(H, FilterWeights):
        H = FilterWeights.from_dense(H, dc.device if torch.is_tensor(dc) else None)
    dev = H.device
    r, d = _as_device(rho, dev), _as_device(dc, dev)
    if r.shape != (H.n,) or d.shape != (H.n,):
        raise ValueError(f"rho and dc must have shape ({H.n},)")
    out = torch.empty(H.n, dtype=torch.float64, device=dev)
    rc = L.lib.feab_filter_apply(L.dptr(H.ptr), L.dptr(H.idx), L.dptr(H.w), L.dptr(H.rowsum), H.n, L.dptr(r),
                                 L.dptr(d), float(eps), L.dptr(out), L.stream_ptr(dev))
    L.raise_for(rc, "sensitivity filter")
    return out if torch.is_tensor(dc) else out.cpu().numpy()


def _oc_device(rho, dc, volume_fraction, move, rho_min_bound, rho_max_bound, bisection_tol, max_bisection_iter):
    """(rho_new, max |rho_new - rho|) as device tensors; rho and dc are device FP64 vectors."""
    dev = rho.device
    n = int(rho.shape[0])
    out = torch.empty(n, dtype=torch.float64, device=dev)
    change = torch.zeros(1, dtype=torch.float64, device=dev)
    wbytes = int(L.lib.feab_oc_workspace_bytes(n))
    ws = torch.empty(wbytes, dtype=torch.uint8, device=dev)
    rc = L.lib.feab_oc_update(L.dptr(rho), L.dptr(dc), n, float(volume_fraction), float(move), float(rho_min_bound),
                              float(rho_max_bound), float(bisection_tol), int(max_bisection_iter), L.dptr(out),
                              L.dptr(change), L.dptr(ws), wbytes, L.stream_ptr(dev))
    L.raise_for(rc, "OC update")
    return out, change


def oc_update(rho, dc, volume_fraction, move=0.2, rho_min_bound=1e-3, rho_max_bound=1.0, bisection_tol=1e-4,
              max_bisection_iter=100):
    """Optimality-criteria density update with the bisection on the volume multiplier run on the
    GPU (topopt.py:259-295).  Returns the type of rho."""
    dev = rho.device if torch.is_tensor(rho) else (dc.device if torch.is_tensor(dc) else cuda_device(None))
    r, d = _as_device(rho, dev), _as_device(dc, dev)
    if r.ndim != 1 or r.shape != d.shape or r.numel() == 0:
        raise ValueError("oc_update: rho and dc must be non-empty vectors of the same length")
    out, _ = _oc_device(r, d, volume_fraction, move, rho_min_bound, rho_max_bound, bisection_tol,
                        max_bisection_iter)
    return out if torch.is_tensor(rho) else out.cpu().numpy()


def topology_optimize_compliance(fesystem, D, F_ext, volume_fraction, p=3.0, rho_min=1e-3, move=0.2, n_iter=50,
                                 filter_radius=None, sensitivity="closed_form", rho_init=None, tol=1e-3,
                                 pcg_tol=1e-12, precision="fp64"):
    """The SIMP compliance-minimisation loop (topopt.py:298-379) with every step on the GPU:
    K(rho) assembly, PCG to ``pcg_tol`` (the reference solves directly), dC/drho (closed form or
    adjoint), the sensitivity filter and the OC update; one host read per iteration (the
    compliance and the largest density change).  Returns {"rho", "compliance_history",
    "u_final"} as the reference does."""
    if sensitivity not in ("closed_form", "adjoint"):
        raise ValueError(f"topology_optimize_compliance: unknown sensitivity={sensitivity!r} "
                         f"-- expected 'closed_form' or 'adjoint'.")
    if is_bbar(fesystem.elem):
        raise ValueError("topology_optimize_compliance: Hex8SolidBbar overrides the element stiffness; the SIMP "
                         "path supports Hex8Solid3D (as the reference's MeshTransformation does)")
    dm = fesystem.device_mesh
    dev = dm.device
    free = fesystem.free_dofs
    prob = SimpProblem(dm, D, free, penal=p, rho_min=rho_min, tol=pcg_tol, precision=precision)
    F_full = _as_device(np.asarray(F_ext, dtype=float), dev)
    if F_full.shape != (fesystem.n_dof,):
        raise ValueError(f"F_ext must have shape ({fesystem.n_dof},)")
    f = F_full[prob.free].contiguous()
    n_el = dm.n_elem
    if rho_init is None:
        rho = torch.full((n_el,), float(volume_fraction), dtype=torch.float64, device=dev)
    else:
        rho = _as_device(np.array(rho_init, dtype=float), dev)
    H = None
    if filter_radius is not None and filter_radius > 0:
        H = build_filter_weights(element_centroids(dm), filter_radius)
    history = []
    u_full = None
    for _ in range(n_iter):
        u_free = prob.solve_free(rho, f)
        u_full = prob.full(u_free)
        history.append(float(torch.dot(F_full, u_full)))
        if sensitivity == "closed_form":
            dc = dm.simp_vjp(prob.D, rho, p, rho_min, u_full)
        else:
            lam = prob.full(prob.solve_free(rho, -f))
            dc = -dm.simp_vjp(prob.D, rho, p, rho_min, u_full, lam=lam)
        if H is not None:
            dc = apply_sensitivity_filter(H, rho, dc)
        rho_new, change = _oc_device(rho, dc, volume_fraction, move, rho_min, 1.0, 1e-4, 100)
        rho = rho_new
        if float(change.item()) < tol:
            break
    return {"rho": rho.cpu().numpy(), "compliance_history": history,
            "u_final": None if u_full is None else u_full.cpu().numpy()}
