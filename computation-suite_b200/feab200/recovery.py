"""Derived results on the GPU: strain, stress, von Mises and support reactions
(fea_engine/src/fea_engine/recovery.py, reached through FESystem.stress / strain / von_mises /
reactions, solver.py:413-445).

Stress is evaluated at the 2x2x2 Gauss points (sigma = D B u) and moved to the corner nodes by
the lumped L2 projection sum(N_a sigma |J| w) / sum(N_a |J| w) over the elements of each node
(recovery.py:196-334); ``at="elements"`` gives the volume-averaged element values.  Both come
from one kernel pair, ``feab_hex8_recover``.  Voigt order xx, yy, zz, xy, yz, xz; strains use
engineering shear.
"""
from __future__ import annotations

import numpy as np
import torch

from .fields import FEField

_NAMES = {"stress": ("sxx", "syy", "szz", "sxy", "syz", "sxz"),
          "strain": ("exx", "eyy", "ezz", "gxy", "gyz", "gxz")}


def _resolve_D(system, D):
    """recovery.py:45-52."""
    if D is not None:
        return np.asarray(D, dtype=float)
    args = getattr(system, "_stiffness_args", None)
    if args is None:
        raise RuntimeError("stress/strain recovery needs the constitutive matrix: call assemble_stiffness() "
                           "first (it is remembered) or pass D=.")
    return np.asarray(args[0], dtype=float)


def _check_vector(system, U):
    """recovery.py:55-62; a device tensor is accepted as it is."""
    if torch.is_tensor(U):
        if tuple(U.shape) != (system.n_dof,):
            raise ValueError(f"expected a displacement vector of length {system.n_dof}, got shape {tuple(U.shape)}.")
        if U.is_complex():
            raise NotImplementedError("recovery of complex (harmonic) fields: pass U.real or U.imag.")
        return U
    U = np.asarray(U)
    if U.ndim != 1 or U.shape[0] != system.n_dof:
        raise ValueError(f"expected a displacement vector of length {system.n_dof}, got shape {U.shape}.")
    if np.iscomplexobj(U):
        raise NotImplementedError("recovery of complex (harmonic) fields: pass U.real or U.imag.")
    return U


def _check_at(at):
    if at not in ("nodes", "elements"):
        raise ValueError("at must be 'nodes' or 'elements'.")


def _recover(system, U, D, kind, at, von_mises=False):
    if type(system.elem).__name__ != "Hex8Solid3D":
        # coefficients.check_supported (coefficients.py:107-111): recovery covers Hex8Solid3D only
        raise NotImplementedError(f"{kind} recovery is not available for {type(system.elem).__name__}; "
                                  f"supported: Hex8Solid3D.")
    U = _check_vector(system, U)
    Dm = _resolve_D(system, D) if kind == "stress" else None
    out = system.device_mesh.recover(U, Dm, nodal=at == "nodes", elements=at == "elements", von_mises=von_mises)
    key = "nodal" if at == "nodes" else "elements"
    return out[key + "_vm"] if von_mises else out[key]


def _field(system, data, names, label):
    n = len(system.mesh.nodes)
    return FEField(np.ascontiguousarray(data).reshape(n * len(names)), n_nodes=n, dofs_per_node=len(names),
                   dof_names=names, label=label, mesh=system.mesh)


def stress(system, U, D=None, at="nodes", vectorized=True, backend="numpy", device="cpu"):
    """Stress components (recovery.py:365-373): an FEField of the nodal values, or with
    ``at="elements"`` an (n_elements, 6) array of element averages.  ``vectorized``, ``backend``
    and ``device`` are accepted for signature compatibility: every path is the GPU kernel."""
    _check_at(at)
    s = _recover(system, U, D, "stress", at).cpu().numpy()
    return s if at == "elements" else _field(system, s, _NAMES["stress"], "stress")


def strain(system, U, at="nodes", vectorized=True, backend="numpy", device="cpu"):
    """Strain components with engineering shear (recovery.py:376-383), laid out as ``stress``."""
    _check_at(at)
    e = _recover(system, U, None, "strain", at).cpu().numpy()
    return e if at == "elements" else _field(system, e, _NAMES["strain"], "strain")


def von_mises(system, U, D=None, plane="stress", nu=None, at="nodes", vectorized=True, backend="numpy",
              device="cpu"):
    """Von Mises equivalent stress (recovery.py:386-420).  ``plane`` / ``nu`` only matter for 2-D
    elements; they are validated as the reference does."""
    if plane not in ("stress", "strain"):
        raise ValueError("plane must be 'stress' or 'strain'.")
    if plane == "strain" and nu is None:
        raise ValueError("von_mises(plane='strain') needs the Poisson ratio nu= to form sigma_zz.")
    _check_at(at)
    v = _recover(system, U, D, "stress", at, von_mises=True).cpu().numpy()
    return v if at == "elements" else _field(system, v, ("von_mises",), "von Mises stress")


def stress_tensor(system, U, D=None, device="cpu", at="nodes"):
    """Stress as a device tensor, (n_nodes, 6) or (n_elements, 6) (recovery.py:349-354).  The
    GPU kernel has no backward, so a U that requires grad is refused."""
    if torch.is_tensor(U) and U.requires_grad:
        raise NotImplementedError("stress_tensor: differentiating the recovery is not available on the GPU path")
    _check_at(at)
    return _recover(system, U, D, "stress", at)


def von_mises_tensor(system, U, D=None, device="cpu", plane="stress", nu=None, at="nodes"):
    """Von Mises stress as a device tensor (recovery.py:357-362); see ``stress_tensor``."""
    if plane == "strain" and nu is None:
        raise ValueError("von_mises(plane='strain') needs the Poisson ratio nu= to form sigma_zz.")
    if torch.is_tensor(U) and U.requires_grad:
        raise NotImplementedError("von_mises_tensor: differentiating the recovery is not available on the GPU path")
    _check_at(at)
    return _recover(system, U, D, "stress", at, von_mises=True)


def reactions(system, U=None):
    """Support reactions R = K U - F at the constrained DOFs, zero elsewhere (recovery.py:422-448).
    K U is formed element by element on the GPU from the assembled element matrices."""
    if U is None:
        U = system.solve_static()
    U = _check_vector(system, U)
    system._require_stiffness("reactions")
    KU = system.device_mesh.apply(system._ke, U).cpu().numpy()
    r = KU - np.asarray(system.F, dtype=float).ravel()
    out = np.zeros(system.n_dof)
    fixed = system.fixed_dofs_array
    out[fixed] = r[fixed]
    return system.field(out, label="reaction")
