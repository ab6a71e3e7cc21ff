"""FESystem: drop-in for fea_engine's FESystem on the hex8 linear-elastic static path.

Same constructor, method names, argument meaning and exceptions as
fea_engine/src/fea_engine/solver.py for: assemble_stiffness (:569-697), fix_dofs
(:1109-1176), add_nodal_force (:1178-1206), add_consistent_facet_load (:1229-1274),
free_dofs / fixed_dofs_array (:1400-1401, :1482-1487), form_linear_system (:1403-1441) and
solve_static (:1726-2038).  Assembly and the solve run in libfeab200 on the GPU; the load
vector F and the boundary-condition bookkeeping stay host-side numpy, as in the reference.

Differences, by design:
- Hex8Solid3D, single block, method="full" only (others raise NotImplementedError).
- solve_static(method=None) (the reference's SuperLU direct solve) factors K_ff with a banded
  Cholesky on the GPU (feab200.direct) and reuses the factor for later loads; a band that does
  not fit in device memory falls back to Jacobi-PCG to 1e-12, and a singular K_ff gives the
  minimum-norm least-squares solution, as the reference's eigenvalue fallback does.
- ``K`` (the full matrix, built on first access) is the structural CSR: entries that cancel to
  exactly 0.0 are kept, where the reference's LIL storage drops them.
- Extra keyword ``precision="fp64"|"mixed"|"fp32"`` on solve_static selects the PCG precision
  (libfeab200's FEAB_PREC_*); every choice converges on the FP64 residual.
"""
from __future__ import annotations

import functools
import time
import warnings

import numpy as np
import torch

from . import _lib as L
from .device import DeviceMesh, DeviceStatus, cuda_device, pcg_solve
from .elements import is_bbar, is_hex8
from .facet_loads import facet_load_shares_batch
from .fields import FEField


class FESystem:
    def __init__(self, mesh, elem_formulation, thickness=1.0, sparse=False, backend="scipy", device="cpu"):
        if backend not in ("scipy", "torch", "auto"):
            raise ValueError(f"FESystem: unknown backend={backend!r} -- expected 'scipy', 'torch' or 'auto'.")
        if isinstance(elem_formulation, dict):
            raise NotImplementedError("FESystem: multi-block meshes are not supported on the hex8 GPU path")
        if not is_hex8(elem_formulation):
            raise NotImplementedError(
                f"FESystem: only Hex8Solid3D and Hex8SolidBbar are implemented on the GPU path, got "
                f"{type(elem_formulation).__name__}")
        nodes = np.asarray(mesh.nodes, dtype=float)
        if nodes.ndim != 2 or nodes.shape[1] != 3:
            raise ValueError("FESystem: a hex8 solid mesh needs 3-D node coordinates")
        self.mesh = mesh
        self.elem = elem_formulation
        self.thickness = thickness
        self.sparse = sparse
        self.backend = backend
        self.device_name = device
        self.npn = 3
        self.n_dof = 3 * len(nodes)
        self.F = np.zeros(self.n_dof)
        self.fixed_dofs = set()
        self.fixed_dof_values = {}
        self._assembled = set()
        self._warned_reassembly = set()
        self._dmesh = None
        self._ke = None          # packed element matrices on the device (E, 324)
        self._ke_version = 0
        self._op_cache = None    # (key, ReducedOperator)
        self._K_full = None
        self._stiffness_args = None
        self.last_solve_info = None
        self._bc_cache = None    # (frozenset of fixed DOFs, free, fixed, {device: (free_t, fixed_t)})
        self._me = None          # packed consistent element mass matrices on the device (E, 324)
        self._me_version = 0
        self._mop_cache = None   # (key, ReducedOperator of M_ff)
        self._M_full = None
        self.last_modal_iterations = None

    # ------------------------------------------------------------------ device objects
    @property
    def device(self):
        return self.device_mesh.device

    @property
    def device_mesh(self) -> DeviceMesh:
        if self._dmesh is None:
            self._dmesh = DeviceMesh(self.mesh.nodes, self.mesh.elements, device=cuda_device(self.device_name))
        return self._dmesh

    # ------------------------------------------------------------------ named DOFs
    @property
    def dof_names(self):
        return ("ux", "uy", "uz")

    def dof_index(self, name):
        return self._dof_index_by_name(name, "dof_index")

    def _dof_index_by_name(self, name, who):
        low = [n.lower() for n in self.dof_names]
        if str(name).lower() in low:
            return low.index(str(name).lower())
        raise ValueError(f"{who}: unknown DOF name {name!r}; valid names: {list(self.dof_names)}.")

    # ------------------------------------------------------------------ input validation
    # What the reference accepts for node and DOF selections (and the ValueError texts it raises)
    # is part of the drop-in contract; the checks below are written from that contract:
    #   * ids come as a scalar, a sequence, an array or a set; float ids are accepted when every
    #     value is integral; anything else is "must be integers";
    #   * node selections may instead name mesh node sets (one name or a list of names), which
    #     select the sorted union of those sets; unknown names are an error;
    #   * local DOFs may be given by index or by DOF name ("ux", ...);
    #   * an empty selection and ids outside the valid range are errors.
    @staticmethod
    def _as_int_array(values, what, who):
        flat = np.ravel(np.asarray(list(values) if isinstance(values, (set, frozenset)) else values))
        if flat.size == 0 or np.issubdtype(flat.dtype, np.integer):
            return flat.astype(np.int64)
        if np.issubdtype(flat.dtype, np.floating):
            with np.errstate(invalid="ignore"):
                ints = flat.astype(np.int64)
            if np.array_equal(ints.astype(flat.dtype), flat):
                return ints
        raise ValueError(f"{who}: {what} must be integers, got {flat.dtype}.")

    @staticmethod
    def _out_of_range(ids, upper):
        """Sorted distinct ids outside [0, upper)."""
        return np.unique(ids[np.logical_or(ids < 0, ids >= upper)]).tolist()

    def _check_nodes(self, node_ids, who):
        set_names = None
        if isinstance(node_ids, str):
            set_names = [node_ids]
        elif isinstance(node_ids, (list, tuple)) and len(node_ids) and all(isinstance(v, str) for v in node_ids):
            set_names = list(node_ids)
        if set_names is not None:
            known = getattr(self.mesh, "node_sets", {})
            unknown = [nm for nm in set_names if nm not in known]
            if unknown:
                raise ValueError(f"{who}: unknown node set(s) {unknown}; available: {sorted(known)}.")
            node_ids = functools.reduce(np.union1d, [np.asarray(known[nm], dtype=np.int64) for nm in set_names])
        nodes = self._as_int_array(node_ids, "node ids", who)
        if nodes.size == 0:
            raise ValueError(f"{who}: no nodes selected (node_ids is empty).")
        n_nodes = len(self.mesh.nodes)
        outside = self._out_of_range(nodes, n_nodes)
        if outside:
            raise ValueError(f"{who}: node id(s) {outside[:5]} outside the mesh (valid range 0..{n_nodes - 1}).")
        return nodes

    def _check_local_dofs(self, dof_indices, who):
        if isinstance(dof_indices, str) or np.ndim(dof_indices) == 0 and not isinstance(dof_indices, (set, frozenset)):
            entries = [dof_indices]
        else:
            entries = list(dof_indices)
        as_index = [self._dof_index_by_name(e, who) if isinstance(e, str) else e for e in entries]
        dofs = self._as_int_array(np.asarray(as_index), "local DOF indices", who)
        if dofs.size == 0:
            raise ValueError(f"{who}: no DOF indices given.")
        outside = self._out_of_range(dofs, self.npn)
        if outside:
            raise ValueError(f"{who}: local DOF index {outside} is out of range -- "
                             f"Hex8Solid3D has 3 DOF(s) per node, so valid indices are 0..2.")
        return dofs

    # ------------------------------------------------------------------ assembly
    def assemble_stiffness(self, D, method="full", vectorized=False, accumulate=False, **kwargs):
        """Element matrices on the GPU (ke = sum_gp B^T D B detJ w thickness), kept packed on
        the device; the reduced CSR is assembled for the current boundary conditions at solve
        time.  ``vectorized`` is accepted for signature compatibility (every path is batched)."""
        if method not in ("full", "reduced", "hourglass_stabilized"):
            raise ValueError(f"assemble_stiffness: unknown method={method!r} -- expected "
                             f"'full' (default), 'reduced', or 'hourglass_stabilized'.")
        if method != "full":
            raise NotImplementedError("assemble_stiffness: only method='full' is implemented on the GPU path")
        gauss_order = kwargs.pop("gauss_order", None)
        thickness = kwargs.pop("thickness", 1.0)
        kwargs.pop("chunk_size", None)
        kwargs.pop("backend", None)
        kwargs.pop("device", None)
        if kwargs:
            raise TypeError(f"assemble_stiffness: unsupported kwargs {list(kwargs)} -- only gauss_order=/thickness=/"
                            f"chunk_size=/backend=/device= are accepted.")
        if gauss_order not in (None, 2):
            raise NotImplementedError("assemble_stiffness: only the full 2x2x2 Gauss rule is implemented")
        if isinstance(D, dict):
            if len(D) != 1:
                raise NotImplementedError("assemble_stiffness: per-block D needs a multi-block mesh")
            D = next(iter(D.values()))
        D = np.asarray(D, dtype=float)
        if D.shape != (6, 6):
            raise ValueError(f"D has shape {D.shape} but Hex8Solid3D's B matrix has 6 strain rows -- "
                             f"mismatched material/element pair.")
        if not np.allclose(D, D.T, rtol=1e-12, atol=0.0):
            raise ValueError("assemble_stiffness: D must be symmetric (the PCG path needs an SPD K)")
        if "K" in self._assembled and not accumulate and "K" not in self._warned_reassembly:
            warnings.warn("assemble_stiffness: K was already assembled, so it is being REPLACED. Pass "
                          "accumulate=True to add to the existing matrix instead.", UserWarning, stacklevel=2)
            self._warned_reassembly.add("K")
        ke = self.device_mesh.element_stiffness(D, thickness=thickness, bbar=is_bbar(self.elem))
        if accumulate and self._ke is not None:
            self._ke = self._ke + ke
        else:
            self._ke = ke
        self._ke_version += 1
        self._op_cache = None
        self._K_full = None
        self._assembled.add("K")
        self._stiffness_args = (D, {"thickness": thickness})

    def assemble_mass(self, rho_or_matrix, accumulate=False, **kwargs):
        """Consistent mass M = sum_e sum_q Nm^T R Nm |detJ| w thickness on the GPU (solver.py:699-740,
        Element.mass, elements/base.py:711-731).  rho_or_matrix: the 3x3 density matrix of a solid
        (rho * np.eye(3)); a scalar raises ValueError, as it does in the reference."""
        thickness = kwargs.pop("thickness", 1.0)
        if kwargs:
            raise TypeError(f"assemble_mass: unsupported kwargs {list(kwargs)}")
        if np.isscalar(rho_or_matrix):
            raise ValueError(
                f"assemble_mass: {type(self.elem).__name__}.mass() could not use the scalar density "
                f"{rho_or_matrix!r}. This element needs a density MATRIX -- for a solid pass rho * np.eye(3).")
        R = np.asarray(rho_or_matrix, dtype=float)
        if R.shape != (3, 3):
            raise ValueError(f"assemble_mass: the density matrix of a hex8 solid is 3x3, got shape {R.shape}")
        if self._me is not None and not accumulate and "M" not in self._warned_reassembly:
            warnings.warn("assemble_mass: M was already assembled, so it is being REPLACED. Pass accumulate=True "
                          "to add to the existing matrix instead.", UserWarning, stacklevel=2)
            self._warned_reassembly.add("M")
        me = self.device_mesh.element_mass(R, thickness=thickness)
        self._me = self._me + me if (accumulate and self._me is not None) else me
        self._me_version += 1
        self._mop_cache = None
        self._M_full = None

    @property
    def M(self):
        """Full (n_dof x n_dof) consistent mass as a host scipy CSR (None before assemble_mass)."""
        if self._me is None:
            return None
        if self._M_full is None:
            dm = self.device_mesh
            self._M_full = dm.assemble(self._me, dm.pattern(()), want32=False).to_scipy()
        return self._M_full

    def reduced_mass_operator(self):
        """M_ff for the current fixed set on the device, on the stiffness pattern."""
        if self._me is None:
            raise RuntimeError("call assemble_mass() first (the mass matrix M has not been assembled)")
        fixed = self._bc_arrays()[2]
        key = (self._me_version, fixed.tobytes())
        if self._mop_cache is not None and self._mop_cache[0] == key:
            return self._mop_cache[1]
        dm = self.device_mesh
        op = dm.assemble(self._me, dm.pattern(fixed), want32=False)
        self._mop_cache = (key, op)
        return op

    def solve_modal(self, n_modes=4, tol=1e-12, maxiter=300, subspace=None, pcg_tol=1e-10):
        """Natural frequencies (Hz) and M-orthonormal mode shapes of the constrained system
        (solver.py:2047-2114).  The reference's shift-invert eigsh is replaced by GPU block
        subspace iteration (feab200.modal).  Returns (freq_hz (n_modes,), FEField (n_dof, n_modes))."""
        if self._me is None:
            raise RuntimeError("call assemble_mass() first (the mass matrix M has not been assembled)")
        self._require_stiffness("this solve")
        from .modal import subspace_iteration
        Kop = self.reduced_operator(want32=False)
        Mop = self.reduced_mass_operator()
        lam, Phi, iters = subspace_iteration(Kop, Mop, int(n_modes), subspace=subspace, tol=tol, maxiter=maxiter,
                                             pcg_tol=pcg_tol)
        self.last_modal_iterations = iters
        lam = lam.clamp_min(0.0)
        modes = torch.zeros((self.n_dof, int(n_modes)), dtype=torch.float64, device=self.device)
        modes[self._bc_device_index()[0]] = Phi
        freq = (lam.sqrt() / (2 * np.pi)).cpu().numpy()
        return freq, self.field(modes.cpu().numpy(), label="mode shapes")

    def _require_stiffness(self, who):
        if self._ke is None:
            raise RuntimeError(f"{who}: the global stiffness matrix K is all zeros -- call "
                               f"assemble_stiffness(...) before solving.")

    # ------------------------------------------------------------------ boundary conditions / loads
    def fix_dofs(self, node_ids, dof_indices, value=0.0):
        nodes = self._check_nodes(node_ids, "fix_dofs")
        dofs = self._check_local_dofs(dof_indices, "fix_dofs")
        # node-major, the same insertion order as one loop over nodes then local DOFs
        ids = (self.npn * nodes.astype(np.int64)[:, None] + dofs.astype(np.int64)[None, :]).reshape(-1).tolist()
        self.fixed_dofs.update(ids)
        self.fixed_dof_values.update(dict.fromkeys(ids, float(value)))

    def add_nodal_force(self, node_ids, dof_index, total_force):
        nodes = self._check_nodes(node_ids, "add_nodal_force")
        dof = int(self._check_local_dofs(dof_index, "add_nodal_force")[0])
        share = total_force / len(nodes)
        for n in nodes:
            self.F[self.npn * int(n) + dof] += share

    def add_consistent_facet_load(self, formulation, facets, dof_index, traction, quad_order=2, thickness=1.0):
        facets = np.asarray([tuple(f) for f in facets], dtype=int)
        if facets.ndim != 2 or facets.shape[1] != 4:
            raise ValueError("add_consistent_facet_load: hex8 facets are 4-node tuples")
        self._check_nodes(facets.reshape(-1), "add_consistent_facet_load")
        dof_index = int(self._check_local_dofs(dof_index, "add_consistent_facet_load")[0])
        shares = facet_load_shares_batch(np.asarray(self.mesh.nodes)[facets], traction * thickness, quad_order)
        np.add.at(self.F, self.npn * facets.reshape(-1) + dof_index, shares.reshape(-1))

    def _bc_arrays(self):
        """(free, fixed) DOF index arrays for the current fixed set, recomputed only when the set
        changes (the set is compared by value, so direct edits of ``fixed_dofs`` are seen)."""
        key = frozenset(self.fixed_dofs)
        c = self._bc_cache
        if c is None or c[0] != key:
            fixed = np.fromiter(key, dtype=np.int64, count=len(key))
            fixed.sort()
            mask = np.ones(self.n_dof, dtype=bool)
            mask[fixed] = False
            c = self._bc_cache = (key, np.flatnonzero(mask), fixed.astype(int), {})
        return c

    def _bc_device_index(self):
        """Device copies of the (free, fixed) index arrays for the current fixed set."""
        c = self._bc_arrays()
        dev = self.device
        if dev not in c[3]:
            c[3][dev] = (torch.as_tensor(c[1]).to(dev), torch.as_tensor(c[2]).to(dev))
        return c[3][dev]

    @property
    def free_dofs(self):
        return self._bc_arrays()[1].copy()

    @property
    def fixed_dofs_array(self):
        return self._bc_arrays()[2].copy()

    def _fixed_dof_values_array(self, fixed):
        vals = self.fixed_dof_values
        return np.fromiter((vals.get(d, 0.0) for d in np.asarray(fixed).tolist()), dtype=float, count=len(fixed))

    # ------------------------------------------------------------------ reduced operator
    def reduced_operator(self, want32=True):
        """K_ff for the current fixed set on the device (cached until K or the BCs change)."""
        self._require_stiffness("reduced_operator")
        fixed = self._bc_arrays()[2]
        key = (self._ke_version, fixed.tobytes(), bool(want32))
        if self._op_cache is not None and self._op_cache[0] == key:
            return self._op_cache[1]
        dm = self.device_mesh
        pat = dm.pattern(fixed)
        op = dm.assemble(self._ke, pat, want32=want32)
        self._op_cache = (key, op)
        return op

    def _reduced_rhs(self, F=None):
        """F_f - K[free, fixed] u_fixed as a device vector (solver.py:1496-1511)."""
        Fv = self.F if F is None else np.asarray(F, dtype=float)
        _, free, fixed, _ = self._bc_arrays()
        u_fixed = self._fixed_dof_values_array(fixed)
        # the whole F goes to the device and is gathered there with the cached free-DOF index
        Ff = torch.as_tensor(np.ascontiguousarray(Fv, dtype=np.float64)).to(self.device)[self._bc_device_index()[0]]
        if fixed.size and np.any(u_fixed):
            v = np.zeros(self.n_dof)
            v[fixed] = u_fixed
            y = self.device_mesh.apply(self._ke, v)
            Ff = Ff - y[self._bc_device_index()[0]]
        return Ff

    @property
    def K(self):
        """Full (n_dof x n_dof) stiffness as a host scipy CSR (structural pattern)."""
        self._require_stiffness("K")
        if self._K_full is None:
            dm = self.device_mesh
            pat = dm.pattern(())
            self._K_full = dm.assemble(self._ke, pat, want32=False).to_scipy()
        return self._K_full

    def field(self, data, label=None):
        if not isinstance(data, np.ndarray) or data.ndim not in (1, 2) or data.shape[0] != self.n_dof:
            return data
        return FEField(data, n_nodes=len(self.mesh.nodes), dofs_per_node=3, dof_names=self.dof_names, label=label,
                       mesh=self.mesh)

    # ------------------------------------------------------------------ derived results (recovery.py)
    def stress(self, U=None, D=None, at="nodes", vectorized=True, backend="numpy", device="cpu"):
        """Stress components as an FEField (``at="elements"``: element averages), solver.py:413-418."""
        from . import recovery
        return recovery.stress(self, self.solve_static() if U is None else U, D, at, vectorized, backend, device)

    def strain(self, U=None, at="nodes", vectorized=True, backend="numpy", device="cpu"):
        """Strain components (engineering shear), solver.py:420-423."""
        from . import recovery
        return recovery.strain(self, self.solve_static() if U is None else U, at, vectorized, backend, device)

    def von_mises(self, U=None, D=None, plane="stress", nu=None, at="nodes", vectorized=True, backend="numpy",
                  device="cpu"):
        """Von Mises stress as a scalar FEField, solver.py:425-430."""
        from . import recovery
        return recovery.von_mises(self, self.solve_static() if U is None else U, D, plane, nu, at, vectorized,
                                  backend, device)

    def stress_tensor(self, U, D=None, device="cpu", at="nodes"):
        from . import recovery
        return recovery.stress_tensor(self, U, D, device, at)

    def von_mises_tensor(self, U, D=None, device="cpu", plane="stress", nu=None, at="nodes"):
        from . import recovery
        return recovery.von_mises_tensor(self, U, D, device, plane, nu, at)

    def reactions(self, U=None):
        """Support reactions K U - F at the constrained DOFs, solver.py:442-445."""
        from . import recovery
        return recovery.reactions(self, U)

    # ------------------------------------------------------------------ solve
    def solve_static(self, verbose=False, method=None, **method_kwargs):
        U = self.solve_static_device(verbose=verbose, method=method, **method_kwargs)
        return self.field(U.cpu().numpy(), label="displacement")

    def solve_static_device(self, verbose=False, method=None, **method_kwargs):
        """solve_static, returning the full displacement vector as a device tensor."""
        self._require_stiffness("solve_static")
        fixed = self._bc_arrays()[2]
        u_fixed = self._fixed_dof_values_array(fixed)
        if not np.any(self.F) and not np.any(u_fixed):
            warnings.warn("solve_static: the load vector F is all zeros and no non-zero displacement is "
                          "prescribed, so the solution is trivially zero.", UserWarning, stacklevel=3)
        if method not in (None, "cg", "pcg"):
            raise ValueError(f"solve_static: unknown method={method!r} -- choose from 'cg', 'pcg' (or None).")
        kw = dict(method_kwargs)
        precision = kw.pop("precision", "fp64")
        delta = kw.pop("reliable_delta", 0.1)
        precond = kw.pop("preconditioner", "jacobi")
        kw.pop("omega", None)
        if method == "pcg" and precond != "jacobi":
            if precond in ("ssor", "ic0"):
                raise NotImplementedError(f"solve_static(method='pcg', preconditioner={precond!r}): only 'jacobi' "
                                          f"is implemented on the GPU path")
            raise ValueError(f"solve_static(method='pcg'): unknown preconditioner={precond!r} -- choose 'jacobi', "
                             f"'ssor', or 'ic0'.")
        tol = kw.pop("tol", 1e-12 if method is None else 1e-8)
        maxiter = kw.pop("maxiter", None)
        x0 = kw.pop("x0", None)
        if kw:
            raise TypeError(f"solve_static: unsupported keyword(s) {sorted(kw)}")
        t0 = time.perf_counter()
        op = self.reduced_operator(want32=(precision == "fp32"))
        Ff = self._reduced_rhs()
        x = None
        if method is None and precision == "fp64" and x0 is None:
            x, info = self._direct_solve(op, Ff, tol, maxiter)
        if x is None:
            x, info = pcg_solve(op, Ff, x0=x0, tol=tol, maxiter=maxiter, precision=precision,
                                use_dinv=(method != "cg"), reliable_delta=delta)
        self.last_solve_info = info
        if info.status == L.FEAB_NOT_SPD:
            raise np.linalg.LinAlgError("preconditioned_cg: p^T A p <= 0 -- A is not SPD.")
        if info.status == L.FEAB_NOT_CONVERGED:
            raise RuntimeError(f"preconditioned_cg: did not converge in {info.iters} iterations "
                               f"(final relative residual {info.relres:.3e} >= tol={tol:.1e}).")
        L.raise_for(info.status, "solve_static")
        U = torch.zeros(self.n_dof, dtype=torch.float64, device=self.device)
        free_t, fixed_t = self._bc_device_index()
        U[free_t] = x
        if fixed.size and np.any(u_fixed):
            U[fixed_t] = torch.as_tensor(u_fixed).to(self.device)
        if verbose:
            print(f"[feab200] n={op.n} nnz={op.nnz} precision={precision} iters={info.iters} "
                  f"relres={info.relres:.3e} reliable_updates={info.reliable_updates} "
                  f"time={time.perf_counter() - t0:.3f}s")
        return U

    def _direct_solve(self, op, Ff, tol, maxiter):
        """The sparse direct solve of method=None (_sparse_lu_solve, solver.py:1681-1724) as a
        banded Cholesky on the GPU: (x, SolveInfo), or (None, None) when the band does not fit in
        device memory (the Jacobi-PCG then takes over).

        When the factor's pivots show a singular K_ff (min < 1e-10 max, the reference's test), the
        reference solves densely by eigenvalues (_eigen_solve, solver.py:1584-1679) for the
        minimum-norm least-squares answer pinv(K_ff) F.  Here the null space of K_ff is formed from
        the mesh's rigid-body motions that vanish on the fixed DOFs; it is projected out of the
        load, the consistent system is solved by Jacobi-PCG from x0 = 0, and it is projected out of
        the result, which gives pinv(K_ff) F for a connected body."""
        from .device import SolveInfo, pcg_solve, spmv
        try:
            fac = op.direct_factor(coords=self.mesh.nodes)
        except MemoryError as e:
            warnings.warn(f"solve_static: {e}; solving with Jacobi-PCG to tol {tol:g} instead.", UserWarning,
                          stacklevel=4)
            return None, None
        except np.linalg.LinAlgError:
            fac = None
        b = torch.as_tensor(Ff, dtype=torch.float64).to(op.vals64.device)
        if fac is None or fac.near_singular:
            warnings.warn("solve_static: K_ff is singular to working precision (a pivot of its factorisation "
                          "is below 1e-10 of the largest, e.g. a floating structure); returning the minimum-norm "
                          "least-squares solution (rigid-body null space projected out, Jacobi-PCG on the rest).",
                          UserWarning, stacklevel=4)
            Z = self._rigid_null_space(op.vals64.device)
            if Z is not None:
                b = b - Z @ (Z.T @ b)
            x, info = pcg_solve(op, b, tol=tol, maxiter=maxiter, precision="fp64")
            if Z is not None:
                x = x - Z @ (Z.T @ x)
            return x, info
        x = fac.solve(b)
        bn = float(torch.linalg.norm(b)) or 1.0
        rel = float(torch.linalg.norm(b - spmv(op, x, lanes_per_group=16))) / bn
        return x, SolveInfo(L.FEAB_OK, 0, 0, rel, bn, "direct")

    def _rigid_null_space(self, device):
        """Orthonormal basis (n_free x k, k <= 6) of the rigid-body motions of the mesh (three
        translations, three rotations about the centroid) that vanish on the fixed DOFs,
        restricted to the free DOFs; None when no such motion exists."""
        X = np.asarray(self.mesh.nodes, dtype=float)
        c = X - X.mean(0)
        R = np.zeros((3 * len(X), 6))
        for k in range(3):
            R[k::3, k] = 1.0
        R[0::3, 3], R[1::3, 3] = -c[:, 1], c[:, 0]
        R[1::3, 4], R[2::3, 4] = -c[:, 2], c[:, 1]
        R[0::3, 5], R[2::3, 5] = c[:, 2], -c[:, 0]
        fixed, free = self.fixed_dofs_array, self.free_dofs
        N = np.eye(6)
        if fixed.size:
            _, sv, vt = np.linalg.svd(R[fixed], full_matrices=True)
            rank = int(np.sum(sv > 1e-10 * max(sv.max(), 1e-300)))
            N = vt[rank:].T
        if N.shape[1] == 0:
            return None
        Q, _ = np.linalg.qr(R[free] @ N)
        return torch.as_tensor(Q).to(device)

    def form_linear_system(self, F=None, K=None):
        from .linear_system import ReducedSystem
        if K is not None:
            raise NotImplementedError("form_linear_system: a caller-supplied K is not supported on the GPU path")
        self._require_stiffness("form_linear_system")
        Fv = self.F if F is None else np.asarray(F, dtype=float)
        if Fv.shape != (self.n_dof,):
            raise ValueError(f"F must have shape ({self.n_dof},), got {Fv.shape}")
        fixed = self.fixed_dofs_array
        op = self.reduced_operator()
        Ff = self._reduced_rhs(Fv)
        return ReducedSystem(operator=op, F_device=Ff, free=self.free_dofs, fixed=fixed,
                             u_fixed=self._fixed_dof_values_array(fixed), n_dof=self.n_dof, _system=self)
