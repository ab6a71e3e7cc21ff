"""GPU-resident hex8 mesh, reduced stiffness operator and PCG, on top of libfeab200.

Everything here keeps its arrays in device memory (torch tensors used as plain buffers) and
calls the C ABI in ``_lib``.  The public, reference-shaped API (``FESystem`` and friends) is
built on these pieces.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


def cuda_device(device=None):
    """Resolve the CUDA device to run on.  The reference's default ``device="cpu"`` selects the
    current CUDA device: this library has no CPU compute path."""
    if not torch.cuda.is_available():
        raise RuntimeError("feab200: no CUDA device is available (the library has no CPU fallback)")
    if device is None or (isinstance(device, str) and device in ("cpu", "cuda")):
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError(f"feab200 runs on CUDA devices only, got device={device!r}")
    return d if d.index is not None else torch.device("cuda", torch.cuda.current_device())


class DeviceStatus:
    """A feab_device_status in device memory (first device-side failure + its index)."""

    def __init__(self, device):
        self.t = torch.zeros(2, dtype=torch.int64, device=device)

    def ptr(self):
        return L.dptr(self.t)

    def check(self, what):
        v = self.t.cpu().numpy()
        code = int(v[0]) & 0xFFFFFFFF
        if code:
            L.raise_for(code, what, v[1])

    def reset(self):
        self.t.zero_()


@dataclass
class Topology:
    inc_ptr: torch.Tensor      # (N+1,) int32: node -> incident elements, sorted
    inc_elem: torch.Tensor     # (8E,) int32
    nbr_ptr: torch.Tensor      # (N+1,) int32: node -> sorted neighbour nodes
    nbr_idx: torch.Tensor
    max_elems: int
    max_nbrs: int


@dataclass
class Pattern:
    n: int
    nnz: int
    n_groups: int
    row_ptr: torch.Tensor      # (n+1,) int32
    col_idx: torch.Tensor      # (nnz,) int32
    group_ptr: torch.Tensor    # (n_groups+1,) int32
    free_map: torch.Tensor     # (3N,) int32, -1 = fixed


@dataclass
class ReducedOperator:
    """K_ff in CSR on the device with its FP32 copy, Jacobi inverse diagonals and (built on
    first use by the mixed-precision solver) the difference-form operator."""
    pattern: Pattern
    vals64: torch.Tensor
    vals32: torch.Tensor | None
    dinv64: torch.Tensor
    dinv32: torch.Tensor | None
    _diff: object = None
    _sell: dict = None
    _tiles: dict = None
    _direct: object = None   # banded Cholesky factor (direct.BandCholesky), built on first direct solve

    def direct_factor(self, coords=None):
        """The banded Cholesky factor of K_ff (direct.BandCholesky; coords: the mesh's node
        coordinates, for the ordering along the longest axis), cached."""
        if self._direct is None:
            from .direct import BandCholesky
            self._direct = BandCholesky(self, coords=coords)
        return self._direct

    def diff_operator(self):
        """The difference-form operator of the mixed block-PCG (7-byte values, 44-bit mantissas;
        feab_diff_operator_build), cached."""
        if self._diff is None:
            p = self.pattern
            if p.group_ptr is None or p.free_map.numel() == 0:
                raise ValueError("the mixed-precision operator needs node row groups (an assembled K_ff)")
            dev = self.vals64.device
            dof_of = torch.nonzero(p.free_map >= 0).flatten().to(torch.int32)
            nbytes = int(L.lib.feab_diff_operator_bytes(p.n, p.nnz, p.n_groups))
            storage = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            d = L.DiffOperator()
            csr = self.csr_struct()
            rc = L.lib.feab_diff_operator_build(C.byref(csr), L.dptr(dof_of), L.dptr(storage), nbytes, C.byref(d),
                                                L.stream_ptr(dev))
            L.raise_for(rc, "difference-form operator")
            self._diff = (storage, d)
        return self._diff[1]

    def tile_operator(self, precision="fp64", problem_groups=None):
        """Node tiles of the block SpMM (feab_tile_operator_build): FEAB_TILE_GROUPS consecutive
        row groups whose column lists are merged, with "fp64" (CSR) or "mixed" (difference-form,
        44-bit) values.  Tiles never cross the boundaries in problem_groups (the first row group
        of each problem, then n_groups; default one problem).  Cached per (precision, boundaries)."""
        if precision not in ("fp64", "mixed"):
            raise ValueError("the tile operator holds 'fp64' or 'mixed' values")
        p = self.pattern
        if p.group_ptr is None:
            raise ValueError("the tile operator needs node row groups (an assembled K_ff)")
        pg = np.asarray([0, p.n_groups] if problem_groups is None else problem_groups, dtype=np.int32)
        key = (precision, pg.tobytes())
        if self._tiles is None:
            self._tiles = {}
        if key not in self._tiles:
            dev = self.vals64.device
            pg_t = torch.as_tensor(pg).to(dev)
            n_prob = len(pg) - 1
            diff = C.byref(self.diff_operator()) if precision == "mixed" else None
            sbytes = int(L.lib.feab_tile_scratch_bytes(p.n_groups, n_prob))
            scratch = torch.empty(max(sbytes, 1), dtype=torch.uint8, device=dev)
            csr = self.csr_struct()
            need = C.c_size_t(0)
            args = (C.byref(csr), diff, L.dptr(pg_t), n_prob, PRECISIONS[precision], L.dptr(scratch), sbytes)
            L.raise_for(L.lib.feab_tile_operator_build(*args, None, 0, C.byref(need), None, L.stream_ptr(dev)),
                        "tile operator")
            storage = torch.empty(need.value, dtype=torch.uint8, device=dev)
            t = L.TileOperator()
            L.raise_for(L.lib.feab_tile_operator_build(*args, L.dptr(storage), need.value, None, C.byref(t),
                                                       L.stream_ptr(dev)), "tile operator")
            self._tiles[key] = (storage, t)
        return self._tiles[key][1]

    def max_row_len(self):
        rp = self.pattern.row_ptr
        return int((rp[1:] - rp[:-1]).max().item()) if self.pattern.n > 0 else 0

    def sell_operator(self, precision="fp64"):
        """The sliced (SELL-32) node-group operator (feab_sell_operator_build) for "fp64"
        (plain FP64 values) or "mixed" (48-bit values, difference form), cached."""
        if precision not in ("fp64", "mixed"):
            raise ValueError("the sliced operator holds 'fp64' or 'mixed' values")
        if self._sell is None:
            self._sell = {}
        if precision not in self._sell:
            p = self.pattern
            if p.group_ptr is None or p.free_map.numel() == 0:
                raise ValueError("the sliced operator needs node row groups (an assembled K_ff)")
            dev = self.vals64.device
            kind = PRECISIONS[precision]
            mrl = self.max_row_len()
            dof_of = torch.nonzero(p.free_map >= 0).flatten().to(torch.int32) if precision == "mixed" else None
            nbytes = int(L.lib.feab_sell_operator_bytes(p.n, p.n_groups, mrl, kind))
            storage = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            d = L.SellOperator()
            csr = self.csr_struct()
            rc = L.lib.feab_sell_operator_build(C.byref(csr), L.dptr(dof_of), kind, mrl, L.dptr(storage), nbytes,
                                                C.byref(d), L.stream_ptr(dev))
            L.raise_for(rc, "sliced operator")
            self._sell[precision] = (storage, d, dof_of)
        return self._sell[precision][1]

    @property
    def n(self):
        return self.pattern.n

    @property
    def nnz(self):
        return self.pattern.nnz

    def csr_struct(self):
        p = self.pattern
        return L.CSR(p.n, p.n_groups, p.nnz, p.row_ptr.data_ptr(), p.col_idx.data_ptr(), self.vals64.data_ptr(),
                     self.vals32.data_ptr() if self.vals32 is not None else None, p.group_ptr.data_ptr())

    def to_scipy(self):
        """Host scipy.sparse.csr_matrix copy (int32 indices, like SciPy's own)."""
        import scipy.sparse as sp
        p = self.pattern
        return sp.csr_matrix((self.vals64.cpu().numpy(), p.col_idx.cpu().numpy(), p.row_ptr.cpu().numpy()),
                             shape=(p.n, p.n))


class DeviceMesh:
    """Hex8 mesh resident on one GPU: coordinates (N, 3) FP64, connectivity (E, 8) int32."""

    def __init__(self, nodes, elements, device=None):
        self.device = cuda_device(device)
        if torch.is_tensor(nodes):
            coords = nodes.to(device=self.device, dtype=torch.float64).contiguous()
        else:
            coords = torch.as_tensor(np.ascontiguousarray(nodes, dtype=np.float64)).to(self.device)
        if torch.is_tensor(elements):
            conn = elements.to(device=self.device, dtype=torch.int32).contiguous()
        else:
            # copied as given and range-checked / narrowed to int32 on the device (no host passes)
            arr = np.ascontiguousarray(elements)
            if arr.dtype.kind == "u":          # unsigned ids: torch has no general uint64 tensors
                arr = arr.astype(np.int64)
            el = torch.as_tensor(arr).to(self.device)
            if el.dtype.is_floating_point or el.dtype == torch.bool:
                el = el.to(torch.int64)
            if el.numel():
                lo, hi = torch.stack(torch.aminmax(el)).cpu().tolist()   # one read-back
                if lo < 0 or hi >= coords.shape[0]:
                    raise ValueError("element connectivity refers to node ids outside the mesh")
            conn = el.to(torch.int32).contiguous()
        if coords.ndim != 2 or coords.shape[1] != 3:
            raise ValueError(f"hex8 solid mesh needs (n_nodes, 3) coordinates, got {tuple(coords.shape)}")
        if conn.ndim != 2 or conn.shape[1] != 8:
            raise ValueError(f"hex8 connectivity must be (n_elements, 8), got {tuple(conn.shape)}")
        self.coords = coords
        self.conn = conn
        self.n_nodes = int(coords.shape[0])
        self.n_elem = int(conn.shape[0])
        self._topo = None
        self._patterns = {}

    @property
    def stream(self):
        return L.stream_ptr(self.device)

    # ------------------------------------------------------------------ topology
    def topology(self) -> Topology:
        if self._topo is not None:
            return self._topo
        dev, N, E = self.device, self.n_nodes, self.n_elem
        sbytes = int(L.lib.feab_topology_scratch_bytes(N, E))
        scratch = torch.empty(sbytes, dtype=torch.uint8, device=dev)
        st = DeviceStatus(dev)
        inc_ptr = torch.empty(N + 1, dtype=torch.int32, device=dev)
        inc_elem = torch.empty(max(8 * E, 1), dtype=torch.int32, device=dev)
        mx = C.c_int32(0)
        rc = L.lib.feab_node_incidence(L.dptr(self.conn), E, N, L.dptr(inc_ptr), L.dptr(inc_elem), L.dptr(scratch),
                                       sbytes, st.ptr(), C.byref(mx), self.stream)
        st.check("node incidence")
        L.raise_for(rc, "node incidence")
        nbr_ptr = torch.empty(N + 1, dtype=torch.int32, device=dev)
        tot, mxn = C.c_int64(0), C.c_int32(0)
        rc = L.lib.feab_node_adjacency(L.dptr(self.conn), L.dptr(inc_ptr), L.dptr(inc_elem), N, L.dptr(nbr_ptr), None,
                                       L.dptr(scratch), sbytes, st.ptr(), C.byref(tot), C.byref(mxn), self.stream)
        st.check("node adjacency")
        L.raise_for(rc, "node adjacency")
        nbr_idx = torch.empty(max(int(tot.value), 1), dtype=torch.int32, device=dev)
        rc = L.lib.feab_node_adjacency(L.dptr(self.conn), L.dptr(inc_ptr), L.dptr(inc_elem), N, L.dptr(nbr_ptr),
                                       L.dptr(nbr_idx), L.dptr(scratch), sbytes, st.ptr(), None, None, self.stream)
        L.raise_for(rc, "node adjacency")
        self._topo = Topology(inc_ptr, inc_elem, nbr_ptr, nbr_idx, int(mx.value), int(mxn.value))
        return self._topo

    # ------------------------------------------------------------------ pattern
    def free_map(self, fixed_dofs):
        """int32 map DOF -> reduced row (-1 fixed); free rows numbered in increasing DOF order
        (free_dofs, fea_engine/src/fea_engine/solver.py:1400-1401)."""
        n_dof = 3 * self.n_nodes
        mask = np.ones(n_dof, dtype=bool)
        fixed = np.asarray(fixed_dofs, dtype=np.int64).reshape(-1)
        if fixed.size:
            if fixed.min() < 0 or fixed.max() >= n_dof:
                raise ValueError("fixed DOF index outside the system")
            mask[fixed] = False
        fm = np.full(n_dof, -1, dtype=np.int32)
        fm[mask] = np.arange(int(mask.sum()), dtype=np.int32)
        return fm

    def _fixed_set(self, fixed_dofs):
        """The fixed DOFs as a sorted, duplicate-free int64 array (range-checked)."""
        fixed = np.unique(np.asarray(fixed_dofs, dtype=np.int64).reshape(-1))
        if fixed.size and (fixed[0] < 0 or fixed[-1] >= 3 * self.n_nodes):
            raise ValueError("fixed DOF index outside the system")
        return fixed

    def pattern(self, fixed_dofs=()) -> Pattern:
        # the free map is a function of the fixed-DOF set alone: the set is the cache key, and the
        # map is built on the device (no host pass over all DOFs)
        fixed = self._fixed_set(fixed_dofs)
        key = fixed.tobytes()
        hit = self._patterns.get(key)
        if hit is not None:
            return hit
        topo = self.topology()
        dev, N = self.device, self.n_nodes
        n_free = 3 * N - int(fixed.size)
        if n_free == 0:
            raise ValueError("every DOF is fixed: the reduced system is empty")
        keep = torch.ones(3 * N, dtype=torch.int32, device=dev)
        if fixed.size:
            keep[torch.as_tensor(fixed).to(dev)] = 0
        free_map = torch.where(keep > 0, torch.cumsum(keep, 0, dtype=torch.int32) - 1, -1).to(torch.int32)
        sbytes = int(L.lib.feab_topology_scratch_bytes(N, self.n_elem))
        scratch = torch.empty(sbytes, dtype=torch.uint8, device=dev)
        row_ptr = torch.empty(n_free + 1, dtype=torch.int32, device=dev)
        group_ptr = torch.empty(n_free + 1, dtype=torch.int32, device=dev)
        nnz, ng = C.c_int64(0), C.c_int32(0)
        rc = L.lib.feab_csr_pattern(L.dptr(topo.nbr_ptr), L.dptr(topo.nbr_idx), N, L.dptr(free_map), n_free,
                                    L.dptr(row_ptr), L.dptr(group_ptr), None, L.dptr(scratch), sbytes, C.byref(nnz),
                                    C.byref(ng), self.stream)
        L.raise_for(rc, "CSR pattern")
        col_idx = torch.empty(max(int(nnz.value), 1), dtype=torch.int32, device=dev)
        rc = L.lib.feab_csr_pattern(L.dptr(topo.nbr_ptr), L.dptr(topo.nbr_idx), N, L.dptr(free_map), n_free,
                                    L.dptr(row_ptr), None, L.dptr(col_idx), L.dptr(scratch), sbytes, None, None,
                                    self.stream)
        L.raise_for(rc, "CSR pattern")
        pat = Pattern(n_free, int(nnz.value), int(ng.value), row_ptr, col_idx[: int(nnz.value)],
                      group_ptr[: int(ng.value) + 1], free_map)
        self._patterns[key] = pat
        return pat

    # ------------------------------------------------------------------ element matrices
    def element_stiffness(self, D, scale=None, thickness=1.0, layout=L.KE_PACKED, status=None, bbar=False):
        """Element stiffness matrices, (E, 324) packed upper node blocks or (E, 24, 24); with
        bbar=True those of Hex8SolidBbar (mean-dilatation B-bar)."""
        st = status or DeviceStatus(self.device)
        width = L.KE_PACKED if layout == L.KE_PACKED else L.KE_FULL
        ke = torch.empty((self.n_elem, width), dtype=torch.float64, device=self.device)
        sc = None
        if scale is not None:
            sc = torch.as_tensor(scale, dtype=torch.float64).to(self.device).contiguous()
            if sc.shape != (self.n_elem,):
                raise ValueError(f"scale must have shape ({self.n_elem},)")
        fn = L.lib.feab_hex8_bbar_element_stiffness if bbar else L.lib.feab_hex8_element_stiffness
        rc = fn(L.dptr(self.coords), L.dptr(self.conn), self.n_elem, L.dmat(D), L.dptr(sc), float(thickness),
                L.dptr(ke), width, st.ptr(), self.stream)
        L.raise_for(rc, "hex8 element stiffness")
        if status is None:
            st.check("hex8 element stiffness")
        return ke if width == L.KE_PACKED else ke.view(self.n_elem, 24, 24)

    def element_mass(self, R, scale=None, thickness=1.0, layout=L.KE_PACKED, status=None):
        """Consistent element mass matrices for the 3x3 density matrix R (e.g. rho * I), in the
        layouts of element_stiffness (Element.mass, elements/base.py:711-731)."""
        R = np.asarray(R, dtype=float)
        if R.shape != (3, 3):
            raise ValueError(f"the density matrix of a hex8 solid must be 3x3, got shape {R.shape}")
        if not np.array_equal(R, R.T):
            raise ValueError("the density matrix must be symmetric")
        st = status or DeviceStatus(self.device)
        width = L.KE_PACKED if layout == L.KE_PACKED else L.KE_FULL
        me = torch.empty((self.n_elem, width), dtype=torch.float64, device=self.device)
        sc = None
        if scale is not None:
            sc = torch.as_tensor(scale, dtype=torch.float64).to(self.device).contiguous()
        Rh = (C.c_double * 9)(*R.reshape(9).tolist())
        rc = L.lib.feab_hex8_element_mass(L.dptr(self.coords), L.dptr(self.conn), self.n_elem, Rh, L.dptr(sc),
                                          float(thickness), L.dptr(me), width, st.ptr(), self.stream)
        L.raise_for(rc, "hex8 element mass")
        if status is None:
            st.check("hex8 element mass")
        return me if width == L.KE_PACKED else me.view(self.n_elem, 24, 24)

    def assemble(self, ke_packed, pattern: Pattern, want32=True, status=None) -> ReducedOperator:
        topo = self.topology()
        dev = self.device
        st = status or DeviceStatus(dev)
        vals64 = torch.empty(max(pattern.nnz, 1), dtype=torch.float64, device=dev)
        vals32 = torch.empty(max(pattern.nnz, 1), dtype=torch.float32, device=dev) if want32 else None
        dinv64 = torch.empty(pattern.n, dtype=torch.float64, device=dev)
        dinv32 = torch.empty(pattern.n, dtype=torch.float32, device=dev) if want32 else None
        rc = L.lib.feab_assemble_csr(L.dptr(ke_packed), L.dptr(self.conn), L.dptr(topo.inc_ptr), L.dptr(topo.inc_elem),
                                     L.dptr(topo.nbr_ptr), L.dptr(topo.nbr_idx), self.n_nodes, max(topo.max_nbrs, 1),
                                     L.dptr(pattern.free_map), L.dptr(pattern.row_ptr), L.dptr(vals64),
                                     L.dptr(vals32), L.dptr(dinv64), L.dptr(dinv32), st.ptr(), self.stream)
        L.raise_for(rc, "CSR assembly")
        if status is None:
            st.check("CSR assembly")
        return ReducedOperator(pattern, vals64[: pattern.nnz], vals32[: pattern.nnz] if want32 else None, dinv64,
                               dinv32)

    def apply(self, ke_packed, v):
        """y = K v over all DOFs (element by element)."""
        topo = self.topology()
        v = torch.as_tensor(v, dtype=torch.float64).to(self.device).contiguous()
        y = torch.empty(3 * self.n_nodes, dtype=torch.float64, device=self.device)
        rc = L.lib.feab_hex8_apply(L.dptr(ke_packed), L.dptr(self.conn), L.dptr(topo.inc_ptr), L.dptr(topo.inc_elem),
                                   self.n_nodes, L.dptr(v), L.dptr(y), self.stream)
        L.raise_for(rc, "hex8 apply")
        return y

    def recover(self, u, D=None, nodal=True, elements=False, von_mises=False, status=None):
        """Strain (D is None) or stress (D given) recovered from the full displacement vector u
        (3 n_nodes) by the lumped L2 projection of the Gauss-point values to the nodes
        (recovery.py:196-334).  Returns a dict of device tensors: "nodal" (n_nodes, 6),
        "elements" (n_elem, 6), and with von_mises (stress only) "nodal_vm" (n_nodes,) and
        "elements_vm" (n_elem,), for the parts asked for."""
        if von_mises and D is None:
            raise ValueError("von Mises recovery needs the constitutive matrix D")
        topo = self.topology()
        dev = self.device
        st = status or DeviceStatus(dev)
        u = torch.as_tensor(u, dtype=torch.float64).to(dev).contiguous()
        if u.shape != (3 * self.n_nodes,):
            raise ValueError(f"expected a displacement vector of length {3 * self.n_nodes}, got {tuple(u.shape)}")
        out = {}
        f64 = dict(dtype=torch.float64, device=dev)
        if nodal:
            out["nodal"] = torch.empty((self.n_nodes, 6), **f64)
        if elements:
            out["elements"] = torch.empty((self.n_elem, 6), **f64)
        if von_mises and nodal:
            out["nodal_vm"] = torch.empty(self.n_nodes, **f64)
        if von_mises and elements:
            out["elements_vm"] = torch.empty(self.n_elem, **f64)
        sbytes = int(L.lib.feab_hex8_recover_scratch_bytes(self.n_elem))
        scratch = torch.empty(max(sbytes, 1), dtype=torch.uint8, device=dev)
        rc = L.lib.feab_hex8_recover(L.dptr(self.coords), L.dptr(self.conn), self.n_elem, self.n_nodes,
                                     L.dptr(topo.inc_ptr), L.dptr(topo.inc_elem),
                                     None if D is None else L.dmat(D), L.dptr(u), L.dptr(out.get("nodal")),
                                     L.dptr(out.get("nodal_vm")), L.dptr(out.get("elements")),
                                     L.dptr(out.get("elements_vm")), L.dptr(scratch), sbytes, st.ptr(), self.stream)
        L.raise_for(rc, "strain/stress recovery")
        if status is None:
            st.check("strain/stress recovery")
        return out

    def simp_vjp(self, D_unit, rho, penal, rho_min, u, lam=None, status=None):
        """-p (1-rho_min) rho^(p-1) lam_e^T K0_e u_e per element (lam = u: dC/drho)."""
        st = status or DeviceStatus(self.device)
        rho = torch.as_tensor(rho, dtype=torch.float64).to(self.device).contiguous()
        u = torch.as_tensor(u, dtype=torch.float64).to(self.device).contiguous()
        lam = u if lam is None else torch.as_tensor(lam, dtype=torch.float64).to(self.device).contiguous()
        out = torch.empty(self.n_elem, dtype=torch.float64, device=self.device)
        rc = L.lib.feab_hex8_simp_vjp(L.dptr(self.coords), L.dptr(self.conn), self.n_elem, L.dmat(D_unit), L.dptr(rho),
                                      float(penal), float(rho_min), L.dptr(u), L.dptr(lam), L.dptr(out), st.ptr(),
                                      self.stream)
        L.raise_for(rc, "SIMP sensitivity")
        if status is None:
            st.check("SIMP sensitivity")
        return out


@dataclass
class SolveInfo:
    status: int
    iters: int
    reliable_updates: int
    relres: float
    bnorm: float
    precision: str
    graph_launches: int = 0


PRECISIONS = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED, "fp32": L.PREC_FP32}


LANES_PER_GROUP = (4, 8, 16, 32)
_tuned = {}


def tuned_lanes_per_group(op: ReducedOperator, precision="fp64", iters=24, b=None):
    """CSR SpMV launch shape picked by timing: lanes per node row group in (4, 8, 16, 32), i.e.
    how many node groups each warp keeps in flight.  Each candidate runs `iters` iterations of
    the CSR-layout PCG itself (the fused step kernels, not a bare SpMV), timed with CUDA events
    on the current stream; the fastest is cached for the process per (n, nnz, groups,
    precision, device)."""
    key = (op.n, op.nnz, op.pattern.n_groups, precision, op.vals64.device.index)
    hit = _tuned.get(key)
    if hit is not None:
        return hit
    dev = op.vals64.device
    rhs = torch.ones(op.n, dtype=torch.float64, device=dev) if b is None else b
    best, best_t = 16, float("inf")
    for lpg in LANES_PER_GROUP:
        pcg_solve(op, rhs, tol=0.0, maxiter=4, precision=precision, lanes_per_group=lpg, layout="csr")   # load
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        pcg_solve(op, rhs, tol=0.0, maxiter=iters, precision=precision, lanes_per_group=lpg, chunk=8, layout="csr")
        e.record()
        e.synchronize()
        t = a.elapsed_time(e)
        if t < best_t:
            best, best_t = lpg, t
    _tuned[key] = best
    return best


LAYOUTS = ("sell", "csr")


def pcg_solve(op: ReducedOperator, b, x0=None, tol=1e-8, maxiter=None, precision="fp64", use_dinv=True,
              reliable_delta=0.1, chunk=16, out=None, workspace=None, lanes_per_group=None, layout="sell"):
    """Jacobi-PCG on the device.  Returns (x, SolveInfo); the caller decides how to treat a
    non-OK status (see ``raise_for``).  ``layout`` picks the SpMV operator for "fp64": the
    sliced SELL-32 copy of K ("sell", built on first use; a K without node row groups, such as
    a host SciPy matrix, falls back to its CSR) or the CSR itself ("csr"); "mixed" always runs
    on its sliced 48-bit difference-form operator and "fp32" on the CSR."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {precision!r}")
    prec = PRECISIONS[precision]
    dev = op.vals64.device
    n = op.n
    b = torch.as_tensor(b, dtype=torch.float64).to(dev).contiguous()
    if b.shape != (n,):
        raise ValueError(f"b must have shape ({n},), got {tuple(b.shape)}")
    if x0 is not None:
        x0 = torch.as_tensor(x0, dtype=torch.float64).to(dev).contiguous()
        if x0.shape != (n,):
            raise ValueError(f"x0 must have shape ({n},)")
    x = out if out is not None else torch.empty(n, dtype=torch.float64, device=dev)
    wbytes = int(L.lib.feab_pcg_workspace_bytes(n, prec))
    if workspace is None or workspace.numel() < wbytes:
        workspace = torch.empty(wbytes, dtype=torch.uint8, device=dev)
    if precision == "fp32" and op.vals32 is None:
        raise ValueError("fp32 precision needs the FP32 copy of K (assemble with want32=True)")
    if layout not in LAYOUTS:
        raise ValueError(f"layout must be one of {LAYOUTS}, got {layout!r}")
    grouped = op.pattern.group_ptr is not None and op.pattern.free_map.numel() > 0
    use_sell = precision == "mixed" or (precision == "fp64" and layout == "sell" and grouped)
    sell = C.byref(op.sell_operator(precision)) if use_sell else None
    csr = op.csr_struct()
    if lanes_per_group is None:
        lanes_per_group = 8 if use_sell else tuned_lanes_per_group(op, precision)
    params = L.PcgParams(float(tol), int(maxiter or 0), prec, float(reliable_delta), int(chunk), 1 if use_dinv else 0,
                         int(lanes_per_group), 0)
    res = L.PcgResult()
    rc = L.lib.feab_pcg_solve(C.byref(csr), sell, L.dptr(op.dinv64), L.dptr(op.dinv32), L.dptr(b), L.dptr(x0), L.dptr(x),
                              C.byref(params), L.dptr(workspace), wbytes, C.byref(res), L.stream_ptr(dev))
    if rc in (L.FEAB_BAD_ARG, L.FEAB_CUDA_ERROR) and res.status == 0:
        res.status = rc
    return x, SolveInfo(int(res.status), int(res.iters), int(res.reliable_updates), float(res.relres),
                        float(res.bnorm), precision, int(res.graph_launches))


def sell_spmv(op: ReducedOperator, x, precision="fp64", out=None):
    """y = K_ff x through the sliced operator ("fp64" or "mixed" values)."""
    x = torch.as_tensor(x).to(device=op.vals64.device, dtype=torch.float64).contiguous()
    y = out if out is not None else torch.empty(op.n, dtype=torch.float64, device=op.vals64.device)
    sell = op.sell_operator(precision)
    csr = op.csr_struct()
    rc = L.lib.feab_sell_spmv(C.byref(csr), C.byref(sell), L.dptr(x), L.dptr(y), L.stream_ptr(op.vals64.device))
    L.raise_for(rc, "sliced spmv")
    return y


def spmv(op: ReducedOperator, x, precision="fp64", out=None, lanes_per_group=None):
    """y = K_ff x with the CSR SpMV kernel of the PCG (FP64 or FP32 values); "mixed" runs the
    sliced difference-form product."""
    if precision == "mixed":
        return sell_spmv(op, x, "mixed", out=out)
    prec = PRECISIONS[precision]
    dt = torch.float32 if precision == "fp32" else torch.float64
    x = torch.as_tensor(x).to(device=op.vals64.device, dtype=dt).contiguous()
    y = out if out is not None else torch.empty(op.n, dtype=dt, device=op.vals64.device)
    csr = op.csr_struct()
    lpg = lanes_per_group if lanes_per_group is not None else tuned_lanes_per_group(op, precision)
    rc = L.lib.feab_csr_spmv(C.byref(csr), None, prec, int(lpg), L.dptr(x), L.dptr(y), L.stream_ptr(op.vals64.device))
    L.raise_for(rc, "csr spmv")
    return y
