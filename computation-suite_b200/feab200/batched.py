"""Batched multi-RHS solves on the GPU.

``solve_static_batched(fesystem, F_batch)`` keeps the reference's signature and meaning
(fea_engine/src/fea_engine/batched_solve.py:105-164): every column of F_batch is solved against
the system's K with its boundary conditions (non-homogeneous Dirichlet values included); the
one factorisation the reference reuses across columns is replaced by a block-PCG whose SpMM
reads K once per step for the whole panel of columns.

``ProblemBatch`` solves many independent problems (different meshes, moduli and load panels)
in one launch sequence: the meshes are concatenated into one disconnected mesh, so node
topology, CSR pattern, element matrices and assembly each run once over the whole batch, and
K is block diagonal by construction.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import tempfile
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .device import DeviceMesh, ReducedOperator, cuda_device

PANELS = (1, 2, 4, 8, 16, 32, 64)


def panel_width(k):
    for w in PANELS:
        if k <= w:
            return w
    raise ValueError(f"at most {PANELS[-1]} right-hand sides per problem in one panel, got {k}")


@dataclass
class BatchResult:
    status: np.ndarray        # (P,) FEAB_* per problem
    iters: np.ndarray         # (P, K) CG iterations per column
    relres: np.ndarray        # (P, K) final FP64 relative residual per column


def _problem_groups(group_ptr_host, row_bounds):
    """The first node row group of each problem, then the group count."""
    return np.searchsorted(np.asarray(group_ptr_host, dtype=np.int64), row_bounds, side="left").astype(np.int32)


def _work_items(group_ptr_host, row_bounds, max_groups=64):
    """Cut each problem's node row groups into items of <= max_groups groups (whole node tiles of
    the SpMM when max_groups is a multiple of TILE_GROUPS)."""
    g_bounds = _problem_groups(group_ptr_host, row_bounds)
    item_problem, g0s, g1s, prob_items = [], [], [], [0]
    for p in range(len(row_bounds) - 1):
        a, b = int(g_bounds[p]), int(g_bounds[p + 1])
        if b <= a:
            raise ValueError(f"problem {p} has no free DOF")
        for s in range(a, b, max_groups):
            item_problem.append(p)
            g0s.append(s)
            g1s.append(min(b, s + max_groups))
        prob_items.append(len(item_problem))
    return (np.array(item_problem, np.int32), np.array(g0s, np.int32), np.array(g1s, np.int32),
            np.array(prob_items, np.int32))


def shard_problems(costs, world):
    """Assign independent problems to `world` ranks: longest cost first, each to the least
    loaded rank (ties to the lowest rank).  Deterministic, so every rank computes the same
    assignment with no communication.  Returns one ascending index array per rank."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = np.zeros(world)
    shards = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        shards[r].append(i)
        load[r] += costs[i]
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def problem_cost(n_nodes, n_rhs):
    """Work of one problem in a block-PCG panel: rows x panel width (the SpMM streams K once per
    step for the whole panel; iteration counts are similar across the batch)."""
    return 3.0 * n_nodes * panel_width(n_rhs)


TILE_GROUPS = L.TILE_GROUPS


def _block_pcg_call(op, item_problem, g0, g1, prob_items, B_panel, cols, tol, maxiter, precision, reliable_delta,
                    chunk, problem_groups=None):
    """One feab_block_pcg_solve over a panel of width B_panel.shape[1] (a power of two).  With
    problem_groups (and items of whole tiles) the SpMM walks the operator's node tiles."""
    dev = op.vals64.device
    n, K = B_panel.shape
    P = len(prob_items) - 1
    t = lambda a: torch.as_tensor(a).to(dev)  # noqa: E731
    ip, ig0, ig1, pit, pcols = t(item_problem), t(g0), t(g1), t(prob_items), t(np.asarray(cols, np.int32))
    batch = L.Batch(P, K, len(item_problem), 0, ip.data_ptr(), ig0.data_ptr(), ig1.data_ptr(), pit.data_ptr(),
                    pcols.data_ptr())
    wbytes = int(L.lib.feab_block_pcg_workspace_bytes(n, K, P, len(item_problem)))
    ws = torch.empty(wbytes, dtype=torch.uint8, device=dev)
    X = torch.empty((n, K), dtype=torch.float64, device=dev)
    B_panel = B_panel.to(dev, torch.float64).contiguous()
    prec = L.PREC_MIXED if precision == "mixed" else L.PREC_FP64
    diff = C.byref(op.diff_operator()) if precision == "mixed" else None
    tiles = C.byref(op.tile_operator(precision, problem_groups)) if problem_groups is not None else None
    params = L.PcgParams(float(tol), int(maxiter or 0), prec, float(reliable_delta), int(chunk), 1, 0, 0)
    iters = np.zeros(P * K, np.int32)
    relres = np.zeros(P * K, np.float64)
    status = np.zeros(P, np.int32)
    csr = op.csr_struct()
    rc = L.lib.feab_block_pcg_solve(C.byref(csr), diff, tiles, C.byref(batch), L.dptr(op.dinv64), L.dptr(B_panel),
                                    L.dptr(X), C.byref(params), L.dptr(ws), wbytes,
                                    iters.ctypes.data_as(C.POINTER(C.c_int32)),
                                    relres.ctypes.data_as(C.POINTER(C.c_double)),
                                    status.ctypes.data_as(C.POINTER(C.c_int32)), L.stream_ptr(dev))
    if rc in (L.FEAB_BAD_ARG, L.FEAB_CUDA_ERROR):
        L.raise_for(rc, "block PCG")
    return X, BatchResult(status, iters.reshape(P, K), relres.reshape(P, K))


def block_pcg(op: ReducedOperator, row_bounds, B_panel, cols, tol=1e-8, maxiter=None, precision="fp64",
              reliable_delta=0.1, chunk=16, max_groups=None, tile_width=None, tune=True, node_tiles=None):
    """Solve the panel B_panel (n x K, row-major, device) for the problems whose free rows are
    [row_bounds[p], row_bounds[p+1]).  Returns (X_panel, BatchResult).

    Launch shape: work items of ``max_groups`` node row groups, and the panel processed in
    column tiles of ``tile_width`` (each tile is its own block solve; K is streamed once per
    tile and step), and ``node_tiles``: the SpMM walks tiles of TILE_GROUPS row groups with merged
    column lists (``ReducedOperator.tile_operator``; needs max_groups a multiple of TILE_GROUPS)
    instead of single row groups.  Left as None they come from ``tuned_block_shape`` (timed once
    per operator shape and cached) when ``tune`` is true, else 64 groups, the full width and node
    tiles (node tiles whenever max_groups allows them, if the shape is given)."""
    if precision not in ("fp64", "mixed"):
        raise ValueError("block PCG precision must be 'fp64' or 'mixed'")
    n, K = B_panel.shape
    if n != op.n or K not in PANELS:
        raise ValueError(f"panel must be ({op.n}, k) with k in {PANELS}")
    cols = np.asarray(cols, np.int64)
    if max_groups is None or tile_width is None:
        if tune:
            shape = tuned_block_shape(op, row_bounds, B_panel, cols, precision)
        else:
            shape = BlockShape(64, K, None, True)
        max_groups = shape.item_groups if max_groups is None else max_groups
        tile_width = shape.tile_width if tile_width is None else tile_width
        node_tiles = shape.node_tiles if node_tiles is None else node_tiles
    if node_tiles is None:
        node_tiles = max_groups % TILE_GROUPS == 0
    if tile_width not in PANELS or tile_width > K:
        raise ValueError(f"tile_width must be a panel width <= {K}, got {tile_width}")
    if int(max_groups) < 1:
        raise ValueError("max_groups must be >= 1")
    gp = op.pattern.group_ptr.cpu().numpy()
    items = _work_items(gp, np.asarray(row_bounds), int(max_groups))
    if node_tiles and max_groups % TILE_GROUPS:
        raise ValueError(f"node tiles need work items of a multiple of {TILE_GROUPS} row groups, got {max_groups}")
    pgroups = _problem_groups(gp, np.asarray(row_bounds)) if node_tiles else None
    if tile_width == K:
        return _block_pcg_call(op, *items, B_panel, cols, tol, maxiter, precision, reliable_delta, chunk, pgroups)
    P = len(row_bounds) - 1
    X = torch.zeros((n, K), dtype=torch.float64, device=op.vals64.device)
    status = np.zeros(P, np.int32)
    iters = np.zeros((P, K), np.int32)
    relres = np.zeros((P, K), np.float64)
    for c0 in range(0, K, tile_width):
        ct = np.clip(cols - c0, 0, tile_width)
        if not ct.any():
            continue
        Xt, rt = _block_pcg_call(op, *items, B_panel[:, c0:c0 + tile_width], ct, tol, maxiter, precision,
                                 reliable_delta, chunk, pgroups)
        X[:, c0:c0 + tile_width] = Xt
        iters[:, c0:c0 + tile_width] = rt.iters
        relres[:, c0:c0 + tile_width] = rt.relres
        status = np.where(status == 0, rt.status, status)
    return X, BatchResult(status, iters, relres)


# ----------------------------------------------------------------------------- launch-shape tuner
ITEM_GROUPS = (16, 32, 64, 128, 256)


@dataclass
class BlockShape:
    item_groups: int          # node row groups per work item (the "elements per block" of the SpMM)
    tile_width: int           # right-hand-side columns per block solve
    us_per_step: float | None  # measured cost of one block-PCG step of the whole panel
    node_tiles: bool = False   # the SpMM walks node tiles (ReducedOperator.tile_operator)


_tuned_block = {}


def tuning_cache_path():
    """JSON file of tuned block-PCG launch shapes: $FEAB_TUNING_CACHE, else
    ~/.cache/feab200/block_pcg_tuning.json."""
    return os.environ.get("FEAB_TUNING_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "feab200",
                                                               "block_pcg_tuning.json")


def tuning_key(device_name, n, nnz, n_problems, k, precision):
    return f"{device_name}|n={n}|nnz={nnz}|problems={n_problems}|k={k}|{precision}|spmm=tiles{TILE_GROUPS}"


def load_tuning(path=None):
    path = path or tuning_cache_path()
    try:
        with open(path) as fh:
            raw = json.load(fh)
    except (OSError, ValueError):
        return {}
    out = {}
    for key, v in raw.items() if isinstance(raw, dict) else ():
        try:
            shape = BlockShape(int(v["item_groups"]), int(v["tile_width"]),
                               None if v.get("us_per_step") is None else float(v["us_per_step"]),
                               bool(v.get("node_tiles", False)))
        except (KeyError, TypeError, ValueError):
            continue
        if shape.item_groups >= 1 and shape.tile_width in PANELS and not (
                shape.node_tiles and shape.item_groups % TILE_GROUPS):
            out[key] = shape
    return out


def save_tuning(key, shape, path=None):
    """Merge one entry into the cache file (written to a temporary file and renamed, so a
    concurrent reader never sees a partial file)."""
    path = path or tuning_cache_path()
    entries = {k: {"item_groups": s.item_groups, "tile_width": s.tile_width, "us_per_step": s.us_per_step,
                   "node_tiles": s.node_tiles} for k, s in load_tuning(path).items()}
    entries[key] = {"item_groups": shape.item_groups, "tile_width": shape.tile_width,
                    "us_per_step": shape.us_per_step, "node_tiles": shape.node_tiles}
    try:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path) or ".", suffix=".tmp")
        with os.fdopen(fd, "w") as fh:
            json.dump(entries, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass                   # a read-only home directory keeps the in-process cache only


def _step_cost_us(op, items, B_panel, cols, precision, short=4, long=20, problem_groups=None):
    """Device time of one block-PCG step over this panel: two runs of tol 0 (no column
    converges) of `short` and `long` steps, timed with CUDA events; the difference over
    long - short removes setup and graph capture."""
    times = []
    for steps in (short, long, short, long):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _block_pcg_call(op, *items, B_panel, cols, 0.0, steps, precision, 0.1, 8, problem_groups)
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b) * 1e3)
    return max(1e-3, (min(times[1], times[3]) - min(times[0], times[2])) / (long - short))


def tuned_block_shape(op, row_bounds, B_panel, cols, precision="fp64", candidates=None):
    """The (work-item groups, column tile width, node tiles or single row groups) with the
    cheapest measured block-PCG step for this operator and panel, timed on the actual operator
    and right-hand sides over ITEM_GROUPS x {panel widths <= K} x {node tiles, row groups}; a
    tile narrower than K costs K / width tile steps.
    Cached in this process and in the JSON file of tuning_cache_path(), keyed by (GPU, n, nnz,
    problems, K, precision)."""
    n, K = B_panel.shape
    P = len(row_bounds) - 1
    dev = op.vals64.device
    key = tuning_key(torch.cuda.get_device_name(dev), op.n, op.nnz, P, K, precision)
    hit = _tuned_block.get(key)
    if hit is None:
        hit = load_tuning().get(key)
    if hit is not None:
        _tuned_block[key] = hit
        return hit
    gp = op.pattern.group_ptr.cpu().numpy()
    cols = np.asarray(cols, np.int64)
    if candidates is None:
        candidates = [(g, w, nt) for g in ITEM_GROUPS for w in PANELS if 16 <= w <= K or w == K
                      for nt in (False, True) if not (nt and g % TILE_GROUPS)]
    best = None
    for g, w, nt in candidates:
        items = _work_items(gp, np.asarray(row_bounds), g)
        ct = np.clip(cols, 0, w)
        pgroups = _problem_groups(gp, np.asarray(row_bounds)) if nt else None
        cost = _step_cost_us(op, items, B_panel[:, :w].contiguous(), ct, precision, problem_groups=pgroups) * (K // w)
        if best is None or cost < best.us_per_step:
            best = BlockShape(g, w, cost, nt)
    _tuned_block[key] = best
    save_tuning(key, best)
    return best


class ProblemBatch:
    """Independent hex8 problems solved together.  Each problem is (nodes, elements, D, fixed
    DOFs, F (n_dof,) or (n_dof, k)); D of every problem must be a positive multiple of the
    first problem's D (same Poisson ratio, any modulus), which becomes a per-element scale."""

    def __init__(self, problems, device=None):
        self.device = cuda_device(device)
        if not problems:
            raise ValueError("empty problem batch")
        D_ref = np.asarray(problems[0][2], dtype=float)
        nodes, elems, scale, fixed, self.sizes = [], [], [], [], []
        off = 0
        for (X, el, D, fx, F) in problems:
            X = np.asarray(X, float)
            el = np.asarray(el)
            s = float(np.asarray(D)[0, 0] / D_ref[0, 0])
            if not (s > 0 and np.allclose(np.asarray(D), s * D_ref, rtol=1e-12, atol=0)):
                raise ValueError("every problem's D must be a positive multiple of the first problem's D")
            nodes.append(X)
            elems.append(el + off)
            scale.append(np.full(len(el), s))
            fixed.append(np.asarray(fx, np.int64) + 3 * off)
            self.sizes.append(len(X))
            off += len(X)
        self.node_offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        self.D_ref = D_ref
        self.dm = DeviceMesh(np.concatenate(nodes), np.concatenate(elems), device=self.device)
        self.scale = np.concatenate(scale)
        self.fixed = np.concatenate(fixed)
        self.loads = [np.asarray(pr[4], float).reshape(3 * len(pr[0]), -1) for pr in problems]
        mask = np.ones(3 * off, dtype=bool)
        mask[self.fixed] = False
        self.free = np.flatnonzero(mask)
        self.row_bounds = np.searchsorted(self.free, 3 * self.node_offsets)
        self.cols = [F.shape[1] for F in self.loads]
        self.K = panel_width(max(self.cols))
        self.op = None
        self._didx = None

    def _device_index(self):
        """Device int64 copies of (each free row's DOF within its own problem, its DOF in the
        concatenated system), uploaded once."""
        if self._didx is None:
            local = self.free - 3 * np.repeat(self.node_offsets[:-1], np.diff(self.row_bounds))
            self._didx = (torch.as_tensor(local).to(self.device), torch.as_tensor(self.free).to(self.device))
        return self._didx

    def assemble(self):
        pat = self.dm.pattern(self.fixed)
        ke = self.dm.element_stiffness(self.D_ref, scale=self.scale)
        self.op = self.dm.assemble(ke, pat, want32=False)
        return self.op

    def rhs_panel(self):
        """The (n, K) right-hand-side panel on the device: each problem's load columns are
        uploaded as given and their free rows gathered on the device."""
        local_t, _ = self._device_index()
        B = torch.zeros((len(self.free), self.K), dtype=torch.float64, device=self.device)
        for p, F in enumerate(self.loads):
            a, b = int(self.row_bounds[p]), int(self.row_bounds[p + 1])
            Fd = torch.from_numpy(np.ascontiguousarray(F)).to(self.device)
            B[a:b, : F.shape[1]] = Fd.index_select(0, local_t[a:b])
        return B

    def solve(self, tol=1e-8, maxiter=None, precision="fp64", reliable_delta=0.1, chunk=16):
        """Returns ([U_p (n_dof_p, k_p) numpy], BatchResult)."""
        if self.op is None:
            self.assemble()
        X, res = block_pcg(self.op, self.row_bounds, self.rhs_panel(), self.cols, tol=tol, maxiter=maxiter,
                           precision=precision, reliable_delta=reliable_delta, chunk=chunk)
        # scatter the free rows into the concatenated DOF vectors on the device (fixed DOFs stay 0),
        # copy once, and hand out each problem's rows and load columns as views
        _, free_t = self._device_index()
        U = torch.zeros((3 * int(self.node_offsets[-1]), self.K), dtype=torch.float64, device=self.device)
        U.index_copy_(0, free_t, X)
        Uh = U.cpu().numpy()
        out = [Uh[3 * int(self.node_offsets[p]): 3 * int(self.node_offsets[p + 1]), : F.shape[1]]
               for p, F in enumerate(self.loads)]
        return out, res


def solve_static_batched(fesystem, F_batch, backend=None, tol=1e-10, precision="fp64", maxiter=None):
    """U_batch (n_dof, n_batch) for every load column, with fesystem's K and boundary
    conditions (batched_solve.py:105-164).  The direct factorisation is replaced by the GPU
    block-PCG to relative residual `tol` per column; columns are processed in panels of <= 64."""
    F_batch = np.asarray(F_batch, dtype=float)
    if F_batch.ndim != 2 or F_batch.shape[0] != fesystem.n_dof:
        raise ValueError(f"F_batch must have shape ({fesystem.n_dof}, n_batch)")
    op = fesystem.reduced_operator(want32=False)
    free = fesystem.free_dofs
    fixed = fesystem.fixed_dofs_array
    u_fixed = fesystem._fixed_dof_values_array(fixed)
    corr = fesystem._reduced_rhs(np.zeros(fesystem.n_dof)).cpu().numpy()   # = -K[free, fixed] u_fixed
    U = np.zeros((fesystem.n_dof, F_batch.shape[1]))
    U[fixed, :] = u_fixed[:, None]
    for c0 in range(0, F_batch.shape[1], 64):
        Fc = F_batch[:, c0:c0 + 64]
        k = Fc.shape[1]
        K = panel_width(k)
        B = np.zeros((len(free), K))
        B[:, :k] = Fc[free] + corr[:, None]
        X, res = block_pcg(op, [0, len(free)], torch.as_tensor(B), [k], tol=tol, maxiter=maxiter,
                           precision=precision)
        st = int(res.status[0])
        if st == L.FEAB_NOT_SPD:
            raise np.linalg.LinAlgError("solve_static_batched: K is not SPD")
        if st == L.FEAB_NOT_CONVERGED:
            raise RuntimeError("solve_static_batched: block PCG did not converge")
        L.raise_for(st, "solve_static_batched")
        U[free, c0:c0 + k] = X.cpu().numpy()[:, :k]
    return U
