#!/usr/bin/env python
"""Benchmark: hex8 assemble + PCG + compliance gradient, mixed precision vs plain FP64, on B200.

One step = the whole hot path over one synthetic cantilever (default 128x32x32 hex8, 2.0 x 0.4 x
0.4 m, E = 210 GPa, nu = 0.3, x = 0 clamped, random N(0,1)*1e6 Pa per-node tip traction):
node topology + CSR pattern + element matrices + CSR values (FP64 + FP32 copy + Jacobi
diagonal) + Jacobi-PCG to the residual tolerance + SIMP compliance gradient dC/drho_e (p = 3,
rho = 1, rho_min = 1e-9).  Inputs are resident in HBM when the timed region starts; K_ff
(> 400 MB FP64) is larger than the 126 MB L2, so no explicit L2 flush is done between steps.

`value` is the mixed-precision step time (ms, lower is better); the plain FP64 step time is
reported beside it.  `e2e` is the same step through the public FESystem API from host numpy
arrays, host<->device copies included.  With --gpus N (torchrun) every rank runs an
independent replica of the workload (the path has no cross-GPU exchange) and the slowest
rank's time is reported.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "computation-suite_b200"))

import numpy as np  # noqa: E402

METRIC = "hex8 assemble+PCG+grad time at rel err 1e-8, mixed vs plain FP64, 1 B200"
PENAL, RHO_MIN = 3.0, 1e-9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 20 for the headline workload and the reference arm, 3 otherwise)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--shape", type=int, nargs=3, default=(128, 32, 32))
    ap.add_argument("--tol", type=float, default=1e-9)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--snapshot-shape", type=int, nargs=3, default=(192, 48, 48),
                    help="mesh of the snapshot workload (the 192x48x48 case by default)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle job (CPU baseline and the full-size accuracy check against the oracle)")
    ap.add_argument("--spmv-reps", type=int, default=20)
    ap.add_argument("--workload", choices=["cantilever", "simp", "batch", "snapshot", "gram", "spmv", "recovery",
                                           "simp_oc", "elements", "modal", "block_step", "direct"],
                    default="cantilever",
                    help="cantilever: the headline (assemble + PCG + dC/drho); the others measure the SIMP "
                         "adjoint, the uneven batch and the snapshot/POD cases")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if (args.workload == "cantilever" or args.impl == "reference") else 3
    return args


# ----------------------------------------------------------------------------- distributed
def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    import torch
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(v, world):
    import torch
    if world == 1:
        return v
    dev = "cpu" if torch.distributed.get_backend() == "gloo" else "cuda"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.path = None
        self.gpu = gpu_index

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def wait_first_sample(self, timeout=20.0):
        """nvidia-smi's start-up can stall the GPU for a moment: wait until it has written its
        first sample, so that this happens before a timed region, not inside it."""
        if self.proc is None:
            return
        t0 = time.time()
        while time.time() - t0 < timeout and self.proc.poll() is None:
            self.out.flush()
            if os.path.getsize(self.path) > 0:
                return
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- workload
def build_workload(shape):
    from feab200 import cantilever
    return cantilever.random_tip_cantilever(*shape)


class DeviceProblem:
    """Inputs resident in HBM: coordinates, connectivity, reduced load vector, densities."""

    def __init__(self, c, device):
        import torch
        self.c = c
        self.device = device
        self.coords = torch.as_tensor(c.mesh.nodes).to(device)
        self.conn = torch.as_tensor(c.mesh.elements.astype(np.int32)).to(device)
        self.fixed = c.fixed
        self.free = torch.as_tensor(c.free).to(device)
        self.Ff = torch.as_tensor(c.F[c.free]).to(device)
        self.rho = torch.ones(len(c.mesh.elements), dtype=torch.float64, device=device)
        self.n_dof = c.n_dof

    def step(self, precision, tol):
        import torch
        from feab200.device import DeviceMesh, pcg_solve
        dm = DeviceMesh(self.coords, self.conn, device=self.device)
        pat = dm.pattern(self.fixed)
        ke = dm.element_stiffness(self.c.D)
        op = dm.assemble(ke, pat, want32=(precision == "fp32"))
        x, info = pcg_solve(op, self.Ff, tol=tol, precision=precision)
        if info.status != 0:
            raise RuntimeError(f"PCG failed: {info}")
        u = torch.zeros(self.n_dof, dtype=torch.float64, device=self.device)
        u[self.free] = x
        dc = dm.simp_vjp(self.c.D, self.rho, PENAL, RHO_MIN, u)
        return x, dc, info, op


def time_steps(prob, precision, tol, steps, warmup, world):
    import torch
    from feab200 import _lib as L
    # the warm-up keeps each step's results alive while the next one runs, as the timed loop does,
    # so the caching allocator holds two steps' buffers before timing starts (otherwise the second
    # timed step pays for fresh device allocations: measured 170-245 ms instead of 68-77 ms)
    res = None
    for _ in range(warmup):
        res = prob.step(precision, tol)
    torch.cuda.synchronize()
    barrier(world)
    gc.collect()
    gc.disable()          # no collector pause of the host inside the timed steps
    # an event after every step: the per-step times (no extra synchronisation in the loop)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    n0 = L.lib.feab_launch_count()
    torch.cuda.nvtx.range_push(f"feab_timed_{precision}")     # lets a profiler select the timed steps
    evs[0].record()
    for i in range(steps):
        res = prob.step(precision, tol)
        evs[i + 1].record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    gc.enable()
    launches = int(L.lib.feab_launch_count() - n0)
    ms = evs[0].elapsed_time(evs[-1]) / steps
    each = [round(evs[i].elapsed_time(evs[i + 1]), 2) for i in range(steps)]
    x, dc, info, op = res
    return max_over_ranks(ms, world), x, dc, info, op, launches, each


def e2e_steps(c, precision, tol, steps, warmup):
    """The step through the public API from host numpy arrays (copies inside the timed region)."""
    import torch
    import feab200
    from feab200 import topopt

    def one():
        mesh = feab200.Mesh(nodes=c.mesh.nodes, elements=c.mesh.elements)
        fs = feab200.FESystem(mesh, feab200.Hex8Solid3D(), sparse=True, device="cuda")
        fs.assemble_stiffness(c.D)
        fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
        fs.F[:] = c.F
        U = fs.solve_static(method="pcg", tol=tol, precision=precision)
        ke_unit, conn = topopt.unit_stiffness_stack(fs, c.D)
        dc = topopt.compliance_sensitivity_closed_form(ke_unit, conn, 3, np.asarray(U),
                                                       np.ones(len(c.mesh.elements)), PENAL, RHO_MIN)
        return U, dc

    res = None
    for _ in range(warmup):      # results kept alive as in the timed loop (allocator warm-up)
        res = one()
    torch.cuda.synchronize()
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    for _ in range(steps):
        res = one()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / steps
    gc.enable()
    N, E, n = len(c.mesh.nodes), len(c.mesh.elements), len(c.free)
    h2d = N * 3 * 8 + E * 8 * 4 + n * 8 + 3 * N * 8 + E * 8     # nodes, conn, F_free, U (for dC/drho), rho
    d2h = 3 * N * 8 + E * 8                                      # U, dC/drho
    return ms, h2d, d2h


def spmv_bytes(op, precision):
    """Algorithmic bytes of one launch of the PCG's SpMV kernel for `precision`, counted from
    what the kernel must read and write once: values, column indices (one row per node
    group, since the rows of a node share them; 2 bytes each when the sliced operator holds
    16-bit offsets), row/group pointers, the x vector and y."""
    p = op.pattern
    rp = p.row_ptr.cpu().numpy().astype(np.int64)
    gp = p.group_ptr.cpu().numpy().astype(np.int64)
    f = np.diff(gp)
    lens = rp[gp[:-1] + 1] - rp[gp[:-1]]
    lead = int(lens.sum())
    n, nnz, G = p.n, p.nnz, p.n_groups
    ptrs = 4 * (n + 1) + 4 * (G + 1)
    if precision == "fp32":
        return nnz * 4 + 4 * lead + ptrs + 2 * n * 4
    # the sliced operator reads 2-byte column offsets when they all fit 16 bits
    ib = 2 if op.sell_operator(precision).tcol16 else 4
    if precision == "fp64":
        return nnz * 8 + ib * lead + ptrs + 2 * n * 8
    own = int((f * f).sum())                                   # own-node block entries are skipped
    return (nnz - own) * 6 + ib * (lead - n) + ptrs + G + 24 * n + 2 * n * 8


def spmv_roofline(op, precision, reps, peak_gbs):
    """Average duration of the PCG's SpMV kernel (the sliced SELL-32 product for fp64 and mixed,
    the CSR one for fp32) with CUDA events on the launching stream; L2 is flushed before each
    launch (L2Flush: a 256 MB write, then a 256 MB read)."""
    import torch
    from feab200.device import sell_spmv, spmv, tuned_lanes_per_group
    dev = op.vals64.device
    dt = torch.float32 if precision == "fp32" else torch.float64
    x = torch.randn(op.n, dtype=dt, device=dev)
    y = torch.empty(op.n, dtype=dt, device=dev)
    flush = L2Flush(dev)
    if precision == "fp32":
        lpg = tuned_lanes_per_group(op, precision)
        run = lambda: spmv(op, x, precision, out=y, lanes_per_group=lpg)  # noqa: E731
    else:
        lpg = None
        run = lambda: sell_spmv(op, x, precision, out=y)  # noqa: E731
    run()
    times = []
    for _ in range(reps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        run()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) * 1e-3)
    t = statistics.mean(times)
    nbytes = spmv_bytes(op, precision)
    p = op.pattern
    bytes_csr = p.nnz * ((4 if precision == "fp32" else 8) + 4) + 4 * (p.n + 1) + 2 * p.n * (4 if precision == "fp32" else 8)
    achieved = nbytes / t / 1e9
    kern = {"fp64": "k_sell_spmv<FP64>", "fp32": f"k_spmv<float, {lpg}>", "mixed": "k_sell_spmv<MIXED>"}[precision]
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak_gbs, "unit": "GB/s",
            "frac": round(achieved / peak_gbs, 3), "traffic": None,
            "kernel": f"{kern} (the SpMV of PCG step A, {precision})",
            "bytes_per_launch": int(nbytes),
            "csr_formula_bytes": int(bytes_csr), "launch_us": round(t * 1e6, 2)}


def pcg_iteration_roofline(op, b, tol, precision, peak_gbs):
    """The whole PCG iteration as one unit: a full solve timed with CUDA events on the solve's
    stream, divided by its iterations, against the iteration's algorithmic bytes: the SpMV of
    spmv_bytes (which counts reading p once and writing Ap), plus P (reads z and p, writes p),
    A's own p rows for p.Ap, and B (reads x, p, r, Ap and dinv, writes x, r and z): 12 n doubles."""
    import torch
    from feab200.device import pcg_solve
    pcg_solve(op, b, tol=tol, precision=precision)
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    _, info = pcg_solve(op, b, tol=tol, precision=precision)
    e.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(e) * 1e-3 / max(1, info.iters)
    nbytes = spmv_bytes(op, precision) + 12 * op.n * 8
    return {"us_per_iteration": round(t * 1e6, 2), "iterations": info.iters, "bytes_per_iteration": int(nbytes),
            "achieved": round(nbytes / t / 1e9, 1), "peak": peak_gbs, "unit": "GB/s",
            "frac": round(nbytes / t / 1e9 / peak_gbs, 3),
            "note": "solve time (operator build and setup included) over its iterations; the SpMV step kernel "
                    "dominates"}


class L2Flush:
    """Evicts L2 before a timed launch: writes one 256 MB buffer (twice the 126 MB L2), then reads
    a second one, so that the dirty lines of the write are written back before the timed kernel
    starts and L2 holds only clean, unrelated lines.  Then the GPU spins for about 0.1 ms
    (torch.cuda._sleep), so that the host has enqueued the timed launch before its start event
    runs; otherwise the events also time the host's launch overhead (measured: the mixed sliced
    SpMV read 49.3 us on average that way, against 45.3 us with the pad and a 44.9 us minimum
    either way)."""

    def __init__(self, device):
        import torch
        self.w = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
        self.r = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
        self.sink = torch.empty(1, dtype=torch.float32, device=device)

    def __call__(self):
        import torch
        self.w.fill_(1.0)
        torch.sum(self.r, dim=0, keepdim=True, out=self.sink)
        torch.cuda._sleep(200_000)


def measured_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------- CPU (oracle)
def oracle_step(w, tol, solve_tol=None):
    """One whole step of the reference path on the host cores, through the oracle (the
    NumPy/SciPy restatement of fea_engine; importing it loads no CUDA library): element
    matrices + COO -> CSR + free x free slice + Jacobi diagonal (a7-a9, a14, a16), Jacobi-PCG
    (a17) and the closed-form dC/drho at rho = 1 (a24).  With solve_tol < tol the PCG runs on to
    solve_tol (the accuracy oracle) and the phase times are taken where the residual first
    fell below tol (the PCG iterates do not depend on the stopping tolerance), so one run gives
    both the timed step and the tight reference solution."""
    import oracle as O
    X, el, free = w["nodes"], w["elements"], w["free"]
    t0 = time.perf_counter()
    ke = O.hex8_element_stiffness(X[el], w["D"])
    Kff = O.reduce_free(O.structural_csr(ke, el, w["n_dof"]), free)
    dinv = O.jacobi_inverse_diagonal(Kff)
    t1 = time.perf_counter()
    hist = []
    x, iters, relres = O.preconditioned_cg(Kff, w["F"][free], dinv, tol=min(tol, solve_tol or tol), history=hist)
    t2 = time.perf_counter()
    k_tol, t_tol = next(((k, t) for k, (t, r) in enumerate(hist, 1) if r < tol), (iters, t2))
    u = np.zeros(w["n_dof"])
    u[free] = x
    t3 = time.perf_counter()
    dc = O.compliance_sensitivity_closed_form(ke, el, u, np.ones(len(el)), PENAL, RHO_MIN)
    t4 = time.perf_counter()
    times = {"assembly_s": t1 - t0, "pcg_s": t_tol - t1, "grad_s": t4 - t3}
    times["step_s"] = sum(times.values())
    return {"Kff": Kff, "x": x, "dc": dc, "iters": iters, "iters_at_tol": k_tol, "relres": relres, "times": times}


def _oracle_job(shape, tol, solve_tol, outdir):
    """Child process (started with 'spawn', after the parent's GPU measurements): builds the
    workload with the oracle's own builders, runs oracle_step to solve_tol and leaves the
    reference solution, K_ff and the timings in outdir."""
    sys.path.insert(0, ROOT)
    from oracle import workloads
    w = workloads.random_tip_cantilever(*shape)
    r = oracle_step(w, tol, solve_tol)
    K = r["Kff"]
    for name, arr in (("indptr", K.indptr), ("indices", K.indices), ("data", K.data), ("x", r["x"]), ("dc", r["dc"])):
        np.save(os.path.join(outdir, name + ".npy"), arr)
    json.dump({"iters": r["iters"], "iters_at_tol": r["iters_at_tol"], "relres": r["relres"], "times": r["times"],
               "threads": os.cpu_count()}, open(os.path.join(outdir, "meta.json"), "w"))


class OracleRun:
    """The oracle job of the headline workload, run after the GPU measurements in a separate
    process: its solution is the FP64 accuracy reference (the oracle's PCG to 1e-12, which stands
    in for the reference's sparse direct solve at these sizes) and its phase times are a real full
    CPU step (not extrapolated)."""

    SOLVE_TOL = 1e-12

    def __init__(self, shape, tol):
        import multiprocessing as mp
        self.dir = tempfile.mkdtemp(prefix="feab_oracle_")
        self.proc = mp.get_context("spawn").Process(target=_oracle_job, args=(tuple(shape), tol, self.SOLVE_TOL,
                                                                              self.dir), daemon=True)
        self.proc.start()

    def result(self, timeout):
        self.proc.join(timeout)
        if self.proc.is_alive():
            self.proc.terminate()
            self.proc.join(10)
            return None, f"oracle job still running after {timeout:.0f} s"
        if self.proc.exitcode != 0:
            return None, f"oracle job exited with {self.proc.exitcode}"
        ld = lambda n: np.load(os.path.join(self.dir, n + ".npy"))  # noqa: E731
        out = {n: ld(n) for n in ("indptr", "indices", "data", "x", "dc")}
        out.update(json.load(open(os.path.join(self.dir, "meta.json"))))
        for n in os.listdir(self.dir):
            os.unlink(os.path.join(self.dir, n))
        os.rmdir(self.dir)
        return out, None


def parity_vs_oracle(ref, op, xs, dc):
    """The GPU results against the oracle at the full size: CSR row_ptr / col_idx bit for bit,
    K_ff values normwise, displacements and dC/drho as relative 2-norm errors."""
    import torch
    p = op.pattern
    same = (np.array_equal(p.row_ptr.cpu().numpy(), ref["indptr"]) and
            np.array_equal(p.col_idx.cpu().numpy(), ref["indices"]))
    v = op.vals64.cpu().numpy()
    k_err = float(np.abs(v - ref["data"]).max() / np.abs(ref["data"]).max()) if same else None
    xr = torch.as_tensor(ref["x"]).to(op.vals64.device)
    rel = {k: float(torch.linalg.norm(x - xr) / torch.linalg.norm(xr)) for k, x in xs.items()}
    dr = torch.as_tensor(ref["dc"]).to(dc.device)
    return {"csr_bit_exact": bool(same), "K_rel_err_normwise": k_err, "u_rel_err": rel,
            "dc_rel_err": float(torch.linalg.norm(dc - dr) / torch.linalg.norm(dr)),
            "oracle": (f"oracle FP64 Jacobi-PCG (restatement of preconditioned_cg) to relative residual "
                       f"{OracleRun.SOLVE_TOL:g}, {ref['iters']} iterations; K_ff by COO -> CSR as "
                       f"scatter_global_stiffness + K[free, free]")}


def gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    ids = [v for v in vis.split(",") if v.strip()]
    if ids and local < len(ids) and ids[local].strip().isdigit():
        return int(ids[local])
    return local


# ----------------------------------------------------------------------------- other workloads
def _timed(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        out = fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, out


def workload_simp(args):
    """SIMP compliance on a 96x32x32 cantilever: assemble K(rho), PCG, dC/drho through the
    torch.autograd.Function (forward solve + adjoint solve + VJP kernel)."""
    import torch
    from feab200 import cantilever, topopt
    from feab200._lib import KE_FULL as L_KE_FULL
    from feab200.device import DeviceMesh
    c = cantilever.simp_cantilever(96, 32, 32)
    dev = torch.device("cuda", torch.cuda.current_device())
    dm = DeviceMesh(c.mesh.nodes, c.mesh.elements, device=dev)
    f = torch.as_tensor(c.F[c.free]).to(dev)
    rho0 = torch.as_tensor(c.meta["rho"]).to(dev)
    res = {}
    grads = {}
    for prec in ("fp64", "mixed"):
        prob = topopt.SimpProblem(dm, c.D, c.free, penal=3.0, rho_min=1e-9, tol=args.tol, precision=prec)

        def step():
            rho = rho0.clone().requires_grad_(True)
            C = torch.dot(f, prob(rho, f))
            C.backward()
            return rho.grad

        ms, g = _timed(step, args.steps, args.warmup)
        res[prec] = ms
        grads[prec] = g
    # checks: closed form on the FP64 u, and central differences at 32 elements
    prob = topopt.SimpProblem(dm, c.D, c.free, penal=3.0, rho_min=1e-9, tol=1e-13)
    u = prob.solve_free(rho0, f)
    dc_closed = dm.simp_vjp(c.D, rho0, 3.0, 1e-9, prob.full(u))
    rng = np.random.default_rng(0)
    elems = rng.choice(len(rho0), 32, replace=False)
    h = 1e-6
    # C(rho) to ~1e-18 of itself for single-element perturbations: u from the FP64 solve (relative
    # residual 1e-13), C as the stationary form f.u + r.u with r = f - K(rho) u formed in 80-bit
    # extended precision on the host: K(rho0) plus the perturbed element's (s(rho_e) - s(rho0_e)) ke_e.
    # In FP64 the cancellation in K u (|K||u| ~ 1e4 |K u|) leaves ~1e-15 C of round-off, too much
    # for differences of ~1e-11 C over h = 1e-6.
    K0 = prob.operator(rho0).to_scipy()
    K0_ld, K0_idx, K0_starts = K0.data.astype(np.longdouble), K0.indices, K0.indptr[:-1]
    ke_sel = dm.element_stiffness(c.D, layout=L_KE_FULL)[torch.as_tensor(elems).to(dev)].cpu().numpy()
    pos = np.full(3 * dm.n_nodes, -1)
    pos[c.free] = np.arange(len(c.free))
    f_ld = c.F[c.free].astype(np.longdouble)
    rho0_h = rho0.cpu().numpy()
    simp_s = lambda r: 1e-9 + (1.0 - 1e-9) * r ** 3  # noqa: E731

    def compliance(rho, q):
        e = int(elems[q])
        ul = prob.solve_free(rho, f).cpu().numpy().astype(np.longdouble)
        Ku = np.add.reduceat(K0_ld * ul[K0_idx], K0_starts)
        rows = pos[3 * c.mesh.elements[e][:, None] + np.arange(3)[None, :]].reshape(-1)
        ue = np.where(rows >= 0, ul[np.maximum(rows, 0)], 0)
        ds = np.longdouble(simp_s(float(rho[e])) - simp_s(rho0_h[e]))
        kv = (ke_sel[q].astype(np.longdouble) @ ue) * ds
        np.add.at(Ku, rows[rows >= 0], kv[rows >= 0])
        return float(np.dot(f_ld, ul) + np.dot(f_ld - Ku, ul))

    def central(h):
        out = []
        for q, e in enumerate(elems):
            rp, rm = rho0.clone(), rho0.clone()
            rp[e] += h
            rm[e] -= h
            out.append((compliance(rp, q) - compliance(rm, q)) / (2 * h))
        return np.array(out)

    fd, fd4 = central(h), central(1e-4)
    ge = grads["mixed"].cpu().numpy()[elems]
    big = np.abs(fd4) > 1e-2 * np.abs(fd4).max()     # elementwise only where the sensitivity is not ~0
    return {"metric": "SIMP assemble+PCG+adjoint dC/drho time, 96x32x32 hex8", "value": round(res["mixed"], 3),
            "unit": "ms", "plain_fp64_ms": round(res["fp64"], 3), "mixed_speedup_vs_fp64": round(res["fp64"] / res["mixed"], 3),
            "n_elements": len(rho0),
            "rel_err": {"mixed_grad_vs_closed_form": float(torch.linalg.norm(grads["mixed"] - dc_closed) / torch.linalg.norm(dc_closed)),
                        "fp64_grad_vs_closed_form": float(torch.linalg.norm(grads["fp64"] - dc_closed) / torch.linalg.norm(dc_closed)),
                        "mixed_grad_vs_fd_h1e-6_32_elements": float(np.linalg.norm(ge - fd) / np.linalg.norm(fd)),
                        "mixed_grad_vs_fd_h1e-4_32_elements": float(np.linalg.norm(ge - fd4) / np.linalg.norm(fd4)),
                        "mixed_grad_vs_fd_h1e-4_max_elementwise": float(np.max(np.abs(ge - fd4)[big] / np.abs(fd4)[big])),
                        "fd": ("central differences at 32 random elements, FP64 solves to 1e-13, stationary compliance "
                               "f.u + r.u with the residual r = f - K u formed in 80-bit extended precision on the "
                               "host")}}


def workload_batch(args):
    """256 uneven cantilevers (4-16 load cases each) in one block-PCG."""
    import torch
    from feab200 import cantilever
    from feab200.batched import ProblemBatch, problem_cost, shard_problems
    world, rank = args.world, args.rank
    allp = cantilever.batch_cantilevers(256)
    # independent problems: each rank solves its greedy share, no data-path collective
    mine = shard_problems([problem_cost(len(p.mesh.nodes), p.F.shape[1]) for p in allp], world)[rank]
    probs = [allp[i] for i in mine]
    problems = [(p.mesh.nodes, p.mesh.elements, p.D, p.fixed, p.F) for p in probs]
    res = {}
    out = {}
    for prec in ("fp64", "mixed"):
        def step():
            b = ProblemBatch(problems)
            return b.solve(tol=args.tol, precision=prec)
        barrier(world)
        ms, (U, r) = _timed(step, max(1, args.steps // 2), 1)
        res[prec] = max_over_ranks(ms, world)
        out[prec] = (U, r)
    b = ProblemBatch(problems)
    Ut, rt = b.solve(tol=1e-13, precision="fp64")
    from feab200.batched import tuned_block_shape
    shapes = {prec: tuned_block_shape(b.op, b.row_bounds, b.rhs_panel(), b.cols, prec) for prec in ("fp64", "mixed")}
    errs = [np.linalg.norm(u - t) / np.linalg.norm(t) for u, t in zip(out["mixed"][0], Ut)]
    r = out["mixed"][1]
    n_dof = sum(3 * len(p.mesh.nodes) for p in probs)
    n_rhs = sum(p.F.shape[1] for p in probs)
    return {"metric": "uneven batch block-PCG time (256 cantilevers, 4-16 load cases each)", "value": round(res["mixed"], 3),
            "unit": "ms", "plain_fp64_ms": round(res["fp64"], 3), "mixed_speedup_vs_fp64": round(res["fp64"] / res["mixed"], 3),
            "problems": len(allp), "problems_on_rank0": len(probs), "scaling": "strong",
            "total_dof_rank0": n_dof, "total_rhs_rank0": n_rhs,
            "iters": {"max": int(r.iters.max()), "mean_active": float(r.iters[r.iters > 0].mean())},
            "rel_err_max_vs_fp64_tight": float(max(errs)), "status_ok": bool((r.status == 0).all()),
            "launch_shape": {k: {"item_groups": v.item_groups, "tile_width": v.tile_width, "node_tiles": v.node_tiles,
                                 "us_per_step": round(v.us_per_step, 1)} for k, v in shapes.items()}}


def workload_snapshot(args):
    """192x48x48 cantilever with 64 Fourier load cases: block-PCG, then POD by the tensor-core
    Gram (split bf16 x3) and the FP64 Jacobi eigensolve."""
    import torch
    from feab200 import cantilever
    from feab200.batched import ProblemBatch
    from feab200.pod import gram_bf16x3, gram_fp64, gram_int8, symeig
    c = cantilever.fourier_snapshot_cantilever(*args.snapshot_shape)
    b = ProblemBatch([(c.mesh.nodes, c.mesh.elements, c.D, c.fixed, c.F)])
    t0 = time.perf_counter()
    b.assemble()
    X, r = None, None
    from feab200.batched import block_pcg, tuned_block_shape
    res = {}
    tuned = {}
    for prec in ("mixed", "fp64"):
        # launch-shape tuning (cached per operator shape) and a short warm-up, outside the timing
        tuned[prec] = tuned_block_shape(b.op, b.row_bounds, b.rhs_panel(), b.cols, prec)
        block_pcg(b.op, b.row_bounds, b.rhs_panel(), b.cols, tol=args.tol, maxiter=2, precision=prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        Xp, rp = block_pcg(b.op, b.row_bounds, b.rhs_panel(), b.cols, tol=args.tol, precision=prec)
        e1.record()
        torch.cuda.synchronize()
        res[prec] = (e0.elapsed_time(e1), Xp, rp)
    X = res["mixed"][1]
    X32 = X.to(torch.float32).contiguous()
    gram_ms, (G, gflag) = _timed(lambda: gram_bf16x3(X32, check=False), 5, 2)
    if int(gflag.item()):
        raise RuntimeError("gram_bf16x3: a bounded wait timed out on the device")
    gram64_ms, G64 = _timed(lambda: gram_fp64(X32), 5, 2)
    gram8_ms, (G8, g8flag) = _timed(lambda: gram_int8(X32, check=False), 5, 2)
    if int(g8flag.item()):
        raise RuntimeError("gram_int8: a bounded wait timed out on the device")
    w8, _ = symeig(G8)
    s_gpu8 = torch.sqrt(torch.clamp(w8, min=0)).cpu().numpy()
    eig_ms, (w, V) = _timed(lambda: symeig(G), 3, 1)
    w64, _ = symeig(G64)
    s_gpu = torch.sqrt(torch.clamp(w, min=0)).cpu().numpy()
    s_gpu64 = torch.sqrt(torch.clamp(w64, min=0)).cpu().numpy()
    import oracle as O
    s_ref = O.pod_singular_values(X.cpu().numpy())
    rel = np.abs(s_gpu[:10] - s_ref[:10]) / s_ref[:10]
    rel64 = np.abs(s_gpu64[:10] - s_ref[:10]) / s_ref[:10]
    rel8 = np.abs(s_gpu8[:10] - s_ref[:10]) / s_ref[:10]
    rel8_vs_64 = np.abs(s_gpu8[:10] - s_gpu64[:10]) / s_gpu64[:10]
    n, k = X.shape
    peak, _ = measured_peak()
    gram_bytes = n * k * 4 + k * k * 8
    shp = "x".join(str(v) for v in args.snapshot_shape)
    return {"metric": f"snapshot block-PCG (64 RHS) + Gram POD time, {shp} hex8",
            "value": round(res["mixed"][0] + gram8_ms + eig_ms, 2), "unit": "ms",
            "block_pcg_ms": {"mixed": round(res["mixed"][0], 2), "fp64": round(res["fp64"][0], 2)},
            "launch_shape": {k: {"item_groups": v.item_groups, "tile_width": v.tile_width, "node_tiles": v.node_tiles,
                                 "us_per_step": round(v.us_per_step, 1)} for k, v in tuned.items()},
            "gram_ms": round(gram_ms, 4), "eig_ms": round(eig_ms, 3),
            "gram_roofline": {"bound": "hbm", "achieved": round(gram_bytes / (gram_ms * 1e-3) / 1e9, 1), "peak": peak,
                              "unit": "GB/s", "frac": round(gram_bytes / (gram_ms * 1e-3) / 1e9 / peak, 3),
                              "bytes_per_launch": int(gram_bytes)},
            "n_free": n, "rhs": int(c.F.shape[1]), "iters_max": int(res["mixed"][2].iters.max()),
            "sigma_rel_err_top10_bf16x3": [float(v) for v in rel],
            "sigma_rel_err_top10_fp64_gram": [float(v) for v in rel64],
            "sigma_rel_err_top10_int8_gram": [float(v) for v in rel8],
            "sigma_int8_vs_fp64_gram_top10": [float(v) for v in rel8_vs_64],
            "gram_int8_ms": round(gram8_ms, 4),
            "gram_int8_roofline": {"bound": "hbm", "achieved": round(2 * n * k * 4 / (gram8_ms * 1e-3) / 1e9, 1),
                                   "peak": peak, "unit": "GB/s",
                                   "frac": round(2 * n * k * 4 / (gram8_ms * 1e-3) / 1e9 / peak, 3),
                                   "bytes_per_launch": int(2 * n * k * 4),
                                   "note": "X read twice (column scales, then the digits)"},
            "sigma_over_sigma1_top10": [float(v) for v in s_ref[:10] / s_ref[0]],
            "gram_fp64_ms": round(gram64_ms, 4),
            "pod_value_uses": ("exact-product int8 tensor-core Gram (PodBasis default); the FP64 CUDA-core and "
                               "split-bf16 tensor-core Grams timed and checked beside it"),
            "x_mixed_vs_fp64": float(torch.linalg.norm(res["mixed"][1] - res["fp64"][1]) / torch.linalg.norm(res["fp64"][1]))}


def workload_gram(args):
    """The tensor-core Grams alone on a seeded random 1,382,976 x 64 FP32 panel (the snapshot set's
    size), L2 flushed before each timed launch: the exact-product int8 Gram (the headline of this
    line), the split-bf16 Gram and the FP64 CUDA-core Gram beside them, each against an FP64
    Gram of the same panel."""
    import torch
    from feab200.pod import gram_bf16x3, gram_fp64, gram_int8
    n, k = 1_382_976, 64
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn((n, k), generator=g, device="cuda", dtype=torch.float32)
    flush = L2Flush("cuda")
    ws = torch.empty(int(__import__("feab200")._lib.lib.feab_gram_workspace_bytes(n, k)), dtype=torch.uint8,
                     device="cuda")
    kernels = {"int8": lambda: gram_int8(X, check=False, workspace=ws),
               "bf16x3": lambda: gram_bf16x3(X, check=False, workspace=ws),
               "fp64": lambda: (gram_fp64(X, workspace=ws), None)}
    for _ in range(args.warmup):
        for fn in kernels.values():
            fn()
    times = {name: [] for name in kernels}
    out = {}
    for _ in range(args.steps):
        for name, fn in kernels.items():
            flush()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            G, f = fn()
            b.record()
            torch.cuda.synchronize()
            times[name].append(a.elapsed_time(b))
            if f is not None and int(f.item()):
                raise RuntimeError(f"gram_{name}: a bounded wait timed out on the device")
            out[name] = G
    ref = X.double().T @ X.double()
    scale = torch.sqrt(torch.outer(torch.diagonal(ref), torch.diagonal(ref)))
    peak, kind = measured_peak()
    res = {}
    for name in kernels:
        ms = statistics.mean(times[name])
        nbytes = n * k * 4 * (2 if name == "int8" else 1) + k * k * 8
        res[name] = {"ms": round(ms, 4), "max_rel_err_vs_fp64_product": float(((out[name] - ref).abs() / scale).max()),
                     "achieved_gbs": round(nbytes / (ms * 1e-3) / 1e9, 1), "bytes_per_launch": nbytes}
    ms = res["int8"]["ms"]
    nbytes = res["int8"]["bytes_per_launch"]
    return {"metric": "tensor-core exact-product (int8 digits) Gram X^T X time, 1382976 x 64 FP32", "value": ms,
            "unit": "ms",
            "roofline": {"bound": "hbm", "achieved": round(nbytes / (ms * 1e-3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(nbytes / (ms * 1e-3) / 1e9 / peak, 3), "bytes_per_launch": nbytes,
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs (of {kind})",
                         "note": "X is read twice (column scales, then the digits)"},
            "kernels": res, "timing": "CUDA events around each launch, L2 flushed before each"}


def workload_spmv(args):
    """The PCG's SpMV kernels alone on the 128x32x32 cantilever's K_ff (inputs resident, L2
    flushed before each timed launch): the sliced operator with FP64 and 48-bit values, and the
    CSR kernel; a few PCG iterations of each precision run first, so that a profiler sees the
    step kernels early."""
    import torch
    from feab200.device import DeviceMesh, pcg_solve
    c = build_workload(tuple(args.shape))
    dm = DeviceMesh(c.mesh.nodes, c.mesh.elements)
    op = dm.assemble(dm.element_stiffness(c.D), dm.pattern(c.fixed), want32=True)
    peak, kind = measured_peak()
    b = torch.as_tensor(c.F[c.free]).to(op.vals64.device)
    iters = {}
    for prec in ("mixed", "fp64"):
        _, info = pcg_solve(op, b, tol=0.0, maxiter=8, precision=prec)
        iters[prec] = info.iters
    out = {}
    for prec in ("mixed", "fp64", "fp32"):
        r = spmv_roofline(op, prec, max(1, args.spmv_reps), peak)
        r["peak_source"] = f"MEASURED_PEAKS.json hbm_gbs (of {kind})"
        out[prec] = r
    return {"metric": "PCG SpMV kernel time, 128x32x32 K_ff (n 418176, nnz 32348142), mixed 48-bit sliced",
            "value": out["mixed"]["launch_us"], "unit": "us", "roofline": out["mixed"],
            "roofline_fp64": out["fp64"], "roofline_fp32_csr": out["fp32"], "pcg_probe_iters": iters}


def recovery_bytes(n_nodes, n_elem):
    """Algorithmic bytes of one feab_hex8_recover call with every output: the element kernel reads
    the connectivity (32 B per element) and each node's coordinates and displacement once
    (48 B per node), writes the 8 corner records (448 B per element) and the element stress and
    von Mises (56 B per element); the node kernel reads the incidence lists (4 B per node +
    32 B per element), the connectivity again, the corner records (448 B per element) and writes
    the nodal stress and von Mises (56 B per node)."""
    return n_elem * (32 + 448 + 56 + 32 + 32 + 448) + n_nodes * (48 + 4 + 56)


def workload_recovery(args):
    """Stress recovery on the 128x32x32 cantilever after an FP64 solve: nodal and element stress and
    von Mises in one feab_hex8_recover call (kernel time, L2 flushed before each launch), the same
    through FESystem.stress + von_mises from host arrays, and the oracle on the host cores."""
    import torch
    import oracle as O
    from feab200 import _lib as L
    from feab200.device import DeviceMesh, DeviceStatus, pcg_solve
    c = build_workload(tuple(args.shape))
    X, el = c.mesh.nodes, c.mesh.elements
    dev = torch.device("cuda", torch.cuda.current_device())
    dm = DeviceMesh(X, el, device=dev)
    op = dm.assemble(dm.element_stiffness(c.D), dm.pattern(c.fixed))
    x, info = pcg_solve(op, torch.as_tensor(c.F[c.free]).to(dev), tol=1e-10, precision="fp64")
    u = torch.zeros(c.n_dof, dtype=torch.float64, device=dev)
    u[torch.as_tensor(c.free).to(dev)] = x
    N, E = len(X), len(el)
    topo = dm.topology()
    f64 = dict(dtype=torch.float64, device=dev)
    nodal, nvm, elem, evm = (torch.empty((N, 6), **f64), torch.empty(N, **f64), torch.empty((E, 6), **f64),
                             torch.empty(E, **f64))
    sbytes = int(L.lib.feab_hex8_recover_scratch_bytes(E))
    scratch = torch.empty(sbytes, dtype=torch.uint8, device=dev)
    st = DeviceStatus(dev)
    Dm = L.dmat(c.D)

    def launch():
        rc = L.lib.feab_hex8_recover(L.dptr(dm.coords), L.dptr(dm.conn), E, N, L.dptr(topo.inc_ptr),
                                     L.dptr(topo.inc_elem), Dm, L.dptr(u), L.dptr(nodal), L.dptr(nvm), L.dptr(elem),
                                     L.dptr(evm), L.dptr(scratch), sbytes, st.ptr(), dm.stream)
        L.raise_for(rc, "recovery")

    n0 = L.lib.feab_launch_count()
    for _ in range(max(3, args.warmup)):
        launch()
    torch.cuda.synchronize()
    st.check("recovery")
    flush = L2Flush(dev)
    times = []
    for _ in range(max(1, args.steps) * 4):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        launch()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) * 1e-3)
    launches = int(L.lib.feab_launch_count() - n0)
    t = statistics.mean(times)
    nbytes = recovery_bytes(N, E)
    peak, kind = measured_peak()
    # parity against the oracle on the same displacement
    uh = u.cpu().numpy()
    t0 = time.perf_counter()
    s_ref, e_ref = O.recover(X, el, uh, c.D)
    cpu_s = time.perf_counter() - t0
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    # through the public API from host arrays
    import feab200
    fs = feab200.FESystem(feab200.Mesh(nodes=X, elements=el), feab200.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(c.D)
    fs.stress(uh)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        S = fs.stress(uh)
        V = fs.von_mises(uh)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / 3
    return {"metric": f"hex8 stress recovery (nodal + element stress and von Mises), {'x'.join(map(str, args.shape))}",
            "value": round(t * 1e6, 2), "unit": "us", "n_nodes": N, "n_elements": E,
            "roofline": {"bound": "hbm", "achieved": round(nbytes / t / 1e9, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(nbytes / t / 1e9 / peak, 3), "bytes_per_launch": int(nbytes),
                         "kernels": "k_recover_elements + k_recover_nodes (one feab_hex8_recover call)",
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs (of {kind})"},
            "rel_err_vs_oracle": {"stress_nodes": rel(nodal.cpu().numpy(), s_ref),
                                  "stress_elements": rel(elem.cpu().numpy(), e_ref),
                                  "von_mises_nodes": rel(nvm.cpu().numpy(), O.von_mises(s_ref)),
                                  "fesystem_stress": rel(S.nodal, s_ref),
                                  "fesystem_von_mises": rel(np.asarray(V), O.von_mises(s_ref))},
            "e2e": {"value": round(e2e_ms, 2), "unit": "ms",
                    "path": "FESystem.stress + FESystem.von_mises from a host numpy displacement",
                    "h2d_bytes_per_step": 2 * 3 * N * 8, "d2h_bytes_per_step": N * 6 * 8 + N * 8},
            "cpu_baseline": {"value": round(cpu_s * 1e3, 1), "unit": "ms", "cores": os.cpu_count(), "kind": "port",
                             "sample": "oracle recover (NumPy einsum, all host threads) on the whole mesh, stress nodal "
                                       "+ element"},
            "gpu_launches": launches, "timing": "CUDA events around each call, L2 flushed before each"}


def workload_simp_oc(args):
    """The SIMP optimality-criteria loop on the 96x32x32 cantilever (E0 = 1, unit tip load,
    vf 0.4, p 3, rho_min 1e-3, move 0.2, filter radius 1.5 element lengths): time per iteration
    of topopt.topology_optimize_compliance (assembly, PCG to 1e-9, dC/drho, filter, OC), and the
    filter build, filter apply and OC update alone; the oracle's loop on a 24x8x8 mesh stands
    in for the CPU (its dense filter matrix does not fit at 98,304 elements)."""
    import torch
    import feab200
    import oracle as O
    from feab200 import cantilever, topopt
    c = cantilever.simp_cantilever(96, 32, 32)
    mesh = feab200.Mesh(nodes=c.mesh.nodes, elements=c.mesh.elements)
    fs = feab200.FESystem(mesh, feab200.Hex8Solid3D())
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    radius = 1.5 * 2.0 / 96
    kw = dict(p=3.0, rho_min=1e-3, move=0.2, filter_radius=radius, pcg_tol=1e-9)
    topopt.topology_optimize_compliance(fs, c.D, c.F, 0.4, n_iter=2, **kw)            # warm-up
    n_it = max(4, 2 * args.steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = topopt.topology_optimize_compliance(fs, c.D, c.F, 0.4, n_iter=n_it, tol=0.0, **kw)
    torch.cuda.synchronize()
    ms_iter = (time.perf_counter() - t0) * 1e3 / len(res["compliance_history"])
    dm = fs.device_mesh
    cent = topopt.element_centroids(dm)

    def ev(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            out = fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps, out

    build_ms, H = ev(lambda: topopt.build_filter_weights(cent, radius), 2)
    rho = torch.as_tensor(res["rho"]).to(dm.device)
    dc = -torch.rand(dm.n_elem, dtype=torch.float64, device=dm.device)
    filt_ms, _ = ev(lambda: topopt.apply_sensitivity_filter(H, rho, dc))
    oc_ms, _ = ev(lambda: topopt._oc_device(rho, dc, 0.4, 0.2, 1e-3, 1.0, 1e-4, 100))
    # CPU: the oracle's loop (dense filter, sparse direct solves) on 24x8x8
    cs = cantilever.simp_cantilever(24, 8, 8)
    t0 = time.perf_counter()
    _, hist_cpu, _ = O.topology_optimize_compliance(cs.mesh.nodes, cs.mesh.elements, cs.D, cs.fixed, cs.F, 0.4, p=3.0,
                                                    rho_min=1e-3, move=0.2, n_iter=3, filter_radius=1.5 * 2.0 / 24,
                                                    tol=0.0)
    cpu_ms = (time.perf_counter() - t0) * 1e3 / len(hist_cpu)
    h = res["compliance_history"]
    return {"metric": "SIMP optimality-criteria iteration time (assemble + PCG + dC/drho + filter + OC), 96x32x32 hex8",
            "value": round(ms_iter, 2), "unit": "ms", "iterations_timed": len(h), "n_elements": dm.n_elem,
            "filter_nnz": H.nnz, "filter_build_ms": round(build_ms, 3), "filter_apply_ms": round(filt_ms, 4),
            "oc_update_ms": round(oc_ms, 4), "compliance_first_last": [h[0], h[-1]],
            "volume_fraction_final": float(np.mean(res["rho"])),
            "cpu_baseline": {"value": round(cpu_ms, 1), "unit": "ms per iteration", "cores": os.cpu_count(),
                             "kind": "port", "sample": "oracle loop (dense filter, SciPy sparse direct solve) on "
                                                       "24x8x8, 3 iterations"}}


def workload_elements(args):
    """The element-matrix kernels alone on the 128x32x32 cantilever (packed layout, L2 flushed
    before each launch): Hex8Solid3D and Hex8SolidBbar.  Work per element, counted from the
    contractions: plain 8 x 36 x (54 + 27) FMA (D B for the 3 non-zeros of each B column, then
    B^T (D B)); B-bar 8 x 36 x 162 FMA (full 6 x 3 column blocks), plus the Jacobian per Gauss
    point; HBM: 324 doubles written per element."""
    import torch
    from feab200.device import DeviceMesh
    c = build_workload(tuple(args.shape))
    dm = DeviceMesh(c.mesh.nodes, c.mesh.elements)
    E = dm.n_elem
    flush = L2Flush(dm.device)
    out = {}
    for name, bbar, fma in (("plain", False, 8 * 36 * 81), ("bbar", True, 8 * 36 * 162)):
        dm.element_stiffness(c.D, bbar=bbar)
        times = []
        for _ in range(max(3, args.steps)):
            flush()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            dm.element_stiffness(c.D, bbar=bbar, status=_NO_CHECK)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b) * 1e-3)
        t = statistics.mean(times)
        out[name] = {"us": round(t * 1e6, 1), "fp64_tflops": round(2 * fma * E / t / 1e12, 2),
                     "write_gbs": round(324 * 8 * E / t / 1e9, 1)}
    return {"metric": f"hex8 element stiffness kernel time (Hex8Solid3D and Hex8SolidBbar), "
                      f"{'x'.join(map(str, args.shape))}, packed layout",
            "value": out["plain"]["us"], "unit": "us", "n_elements": E, "kernels": out,
            "timing": "CUDA events around each launch, L2 flushed before each"}


def workload_modal(args):
    """The 6 lowest natural frequencies of the cantilever (2.0 x 0.4 x 0.4 m, steel, x = 0 clamped)
    meshed 64x16x16 (52,224 free DOFs): consistent mass + FESystem.solve_modal (GPU block
    subspace iteration with block-PCG inner solves).  The oracle (the reference's shift-invert
    eigsh with a sparse LU) runs on the 32x8x8 mesh, where the GPU solve is repeated for the
    frequency comparison."""
    import torch
    import feab200
    import oracle as O

    def system(shape):
        nodes, el = O.box_mesh(2.0, 0.4, 0.4, *shape)
        mesh = feab200.Mesh(nodes=nodes, elements=el)
        fs = feab200.FESystem(mesh, feab200.Hex8Solid3D(), sparse=True)
        fs.assemble_stiffness(O.D_solid3d(210e9, 0.3))
        fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
        fs.assemble_mass(7850.0 * np.eye(3))
        return fs, nodes, el

    fs, _, _ = system((64, 16, 16))
    fs.solve_modal(6)                                                   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f, _ = fs.solve_modal(6)
    torch.cuda.synchronize()
    gpu_ms = (time.perf_counter() - t0) * 1e3
    iters = fs.last_modal_iterations
    fs_s, nodes, el = system((32, 8, 8))
    f_s, _ = fs_s.solve_modal(6)
    free = fs_s.free_dofs
    Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(nodes[el], O.D_solid3d(210e9, 0.3)), el,
                                         3 * len(nodes)), free)
    Mff = O.reduce_free(O.structural_csr(O.hex8_element_mass(nodes[el], 7850.0 * np.eye(3)), el, 3 * len(nodes)), free)
    t0 = time.perf_counter()
    f_ref, _ = O.modal(Kff, Mff, 6)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    return {"metric": "hex8 modal solve time (6 lowest modes, consistent mass), 64x16x16 cantilever",
            "value": round(gpu_ms, 1), "unit": "ms", "free_dofs": int(fs.reduced_operator(want32=False).n),
            "subspace_iterations": iters, "freq_hz": [float(v) for v in f],
            "rel_err_vs_eigsh_32x8x8": float(np.max(np.abs(f_s - f_ref) / f_ref)),
            "cpu_baseline": {"value": round(cpu_ms, 1), "unit": "ms", "cores": os.cpu_count(), "kind": "port",
                             "sample": "oracle shift-invert eigsh (SciPy, sparse LU) on the 32x8x8 mesh; the "
                                       "64x16x16 mesh takes about a minute on 8 cores"}}


def workload_block_step(args):
    """The block-PCG step on the 128x32x32 cantilever with a 64-column panel of seeded random
    right-hand sides (the snapshot case's width), FP64 and mixed: the time of one step (three
    kernels) from CUDA events over runs of 4 and 4 + 8 * steps steps at tol 0 (no column
    converges; the difference removes setup and capture), at the tuned launch shape; and the
    block SpMM alone (feab_block_spmm, the same group SpMM code as the step's kernel A) with L2
    flushed before each launch, against the algorithmic bytes of one block SpMM:
    nnz * (8 + 4) + 4 (n + 1) + 2 n k * 8."""
    import torch
    from feab200 import cantilever
    from feab200.batched import ProblemBatch, block_pcg, tuned_block_shape
    from feab200.panel import block_spmm
    c = cantilever.random_tip_cantilever(*args.shape)
    b = ProblemBatch([(c.mesh.nodes, c.mesh.elements, c.D, c.fixed, c.F)])
    op = b.assemble()
    k = 64
    B = torch.as_tensor(np.random.default_rng(0).standard_normal((op.n, k))).cuda()
    long = 4 + 8 * max(1, args.steps)
    out = {}
    for prec in ("fp64", "mixed"):
        shape = tuned_block_shape(op, b.row_bounds, B, [k], prec)

        def run(m):
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            block_pcg(op, b.row_bounds, B, [k], tol=0.0, maxiter=m, precision=prec, max_groups=shape.item_groups,
                      tile_width=shape.tile_width, tune=False, node_tiles=shape.node_tiles)
            e.record()
            e.synchronize()
            return a.elapsed_time(e)
        for _ in range(max(1, args.warmup)):
            run(4)
        t4, tl = min(run(4) for _ in range(2)), min(run(long) for _ in range(2))
        out[prec] = {"us_per_step": round((tl - t4) * 1e3 / (long - 4), 1), "item_groups": shape.item_groups,
                     "tile_width": shape.tile_width, "node_tiles": shape.node_tiles}
    flush = L2Flush(op.vals64.device)
    Y = torch.empty_like(B)
    block_spmm(op, B, out=Y)
    times = []
    for _ in range(max(3, args.steps)):
        flush()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        block_spmm(op, B, out=Y)
        e.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(e) * 1e-3)
    t = statistics.mean(times)
    nbytes = op.nnz * 12 + 4 * (op.n + 1) + 2 * op.n * k * 8
    flops = 2 * op.nnz * k
    peak, kind = measured_peak()
    return {"metric": f"block-PCG step time, {'x'.join(map(str, args.shape))} cantilever, 64 right-hand sides",
            "value": out["fp64"]["us_per_step"], "unit": "us", "steps_timed": long - 4, "step": out,
            "mixed_speedup_vs_fp64": round(out["fp64"]["us_per_step"] / out["mixed"]["us_per_step"], 3),
            "block_spmm": {"us": round(t * 1e6, 1), "bytes": int(nbytes), "fp64_gflop": round(flops / 1e9, 2),
                           "roofline": {"bound": "hbm", "achieved": round(nbytes / t / 1e9, 1), "peak": peak,
                                        "unit": "GB/s", "frac": round(nbytes / t / 1e9 / peak, 3),
                                        "peak_source": f"MEASURED_PEAKS.json hbm_gbs (of {kind})"},
                           "fp64_tflops": round(flops / t / 1e12, 2)},
            "timing": "step: CUDA events over whole runs; SpMM: CUDA events around each launch, L2 flushed before each"}


def workload_direct(args):
    """The direct solve of solve_static(method=None) (the reference's SuperLU splu,
    _sparse_lu_solve) as a banded Cholesky on the GPU, on the random-tip cantilever at 64x16x16
    and at --shape: ordering + band assembly + factorisation, and one solve, with the relative
    residual and the difference from a Jacobi-PCG solve at 1e-12.  The reference's splu at
    64x16x16 took 59.6 s on the survey container's 8 cores; at 128x32x32 its fill does not fit."""
    import torch
    from feab200 import cantilever
    from feab200.device import DeviceMesh, pcg_solve, spmv
    from feab200.direct import BandCholesky
    out = {}
    for shape in ((64, 16, 16), tuple(args.shape)):
        c = cantilever.random_tip_cantilever(*shape)
        dm = DeviceMesh(c.mesh.nodes, c.mesh.elements)
        op = dm.assemble(dm.element_stiffness(c.D), dm.pattern(c.fixed), want32=False)
        b = torch.as_tensor(c.F[c.free]).to(op.vals64.device)
        fac_ms, solve_ms = [], []
        for _ in range(max(1, args.steps)):
            op._direct = None
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fac = op.direct_factor(coords=c.mesh.nodes)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            x = fac.solve(b)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            fac_ms.append(1e3 * (t1 - t0))
            solve_ms.append(1e3 * (t2 - t1))
        rel = float(torch.linalg.norm(b - spmv(op, x, lanes_per_group=16)) / torch.linalg.norm(b))
        xp, info = pcg_solve(op, b, tol=1e-12)
        nt, nb = fac.band.n_tiles, fac.band.bands
        gflop = 2 * nt * nb * (nb + 1) / 2 * 64 ** 3 / 1e9            # the trailing updates dominate
        out["x".join(map(str, shape))] = {
            "n": op.n, "ordering": fac.ordering, "bandwidth": fac.bandwidth, "band_gb": round(fac.storage.numel() / 1e9, 2),
            "factor_ms": round(min(fac_ms), 1), "solve_ms": round(min(solve_ms), 1),
            "update_gflop": round(gflop, 1), "update_tflops": round(gflop / min(fac_ms), 2),
            "relres": rel, "vs_pcg_1e-12": float(torch.linalg.norm(x - xp) / torch.linalg.norm(xp)),
            "pivot_ratio": fac.pivots[0] / fac.pivots[1]}
        del fac, op, dm
        torch.cuda.empty_cache()
    key = "x".join(map(str, args.shape))
    return {"metric": f"direct solve (banded Cholesky) time, {key} cantilever", "value": out[key]["factor_ms"] +
            out[key]["solve_ms"], "unit": "ms", "cases": out,
            "timing": "host clock around synchronised calls; factor includes ordering, band assembly and factorisation",
            "cpu_reference_note": "SuperLU splu (_sparse_lu_solve) at 64x16x16: 59.6 s on the survey container's 8 "
                                  "cores; infeasible at 128x32x32 (fill)"}


class _NoCheck:
    """A device status that is never read back, so a timed element-matrix launch has no sync."""

    def __init__(self):
        self.t = None

    def ptr(self):
        import torch
        if self.t is None:
            self.t = torch.zeros(2, dtype=torch.int64, device="cuda")
        from feab200 import _lib as L
        return L.dptr(self.t)


_NO_CHECK = _NoCheck()


# ----------------------------------------------------------------------------- main
def headline_config(shape, tol, n_free, nnz, world):
    """The workload identity shared by the GPU line and the reference (CPU) line."""
    return {"workload": (f"cantilever hex8 {shape[0]}x{shape[1]}x{shape[2]} (2.0x0.4x0.4 m, random tip traction, "
                         f"x=0 clamped): topology+pattern+Ke+CSR assembly + Jacobi-PCG (rel residual {tol:g}) "
                         f"+ SIMP dC/drho"),
            "n_free": int(n_free), "nnz": int(nnz), "tol": tol,
            "l2": "inputs larger than L2 (K_ff FP64 values alone exceed 126 MB); no flush",
            "parallelism": f"replicas x{world}"}


def reference_arm(args):
    """``--impl reference``: the reference path's CPU implementation (the oracle restatement of
    fea_engine's NumPy/SciPy code; the reference itself is not on the GPU box) on the host cores,
    for the headline workload.  Every step is a whole step (assembly + PCG to tol + dC/drho),
    none extrapolated.  A step takes about a minute, so steps run until a time budget
    (FEAB_REF_BUDGET_S, default 150 s) would be exceeded, at least one; the line reports the
    steps and warm-up that actually ran, and the requested ones beside them.  Under torchrun
    only rank 0 works; the other ranks exit at once.  Nothing here loads the CUDA library."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.workload != "cantilever":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the headline cantilever "
                                                              "workload only"}), flush=True)
        return
    sys.path.insert(0, ROOT)
    from oracle import workloads
    shape = tuple(args.shape)
    w = workloads.random_tip_cantilever(*shape)
    budget = float(os.environ.get("FEAB_REF_BUDGET_S", "150"))
    runs = []
    t_start = time.perf_counter()
    while True:
        r = oracle_step(w, args.tol)
        runs.append(r)
        if len(runs) >= args.steps or time.perf_counter() - t_start + r["times"]["step_s"] > budget:
            break
    ms = [1e3 * r["times"]["step_s"] for r in runs]
    v = statistics.mean(ms)
    phases = {k: round(1e3 * statistics.mean(r["times"][k] for r in runs), 1) for k in ("assembly_s", "pcg_s", "grad_s")}
    last = runs[-1]
    cores = os.cpu_count()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms", "n_gpus": world,
        "steps": len(runs), "warmup": 0, "ms_per_step": round(v, 1), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(shape, args.tol, len(w["free"]), last["Kff"].nnz, world),
        "precision": "FP64 throughout (the reference recurrence)",
        "requested": {"steps": args.steps, "warmup": args.warmup,
                      "note": f"whole CPU steps until a {budget:.0f} s budget; no warm-up step (nothing to warm on "
                              f"the CPU path), no extrapolation"},
        "step_ms": [round(m, 1) for m in ms], "phases_ms": phases, "iters": last["iters"],
        "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": cores, "kind": "port",
                         "sample": (f"{len(runs)} whole step(s) of the oracle (NumPy/SciPy restatement of the reference "
                                    f"path; SciPy's CSR SpMV is single-threaded, NumPy's BLAS uses up to {cores} "
                                    f"threads): assembly {phases['assembly_s'] / 1e3:.2f} s + PCG to {args.tol:g} "
                                    f"({last['iters']} iterations) {phases['pcg_s'] / 1e3:.2f} s + dC/drho "
                                    f"{phases['grad_s'] / 1e3:.2f} s")},
        "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    shape = tuple(args.shape)
    # the oracle job (a 'spawn' child, 1 GPU runs only) starts after the GPU measurements, so its
    # host threads neither slow the host side of the timed GPU steps nor are slowed by it
    want_oracle = (args.workload == "cantilever" and int(os.environ.get("WORLD_SIZE", "1")) == 1
                   and not args.no_cpu_baseline)
    import torch
    world, rank, local = dist_setup(args.gpus)
    args.world, args.rank = world, rank
    if args.workload != "cantilever":
        fn = {"simp": workload_simp, "batch": workload_batch, "snapshot": workload_snapshot,
              "gram": workload_gram, "spmv": workload_spmv, "recovery": workload_recovery,
              "simp_oc": workload_simp_oc, "elements": workload_elements, "modal": workload_modal,
              "block_step": workload_block_step, "direct": workload_direct}[args.workload]
        line = fn(args)
        line.update({"n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                     "data": "synthetic", "workload": args.workload})
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    c = build_workload(shape)
    dev = torch.device("cuda", torch.cuda.current_device())
    prob = DeviceProblem(c, dev)
    clocks = ClockSampler(gpu_index(local))
    # plain FP64 first, then mixed (the headline)
    clocks.start()
    clocks.wait_first_sample()
    ms64, x64, dc64, info64, op64, _, each64 = time_steps(prob, "fp64", args.tol, args.steps, args.warmup, world)
    ms32, x32, dc32, info32, op, launches, each32 = time_steps(prob, "mixed", args.tol, args.steps, args.warmup,
                                                              world)
    clk = clocks.stop()
    # the FP32-everything variant, one solve, for reference
    t0 = time.perf_counter()
    xf, _, infof, _ = prob.step("fp32", args.tol)
    torch.cuda.synchronize()
    msf = (time.perf_counter() - t0) * 1e3
    # a tight GPU FP64 solve of the same system (secondary accuracy reference)
    from feab200.device import pcg_solve
    xt, infot = pcg_solve(op64, prob.Ff, tol=1e-13, precision="fp64")
    rel_t = lambda a: float(torch.linalg.norm(a - xt) / torch.linalg.norm(xt))  # noqa: E731
    dc_err = float(torch.linalg.norm(dc32 - dc64) / torch.linalg.norm(dc64))
    peak, peak_kind = measured_peak()
    roof = spmv_roofline(op, "mixed", args.spmv_reps, peak)
    roof64 = spmv_roofline(op64, "fp64", args.spmv_reps, peak)
    for r in (roof, roof64):
        r["peak_source"] = f"MEASURED_PEAKS.json hbm_gbs (of {peak_kind})"
    try:  # DRAM bytes of the same kernel from one ncu capture (profiles/)
        tr = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))
        for r, prec in ((roof, "mixed"), (roof64, "fp64")):
            t = tr.get(f"cantilever {shape[0]}x{shape[1]}x{shape[2]}", {}).get(prec)
            if t:
                r["traffic"] = t["dram_bytes"]
                r["traffic_kernel"] = t["kernel"]
    except (OSError, ValueError, KeyError):
        pass
    pcg_iter = {prec: pcg_iteration_roofline(o, prob.Ff, args.tol, prec, peak)
                for prec, o in (("mixed", op), ("fp64", op64))}
    e2e_ms, h2d, d2h = e2e_steps(c, "mixed", args.tol, args.e2e_steps, 2)
    e2e_ms = max_over_ranks(e2e_ms, world)
    cpu, parity = None, None
    rel = {"mixed_vs_fp64_tight": rel_t(x32), "fp64_vs_fp64_tight": rel_t(x64), "fp32_vs_fp64_tight": rel_t(xf),
           "dc_mixed_vs_fp64": dc_err, "tight_tol": 1e-13, "mixed_relres_fp64": info32.relres}
    if want_oracle:
        ref, why = OracleRun(shape, args.tol).result(timeout=1200)
        if ref is None:
            parity = {"error": why}
        else:
            parity = parity_vs_oracle(ref, op64, {"mixed": x32, "fp64": x64, "fp32": xf}, dc32)
            rel.update({"mixed_vs_oracle": parity["u_rel_err"]["mixed"], "fp64_vs_oracle": parity["u_rel_err"]["fp64"],
                        "fp32_vs_oracle": parity["u_rel_err"]["fp32"], "dc_mixed_vs_oracle": parity["dc_rel_err"],
                        "oracle_tol": OracleRun.SOLVE_TOL})
            t = ref["times"]
            cpu = {"value": round(1e3 * t["step_s"], 1), "unit": "ms", "cores": ref["threads"], "kind": "port",
                   "sample": (f"one whole step (not extrapolated) of the oracle (NumPy/SciPy restatement of the "
                              f"reference path; SciPy's CSR SpMV is single-threaded) on the same workload, in a "
                              f"separate process after the GPU measurements: assembly {t['assembly_s']:.2f} s + "
                              f"PCG to {args.tol:g} ({ref['iters_at_tol']} iterations) {t['pcg_s']:.2f} s + dC/drho "
                              f"{t['grad_s']:.2f} s")}
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms32, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms32, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": headline_config(shape, args.tol, op.n, op.nnz, world),
            "precision": ("mixed: SpMV on 48-bit (36-bit mantissa) values in difference form, FP64 vectors and "
                          "scalars, FP64 reliable residual replacement"),
            "plain_fp64_ms": round(ms64, 3), "mixed_speedup_vs_fp64": round(ms64 / ms32, 3),
            "step_ms_each": {"mixed": each32, "fp64": each64},
            "fp32_everything_ms": round(msf, 3),
            "iters": {"mixed": info32.iters, "fp64": info64.iters, "fp32": infof.iters,
                      "reliable_updates": info32.reliable_updates},
            "rel_err": rel,
            "parity_vs_oracle": parity,
            "roofline": roof,
            "roofline_fp64": roof64,
            "pcg_iteration": pcg_iter,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_ms, 2), "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "FESystem + topopt from host numpy (pageable) arrays"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
