"""Parity with the oracle at the benchmark configurations' own sizes.

The small-mesh parity tests pin the CUDA path to the reference's golden vectors; these repeat
the comparisons at the sizes the benchmark quotes, against the oracle (the NumPy/SciPy
restatement of the reference path, itself pinned to the golden vectors):

- 128 x 32 x 32 random-tip cantilever (418,176 free DOFs): CSR row_ptr / col_idx bit for bit
  against COO -> CSR + K[free, free] (vectorized_assembly.py:217-288, solver.py:1977-1978),
  K_ff values within 1e-12 normwise, and the FP64 and mixed-precision solutions within 1e-8 of
  the oracle's FP64 Jacobi-PCG run to a relative residual of 1e-12
  (iterative_solvers.py:434-481);
- 96 x 32 x 32 SIMP cantilever (98,304 elements): dC/drho through the autograd Function
  against the closed form on the oracle's u (topopt.py:161-177), and against central
  differences with h = 1e-6 at 32 random elements (the check of
  fea_engine/tests/test_topopt.py:70-95);
- the 256-problem uneven batch: a sample of problems, every load column against independent
  oracle solves (fea_engine/tests/test_batched_solve.py:66-115 compares batched with
  one-at-a-time solves the same way);
- 192 x 48 x 48 (1,382,976 free DOFs, 108.6 M nonzeros): the CSR pattern bit for bit.

Each oracle solve runs once per session (module fixtures).  Tolerances are the parity bars:
CSR exact, K 1e-12 normwise, displacements 1e-8 relative 2-norm.
"""
import numpy as np
import pytest
import torch

import oracle as O
from oracle import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

KTOL = 1e-12
UTOL = 1e-8
BENCH_TOL = 1e-9          # the benchmark's PCG tolerance
ORACLE_TOL = 1e-12        # the oracle solution's relative residual


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _oracle_solve(Kff, b, tol=ORACLE_TOL):
    hist = []
    x, iters, _ = O.preconditioned_cg(Kff, b, O.jacobi_inverse_diagonal(Kff), tol=tol, history=hist)
    at = {t: next((k for k, (_, r) in enumerate(hist, 1) if r < t), None) for t in (1e-8, 1e-9, 1e-10)}
    return x, iters, at


# ----------------------------------------------------------------------------- 128 x 32 x 32
@pytest.fixture(scope="module")
def cantilever_128x32x32():
    w = W.random_tip_cantilever(128, 32, 32)
    X, el = w["nodes"], w["elements"]
    Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(X[el], w["D"]), el, w["n_dof"]), w["free"])
    b = w["F"][w["free"]]
    x, iters, at = _oracle_solve(Kff, b)
    return w, Kff, x, at


def test_csr_pattern_and_values_at_128x32x32(cantilever_128x32x32):
    from feab200.device import DeviceMesh
    w, Kff, _, _ = cantilever_128x32x32
    dm = DeviceMesh(w["nodes"], w["elements"])
    op = dm.assemble(dm.element_stiffness(w["D"]), dm.pattern(w["fixed"]), want32=False)
    assert (op.n, op.nnz) == (418176, 32348142) == (Kff.shape[0], Kff.nnz)
    assert np.array_equal(op.pattern.row_ptr.cpu().numpy(), Kff.indptr)
    assert np.array_equal(op.pattern.col_idx.cpu().numpy(), Kff.indices)
    v = op.vals64.cpu().numpy()
    big = np.abs(Kff.data).max()
    assert np.abs(v - Kff.data).max() / big < KTOL
    sel = np.abs(Kff.data) > 1e-6 * big          # entry-wise where entries do not cancel to ~0
    assert np.max(np.abs(v - Kff.data)[sel] / np.abs(Kff.data)[sel]) < 1e-11
    d = Kff.diagonal()
    assert np.abs(op.dinv64.cpu().numpy() - 1.0 / d).max() * d.min() < KTOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solution_vs_oracle_at_128x32x32(cantilever_128x32x32, precision):
    from feab200.device import DeviceMesh, pcg_solve
    w, _, x_ref, at = cantilever_128x32x32
    dm = DeviceMesh(w["nodes"], w["elements"])
    op = dm.assemble(dm.element_stiffness(w["D"]), dm.pattern(w["fixed"]), want32=False)
    x, info = pcg_solve(op, w["F"][w["free"]], tol=BENCH_TOL, precision=precision)
    assert info.status == 0, info
    assert _rel(x.cpu().numpy(), x_ref) < UTOL
    if precision == "fp64":   # the reference recurrence: the same iteration count as the oracle's
        assert abs(info.iters - at[BENCH_TOL]) <= 2, (info.iters, at)


# ----------------------------------------------------------------------------- 96 x 32 x 32 SIMP
@pytest.fixture(scope="module")
def simp_96x32x32():
    w = W.simp_cantilever(96, 32, 32)
    X, el, rho = w["nodes"], w["elements"], w["rho"]
    ke = O.hex8_element_stiffness(X[el], w["D"])
    s = O.simp_scale(rho, 3.0, 1e-9)
    Kff = O.reduce_free(O.structural_csr(ke * s[:, None, None], el, w["n_dof"]), w["free"])
    u_free, _, _ = _oracle_solve(Kff, w["F"][w["free"]])
    u = np.zeros(w["n_dof"])
    u[w["free"]] = u_free
    dc_ref = O.compliance_sensitivity_closed_form(ke, el, u, rho, 3.0, 1e-9)
    return w, ke, Kff, dc_ref


def _simp_problem(w, precision, tol):
    from feab200 import topopt
    from feab200.device import DeviceMesh
    dm = DeviceMesh(w["nodes"], w["elements"])
    return topopt.SimpProblem(dm, w["D"], w["free"], penal=3.0, rho_min=1e-9, tol=tol, precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_simp_gradient_vs_closed_form_at_96x32x32(simp_96x32x32, precision):
    w, _, _, dc_ref = simp_96x32x32
    prob = _simp_problem(w, precision, BENCH_TOL)
    dev = prob.dm.device
    f = torch.as_tensor(w["F"][w["free"]]).to(dev)
    rho = torch.as_tensor(w["rho"]).to(dev).requires_grad_(True)
    torch.dot(f, prob(rho, f)).backward()
    assert _rel(rho.grad.cpu().numpy(), dc_ref) < UTOL


class _Compliance:
    """C(rho) to ~1e-18 relative, for finite differences of single-element perturbations.

    u is the GPU's FP64 solution of K(rho) u = f (relative residual 1e-13); C is evaluated as
    the stationary form f.u + r.u with r = f - K(rho) u formed in extended precision on the host
    (80-bit long double): K(rho0) from the oracle, plus the perturbed element's term
    (s(rho_e) - s(rho0_e)) ke_e u_e.  The stationary form's error is quadratic in the solve
    error, and the extended-precision residual removes the FP64 cancellation in K u, so
    differences of 1e-11 C over h = 1e-6 are resolved."""

    def __init__(self, w, ke, Kff):
        self.w, self.ke = w, ke
        self.data = Kff.data.astype(np.longdouble)
        self.indices, self.starts = Kff.indices, Kff.indptr[:-1]
        self.f = w["F"][w["free"]].astype(np.longdouble)
        pos = np.full(w["n_dof"], -1)
        pos[w["free"]] = np.arange(len(w["free"]))
        self.pos = pos                      # DOF -> free row, -1 if fixed
        self.prob = _simp_problem(w, "fp64", 1e-13)
        self.f_t = torch.as_tensor(w["F"][w["free"]]).to(self.prob.dm.device)

    def __call__(self, rho, e):
        u = self.prob.solve_free(torch.as_tensor(rho).to(self.prob.dm.device), self.f_t).cpu().numpy()
        assert self.prob.last_info.status == 0
        ul = u.astype(np.longdouble)
        Ku = np.add.reduceat(self.data * ul[self.indices], self.starts)
        ds = O.simp_scale(rho[e], 3.0, 1e-9) - O.simp_scale(self.w["rho"][e], 3.0, 1e-9)
        g = O.global_dofs(self.w["elements"][e:e + 1])[0]
        rows = self.pos[g]
        ue = np.where(rows >= 0, ul[np.maximum(rows, 0)], 0)
        Ke_u = (self.ke[e].astype(np.longdouble) @ ue) * np.longdouble(ds)
        np.add.at(Ku, rows[rows >= 0], Ke_u[rows >= 0])
        r = self.f - Ku
        return float(np.dot(self.f, ul) + np.dot(r, ul))


def test_simp_gradient_vs_central_differences_h1e6_at_96x32x32(simp_96x32x32):
    w, ke, Kff, dc_ref = simp_96x32x32
    prob = _simp_problem(w, "mixed", BENCH_TOL)
    dev = prob.dm.device
    f = torch.as_tensor(w["F"][w["free"]]).to(dev)
    rho = torch.as_tensor(w["rho"]).to(dev).requires_grad_(True)
    torch.dot(f, prob(rho, f)).backward()
    grad = rho.grad.cpu().numpy()
    comp = _Compliance(w, ke, Kff)
    h = 1e-6
    elems = np.random.default_rng(0).choice(len(w["rho"]), 32, replace=False)
    fd = []
    for e in elems:
        rp, rm = w["rho"].copy(), w["rho"].copy()
        rp[e] += h
        rm[e] -= h
        fd.append((comp(rp, e) - comp(rm, e)) / (2 * h))
    fd = np.array(fd)
    assert _rel(grad[elems], fd) < 1e-4
    big = np.abs(fd) > 1e-2 * np.abs(fd).max()
    assert np.max(np.abs(grad[elems] - fd)[big] / np.abs(fd)[big]) < 1e-3
    assert _rel(dc_ref[elems], fd) < 1e-4


# ----------------------------------------------------------------------------- uneven batch
def test_uneven_batch_sample_vs_independent_oracle_solves():
    from feab200 import cantilever
    from feab200.batched import ProblemBatch
    probs = cantilever.batch_cantilevers(256)
    batch = ProblemBatch([(p.mesh.nodes, p.mesh.elements, p.D, p.fixed, p.F) for p in probs])
    sols = {prec: batch.solve(tol=BENCH_TOL, precision=prec) for prec in ("fp64", "mixed")}
    for prec, (_, res) in sols.items():
        assert (res.status == 0).all(), prec
    rng = np.random.default_rng(11)
    sizes = np.array([len(p.free) for p in probs])
    sample = sorted(set(rng.choice(len(probs), 6, replace=False).tolist()) | {int(sizes.argmax())})
    for i in sample:
        p = probs[i]
        X, el = p.mesh.nodes, p.mesh.elements
        Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(X[el], p.D), el, 3 * len(X)), p.free)
        for c in range(min(4, p.F.shape[1])):
            ref, _, _ = _oracle_solve(Kff, p.F[p.free, c])
            for prec, (U, _) in sols.items():
                assert _rel(U[i][p.free, c], ref) < UTOL, (i, c, prec)


# ----------------------------------------------------------------------------- 192 x 48 x 48
def test_csr_pattern_bit_exact_at_192x48x48():
    from feab200.device import DeviceMesh
    nodes, el = O.box_mesh(2.0, 0.4, 0.4, 192, 48, 48)
    fixed = O.fixed_dofs_on_plane(nodes)
    free = O.free_dofs(3 * len(nodes), fixed)
    indptr, indices = O.structural_pattern(el, 3 * len(nodes), free)
    pat = DeviceMesh(nodes, el).pattern(fixed)
    assert (pat.n, pat.nnz) == (1382976, 108615150) == (len(indptr) - 1, len(indices))
    assert np.array_equal(pat.row_ptr.cpu().numpy(), indptr)
    assert np.array_equal(pat.col_idx.cpu().numpy(), indices)
