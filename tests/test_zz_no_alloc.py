"""The allocation-free PCG entry point (feab_pcg_solve_noalloc) against the allocating one.

Some callers cannot allocate device memory -- a host whose own pool owns all device memory, a
thread that must not block on the device synchronisation an allocation can cause, or an
environment that forbids allocation after start-up.  feab_pcg_solve_noalloc serves them with
its workspace in a fixed array inside the library.  This test calls it through the C ABI twice
in a row (the array keeps the previous call's contents, so the second call checks that every
call starts from a clean state) and compares each result with feab_pcg_solve on the same
system, within the displacement tolerance the parity tests use.  The file name makes pytest
collect it last; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

UTOL = 1e-8   # displacements, relative 2-norm (as in the parity tests)


def _system(golden):
    from feab200.device import DeviceMesh
    g = golden("cantilever_20x4x4")
    dm = DeviceMesh(g["nodes"], g["elements"])
    op = dm.assemble(dm.element_stiffness(g["D"]), dm.pattern(g["fixed"]), want32=False)
    return g, op


def _noalloc(op, b, tol, maxiter=0):
    from feab200 import _lib as L
    dev = op.vals64.device
    x = torch.full((op.n,), np.nan, dtype=torch.float64, device=dev)   # garbage in the output
    csr = op.csr_struct()
    prm = L.PcgParams(tol, maxiter, L.PREC_FP64, 0.1, 16, 1, 16, 0)
    res = L.PcgResult()
    rc = L.lib.feab_pcg_solve_noalloc(C.byref(csr), L.dptr(op.dinv64), L.dptr(b), None, L.dptr(x), C.byref(prm),
                                     C.byref(res), L.stream_ptr(dev))
    return rc, x, res


def test_noalloc_pcg_matches_allocating_entry_point(golden):
    from feab200 import _lib as L
    from feab200.device import pcg_solve
    g, op = _system(golden)
    b = torch.as_tensor(g["Ff"]).to(op.vals64.device)
    # the allocating entry point on the same CSR SpMV kernel, so the iterates agree bit for bit
    x_ref, info = pcg_solve(op, b, tol=1e-10, precision="fp64", lanes_per_group=16, layout="csr")
    assert info.status == 0
    u_lu = g["U_lu"][g["free"]]              # the reference's own SuperLU solution
    for _ in range(2):                       # two calls in a row share the fixed scratch
        rc, x, res = _noalloc(op, b, 1e-10)
        assert rc == L.FEAB_OK and res.status == L.FEAB_OK
        assert res.iters == info.iters
        err = float(torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref))
        assert err < UTOL, err
        xh = x.cpu().numpy()
        assert np.linalg.norm(xh - u_lu) / np.linalg.norm(u_lu) < UTOL
    # a second, different right-hand side: no state leaks from the previous call
    b2 = torch.as_tensor(np.random.default_rng(1).standard_normal(op.n)).to(op.vals64.device)
    x2_ref, _ = pcg_solve(op, b2, tol=1e-10, precision="fp64", lanes_per_group=16, layout="csr")
    rc, x2, res = _noalloc(op, b2, 1e-10)
    assert rc == L.FEAB_OK
    assert float(torch.linalg.norm(x2 - x2_ref) / torch.linalg.norm(x2_ref)) < UTOL


def test_noalloc_rejects_sizes_beyond_its_scratch(golden):
    from feab200 import _lib as L
    g, op = _system(golden)
    csr = op.csr_struct()
    csr.n = L.lib.feab_pcg_noalloc_max_n() + 1          # checked before anything is launched
    prm = L.PcgParams(1e-10, 0, L.PREC_FP64, 0.1, 16, 1, 16, 0)
    res = L.PcgResult()
    dev = op.vals64.device
    b = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = L.lib.feab_pcg_solve_noalloc(C.byref(csr), L.dptr(op.dinv64), L.dptr(b), None, L.dptr(b), C.byref(prm),
                                     C.byref(res), L.stream_ptr(dev))
    assert rc == L.FEAB_SCRATCH_LIMIT
    assert "fixed scratch" in L.status_string(rc)
