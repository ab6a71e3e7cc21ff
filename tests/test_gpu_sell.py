"""The sliced (SELL-32) node-group operator: its products against the CSR product and SciPy.

K_ff x through the sliced layout must equal the CSR product up to summation order (FP64 kind)
and the 48-bit difference form up to value rounding (mixed kind), on the golden 20x4x4
cantilever and on meshes whose fixed sets leave nodes with 1 or 2 free DOFs (groups of 1-2
rows, free-DOF masks, padding) and a group count that is not a multiple of 32.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def _reduced(nodes, elements, D, fixed):
    from feab200.device import DeviceMesh
    dm = DeviceMesh(nodes, elements)
    return dm.assemble(dm.element_stiffness(D), dm.pattern(fixed), want32=False)


def _check(op, Kff, xs):
    from feab200.device import sell_spmv
    absK = abs(Kff)
    for x in xs:
        ref = Kff @ x
        scale = np.linalg.norm(absK @ np.abs(x))          # size of the terms that cancel in K x
        y64 = sell_spmv(op, x, "fp64").cpu().numpy()
        ymx = sell_spmv(op, x, "mixed").cpu().numpy()
        assert np.linalg.norm(y64 - ref) / scale < 1e-14
        assert np.linalg.norm(ymx - ref) / scale < 1e-10


def test_sell_spmv_matches_csr_20x4x4(golden):
    g = golden("cantilever_20x4x4")
    op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    Kff = sp.csr_matrix((g["vals"], g["col_idx"], g["row_ptr"]))
    rng = np.random.default_rng(11)
    _check(op, Kff, (rng.standard_normal(op.n), g["U_lu"][g["free"]]))


@pytest.mark.parametrize("shape", [(5, 3, 2), (9, 4, 3)])
def test_sell_spmv_partial_fixes_and_ragged_slices(shape):
    nodes, el = O.box_mesh(1.0, 0.5, 0.3, *shape)
    nodes = O.perturb_interior(nodes, np.array([1.0 / shape[0], 0.5 / shape[1], 0.3 / shape[2]]), 0.1, 3)
    D = O.D_solid3d(7.0, 0.28)
    x0 = O.fixed_dofs_on_plane(nodes, 0, 0.0)
    n_dof = 3 * len(nodes)
    rng = np.random.default_rng(5)
    extra = rng.choice(np.arange(n_dof), size=n_dof // 7, replace=False)   # single DOFs: 1-2 free per node
    fixed = np.unique(np.concatenate([x0, extra]))
    op = _reduced(nodes, el, D, fixed)
    free = O.free_dofs(n_dof, fixed)
    Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(nodes[el], D), el, n_dof), free)
    _check(op, Kff, (rng.standard_normal(op.n), np.linspace(-1.0, 2.0, op.n)))


def test_sell_operator_rejects_short_row_bound(golden):
    from feab200 import _lib as L
    import ctypes as C
    g = golden("cantilever_20x4x4")
    op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    p = op.pattern
    nbytes = int(L.lib.feab_sell_operator_bytes(p.n, p.n_groups, 8, L.PREC_FP64))
    storage = torch.empty(nbytes, dtype=torch.uint8, device=op.vals64.device)
    d = L.SellOperator()
    csr = op.csr_struct()
    rc = L.lib.feab_sell_operator_build(C.byref(csr), None, L.PREC_FP64, 8, L.dptr(storage), nbytes, C.byref(d),
                                        L.stream_ptr(op.vals64.device))
    assert rc == L.FEAB_BAD_ARG


def test_pcg_through_both_layouts_matches_direct_solve(golden):
    """The FP64 PCG through the CSR and through the sliced operator, and the mixed PCG, all land
    within the displacement tolerance of the SuperLU solution, in the reference's iteration
    count (up to summation-order ties)."""
    from feab200.device import pcg_solve
    g = golden("cantilever_20x4x4")
    op = _reduced(g["nodes"], g["elements"], g["D"], g["fixed"])
    u_ref = g["U_lu"][g["free"]]
    for precision, layout in (("fp64", "csr"), ("fp64", "sell"), ("mixed", "sell")):
        x, info = pcg_solve(op, g["Ff"], tol=1e-10, precision=precision, layout=layout)
        assert info.status == 0
        assert abs(info.iters - int(g["pcg_iters"])) <= 2, (precision, layout, info.iters)
        err = np.linalg.norm(x.cpu().numpy() - u_ref) / np.linalg.norm(u_ref)
        assert err < 1e-8, (precision, layout, err)


def test_sell_column_offsets_16_bit_and_wide():
    """The sliced operator stores 2-byte column offsets from each lane's first row when they all
    fit 16 bits, and keeps the 4-byte columns otherwise (a 110 x 100 x 1 box: the second node
    layer lies 11,211 nodes, 33,633 DOFs, above the first).  Both forms give the CSR product,
    and the PCG through either converges to the same solution."""
    from feab200.device import pcg_solve
    rng = np.random.default_rng(17)
    cases = {}
    for shape in ((12, 4, 3), (110, 100, 1)):
        nodes, el = O.box_mesh(2.0, 1.0, 0.1, *shape)
        D = O.D_solid3d(5.0, 0.3)
        fixed = O.fixed_dofs_on_plane(nodes, 0, 0.0)
        n_dof = 3 * len(nodes)
        op = _reduced(nodes, el, D, fixed)
        free = O.free_dofs(n_dof, fixed)
        Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(nodes[el], D), el, n_dof), free)
        _check(op, Kff, (rng.standard_normal(op.n),))
        cases[shape] = (op, Kff)
    assert cases[(12, 4, 3)][0].sell_operator("fp64").tcol16
    assert cases[(12, 4, 3)][0].sell_operator("mixed").tcol16
    assert not cases[(110, 100, 1)][0].sell_operator("fp64").tcol16
    assert not cases[(110, 100, 1)][0].sell_operator("mixed").tcol16
    op, Kff = cases[(110, 100, 1)]
    b = rng.standard_normal(op.n)
    x64, i64 = pcg_solve(op, b, tol=1e-10, precision="fp64", layout="sell")
    xcs, ics = pcg_solve(op, b, tol=1e-10, precision="fp64", layout="csr")
    assert i64.status == 0 and ics.status == 0
    assert float(torch.linalg.norm(x64 - xcs) / torch.linalg.norm(xcs)) < 1e-8
