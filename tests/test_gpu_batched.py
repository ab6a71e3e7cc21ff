"""Batched multi-RHS block-PCG against independent per-column oracle solves
(the reference's batched == independent check, fea_engine/tests/test_batched_solve.py:66-115)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

UTOL = 1e-8


def _oracle_columns(c, tol=1e-12):
    X, el = c.mesh.nodes, c.mesh.elements
    Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(X[el], c.D), el, 3 * len(X)), c.free)
    dinv = O.jacobi_inverse_diagonal(Kff)
    F = c.F.reshape(3 * len(X), -1)
    U = np.zeros_like(F)
    for j in range(F.shape[1]):
        U[c.free, j] = O.preconditioned_cg(Kff, F[c.free, j], dinv, tol=tol)[0]
    return U


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_problem_batch_matches_independent_solves(precision):
    from feab200 import cantilever
    from feab200.batched import ProblemBatch
    probs = cantilever.batch_cantilevers(n_problems=5, seed=21, nx_range=(3, 9), nyz_range=(2, 4), rhs_range=(2, 7))
    batch = ProblemBatch([(p.mesh.nodes, p.mesh.elements, p.D, p.fixed, p.F) for p in probs])
    U, res = batch.solve(tol=1e-10, precision=precision)
    assert (res.status == 0).all(), res.status
    for p, Up in zip(probs, U):
        ref = _oracle_columns(p)
        for j in range(ref.shape[1]):
            err = np.linalg.norm(Up[:, j] - ref[:, j]) / np.linalg.norm(ref[:, j])
            assert err < UTOL, (p.meta["shape"], j, err)
    # padded columns stay inactive
    assert (res.iters[:, 8:] == 0).all() if res.iters.shape[1] > 8 else True


def test_solve_static_batched_drop_in(golden):
    import feab200
    g = golden("cantilever_20x4x4")
    mesh = feab200.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab200.FESystem(mesh, feab200.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(g["D"])
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    rng = np.random.default_rng(0)
    F = np.zeros((fs.n_dof, 5))
    F[:, 0] = g["F"]
    F[:, 1:] = rng.standard_normal((fs.n_dof, 4)) * 1e3
    U = feab200.solve_static_batched(fs, F, tol=1e-11)
    for j in range(5):
        fs.F[:] = F[:, j]
        Uj = np.asarray(fs.solve_static(method="pcg", tol=1e-12))
        assert np.linalg.norm(U[:, j] - Uj) / np.linalg.norm(Uj) < UTOL
    assert np.linalg.norm(U[:, 0] - g["U_lu"]) / np.linalg.norm(g["U_lu"]) < UTOL


def test_block_pcg_wide_panel_single_problem():
    """One mesh, 40 load columns (panel width 64) -- the snapshot-set layout."""
    from feab200 import cantilever
    from feab200.batched import ProblemBatch
    c = cantilever.fourier_snapshot_cantilever(12, 3, 3, n_rhs=40, seed=2)
    batch = ProblemBatch([(c.mesh.nodes, c.mesh.elements, c.D, c.fixed, c.F)])
    assert batch.K == 64
    (U,), res = batch.solve(tol=1e-11)
    assert (res.status == 0).all()
    ref = _oracle_columns(c)
    err = np.linalg.norm(U - ref) / np.linalg.norm(ref)
    assert err < UTOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_block_pcg_launch_shapes_agree_and_tuner_picks_one(tmp_path, monkeypatch, precision):
    """Every work-item size and column-tile width gives the same solution (the launch shape is
    a performance choice only), and the tuner's choice is one of the candidates, cached in the
    JSON file it names."""
    import torch
    from feab200 import cantilever
    from feab200 import batched as bt
    monkeypatch.setenv("FEAB_TUNING_CACHE", str(tmp_path / "tuning.json"))
    monkeypatch.setattr(bt, "_tuned_block", {})
    c = cantilever.random_tip_cantilever(12, 4, 4, seed=3)
    b = bt.ProblemBatch([(c.mesh.nodes, c.mesh.elements, c.D, c.fixed, c.F)])
    op = b.assemble()
    rng = np.random.default_rng(5)
    B = torch.as_tensor(rng.standard_normal((op.n, 32))).cuda()
    ref, _ = bt.block_pcg(op, b.row_bounds, B, [32], tol=1e-11, precision=precision, max_groups=64, tile_width=32)
    for g, w in ((16, 16), (128, 32), (32, 16)):
        X, res = bt.block_pcg(op, b.row_bounds, B, [32], tol=1e-11, precision=precision, max_groups=g, tile_width=w)
        assert (res.status == 0).all()
        assert float(torch.linalg.norm(X - ref) / torch.linalg.norm(ref)) < 1e-9
    shape = bt.tuned_block_shape(op, b.row_bounds, B, [32], precision)
    assert shape.item_groups in bt.ITEM_GROUPS and shape.tile_width in (16, 32) and shape.us_per_step > 0
    key = bt.tuning_key(torch.cuda.get_device_name(op.vals64.device), op.n, op.nnz, 1, 32, precision)
    assert bt.load_tuning()[key] == shape
    X, res = bt.block_pcg(op, b.row_bounds, B, [32], tol=1e-11, precision=precision)   # tuned shape
    assert (res.status == 0).all()
    assert float(torch.linalg.norm(X - ref) / torch.linalg.norm(ref)) < 1e-9



def test_mixed_block_pcg_keeps_fp64_iterations_where_36_bits_would_not():
    """A 48x4x4 cantilever under unit tip loads at 210 GPa: with 36 mantissa bits the
    difference-form operator's FP64 residual floor (about 2e-9 of |b| in the NumPy model of the
    kernels) lies above tol = 1e-9 and costs an extra refinement cycle (278 iterations against
    FP64's 179 in the model).  The block-PCG's operator keeps 44 bits, whose floor lies far
    below, so the mixed solve takes FP64's iteration count."""
    from feab200 import D_solid3d, Material, box_mesh
    from feab200.batched import ProblemBatch
    mesh = box_mesh(2.0, 0.4, 0.4, 48, 4, 4)
    X, el = mesh.nodes, mesh.elements
    fixed = np.sort((3 * mesh.nodes_on_plane(0, 0.0)[:, None] + np.arange(3)).reshape(-1))
    F = np.zeros((3 * len(X), 2))
    F[3 * mesh.nodes_on_plane(0, 2.0) + 2, 0] = 1.0
    F[3 * mesh.nodes_on_plane(0, 2.0) + 1, 1] = 1.0
    D = D_solid3d(Material(E=210e9, nu=0.3))
    batch = ProblemBatch([(X, el, D, fixed, F)])
    U64, r64 = batch.solve(tol=1e-9, precision="fp64")
    Um, rm = batch.solve(tol=1e-9, precision="mixed")
    Ut, _ = batch.solve(tol=1e-13, precision="fp64")
    assert (r64.status == 0).all() and (rm.status == 0).all()
    assert rm.iters[:, :2].max() <= r64.iters[:, :2].max() + 3, (rm.iters[:, :2], r64.iters[:, :2])
    for j in range(2):
        assert np.linalg.norm(Um[0][:, j] - Ut[0][:, j]) / np.linalg.norm(Ut[0][:, j]) < UTOL
