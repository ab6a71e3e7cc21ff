"""Panel products (feab_block_spmm, feab_panel_gram, feab_panel_small) against plain torch FP64
references of the same products, through the C ABI."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _operator(shape=(10, 3, 3)):
    from feab200 import cantilever
    from feab200.device import DeviceMesh
    c = cantilever.random_tip_cantilever(*shape, seed=9)
    dm = DeviceMesh(c.mesh.nodes, c.mesh.elements)
    return dm.assemble(dm.element_stiffness(c.D), dm.pattern(c.fixed), want32=False)


@pytest.mark.parametrize("node_tiles", [True, False])
@pytest.mark.parametrize("k", [1, 4, 16, 32, 64])
def test_block_spmm_matches_csr_product(k, node_tiles):
    from feab200.panel import block_spmm
    op = _operator()
    A = torch.sparse_csr_tensor(op.pattern.row_ptr.long(), op.pattern.col_idx.long(), op.vals64, size=(op.n, op.n))
    X = torch.as_tensor(np.random.default_rng(k).standard_normal((op.n, k))).cuda()
    Y = block_spmm(op, X, node_tiles=node_tiles)
    ref = (A @ X)
    assert float(torch.linalg.norm(Y - ref) / torch.linalg.norm(ref)) < 1e-14
    # deterministic: the same bits on a second call
    assert torch.equal(block_spmm(op, X, node_tiles=node_tiles), Y)


@pytest.mark.parametrize("k", [1, 7, 16, 64])
def test_panel_gram_and_small(k):
    from feab200.panel import panel_gram, panel_small
    rng = np.random.default_rng(3)
    n = 50_001
    P = torch.as_tensor(rng.standard_normal((n, 64))).cuda()
    X, Y = P[:, :k], torch.as_tensor(rng.standard_normal((n, k))).cuda()
    G = panel_gram(X, Y)
    ref = X.t() @ Y
    assert float((G - ref).abs().max() / ref.abs().max()) < 1e-13
    assert torch.equal(panel_gram(X, Y), G)
    V = torch.as_tensor(rng.standard_normal((k, 5))).cuda()
    Z = panel_small(X, V)
    assert float((Z - X @ V).abs().max() / (X @ V).abs().max()) < 1e-14


def test_panel_arguments_are_checked():
    from feab200 import _lib as L
    from feab200.panel import block_spmm, panel_gram, panel_small
    op = _operator((4, 2, 2))
    with pytest.raises(ValueError):
        block_spmm(op, torch.zeros((op.n, 3), dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        panel_gram(torch.zeros((10, 65), dtype=torch.float64, device="cuda"),
                   torch.zeros((10, 65), dtype=torch.float64, device="cuda"))
    Y = torch.zeros((10, 4), dtype=torch.float64, device="cuda")
    assert L.lib.feab_panel_small(L.dptr(Y), 4, 10, 4, L.dptr(Y), 4, L.dptr(Y), 4, None) == L.FEAB_BAD_ARG
    with pytest.raises(ValueError):
        panel_small(Y, torch.zeros((5, 4), dtype=torch.float64, device="cuda"))
