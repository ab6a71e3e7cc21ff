"""POD on the tensor cores: Gram X^T X (split-bf16 x3) + FP64 Jacobi eigensolve, against the
reference's SVD singular values (tests/golden/pod_small.npz) and the FP64 oracle."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def test_gram_matches_fp64_gram():
    from feab200.pod import gram_bf16x3
    rng = np.random.default_rng(0)
    n = 64 * 37 + 19                      # several chunks and a ragged last chunk
    X = rng.standard_normal((n, 64)).astype(np.float32)
    G = gram_bf16x3(torch.as_tensor(X).cuda()).cpu().numpy()
    ref = X.astype(np.float64).T @ X.astype(np.float64)
    # split-bf16 x3 products: ~2^-16 relative per product
    assert np.abs(G - ref).max() / np.abs(ref).max() < 2e-5
    assert np.array_equal(G, G.T)


def test_gram_is_deterministic():
    from feab200.pod import gram_bf16x3
    X = torch.randn(100_000, 64, device="cuda")
    assert torch.equal(gram_bf16x3(X), gram_bf16x3(X))


def test_symeig_jacobi():
    from feab200.pod import symeig
    rng = np.random.default_rng(1)
    A = rng.standard_normal((64, 64))
    A = A @ A.T
    w, V = symeig(torch.as_tensor(A).cuda())
    ref = np.sort(np.linalg.eigvalsh(A))[::-1]
    assert np.abs(w.cpu().numpy() - ref).max() / ref[0] < 1e-12
    Vh = V.cpu().numpy()
    assert np.abs(Vh.T @ Vh - np.eye(64)).max() < 1e-12


def test_pod_singular_values_match_reference(golden):
    from feab200.pod import PodBasis
    g = golden("pod_small")
    basis = PodBasis().fit(g["X"], n_modes=10)
    s, ref = basis.singular_values, g["singular_values"]
    # leading values to bf16x3 accuracy; the reference's spectrum decays by 1e-11 overall
    assert np.abs(s[0] - ref[0]) / ref[0] < 1e-4
    assert np.all(np.abs(s[:3] - ref[:3]) / ref[:3] < 1e-2)
    assert basis.n_modes == 10


def test_pod_on_solution_snapshots():
    """Snapshots from cantilever solves: leading singular values vs the oracle's FP64 SVD."""
    from feab200.pod import PodBasis
    rng = np.random.default_rng(3)
    t = np.linspace(0, 1, 20_000)[:, None]
    X = np.cos(np.pi * np.arange(1, 41)[None, :] * t) * (2.0 ** -np.arange(40))[None, :]
    X = X @ rng.standard_normal((40, 40))
    s = PodBasis().fit(X, n_modes=10).singular_values
    ref = O.pod_singular_values(X)
    rel = np.abs(s[:10] - ref[:10]) / ref[:10]
    assert rel[0] < 1e-5 and np.all(rel[:5] < 1e-3), rel
