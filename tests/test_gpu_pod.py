"""POD: Gram X^T X (FP64 on the CUDA cores, or split-bf16 x3 on the tensor cores) + FP64 Jacobi
eigensolve, against the reference's SVD singular values (tests/golden/pod_small.npz) and the
FP64 oracle."""
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


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gram_fp64_matches_numpy(dtype):
    from feab200.pod import gram_fp64
    rng = np.random.default_rng(2)
    n = 64 * 301 + 37                     # many tiles, more tiles than CTAs, a ragged last tile
    X = (rng.standard_normal((n, 64)) * np.logspace(0, -6, 64)[None, :]).astype(dtype)
    G = gram_fp64(torch.as_tensor(X).cuda()).cpu().numpy()
    ref = X.astype(np.float64).T @ X.astype(np.float64)
    # FP64 accumulation: entrywise relative to sqrt(G_ii G_jj), far below FP32 resolution
    scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))
    assert np.abs(G - ref).max() / 1.0 <= 1e-12 * scale.max()
    assert (np.abs(G - ref) / scale).max() < 1e-13
    assert np.array_equal(G, G.T)
    Xt = torch.as_tensor(X).cuda()
    assert torch.equal(gram_fp64(Xt), gram_fp64(Xt))   # deterministic


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
    # the reference's spectrum spans 12 decades; a Gram (eigenvalues = sigma^2) resolves
    # sigma_k to ~1e-16 (sigma_1 / sigma_k)^2 in FP64: the first six to 1e-6, the first eight
    # to 1e-2
    rel = np.abs(s - ref[: len(s)]) / ref[: len(s)]
    assert np.all(rel[:6] < 1e-6), rel
    assert np.all(rel[:8] < 1e-2), rel
    assert basis.n_modes == 10
    # the tensor-core Gram: leading values to its FP32-accumulation accuracy
    s16 = PodBasis().fit(g["X"], n_modes=10, gram="bf16x3").singular_values
    assert np.abs(s16[0] - ref[0]) / ref[0] < 1e-4
    assert np.all(np.abs(s16[:3] - ref[:3]) / ref[:3] < 1e-2)


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
    assert np.all(rel[:10] < 1e-8), rel
    s16 = PodBasis().fit(X, n_modes=10, gram="bf16x3").singular_values
    rel16 = np.abs(s16[:10] - ref[:10]) / ref[:10]
    assert rel16[0] < 1e-5 and np.all(rel16[:5] < 1e-3), rel16


@pytest.mark.parametrize("n", [64 * 37 + 19, 200_003])
def test_gram_int8_is_exact_to_fp64_level(n):
    """The integer-digit tensor-core Gram against an FP64 Gram of the same FP32 panel: columns
    with six decades of scale, a ragged last chunk, more row ranges than CTAs."""
    from feab200.pod import gram_int8
    rng = np.random.default_rng(7)
    X = (rng.standard_normal((n, 64)) * np.logspace(0, -6, 64)[None, :]).astype(np.float32)
    G = gram_int8(torch.as_tensor(X).cuda()).cpu().numpy()
    ref = X.astype(np.float64).T @ X.astype(np.float64)
    scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))
    assert (np.abs(G - ref) / scale).max() < 1e-13
    assert np.array_equal(G, G.T)
    Xt = torch.as_tensor(X).cuda()
    assert torch.equal(gram_int8(Xt), gram_int8(Xt))       # deterministic


def test_gram_int8_zero_and_tiny_columns():
    from feab200.pod import gram_int8
    rng = np.random.default_rng(8)
    X = rng.standard_normal((5000, 64)).astype(np.float32)
    X[:, 3] = 0.0
    X[:, 5] *= 1e-30
    X[100:, 7] = 0.0
    G = gram_int8(torch.as_tensor(X).cuda()).cpu().numpy()
    ref = X.astype(np.float64).T @ X.astype(np.float64)
    assert np.all(G[3] == 0) and np.all(G[:, 3] == 0)
    scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref))) + 1e-300
    ok = scale > 0
    assert (np.abs(G - ref)[ok] / scale[ok]).max() < 1e-13


def test_pod_int8_gram_matches_the_fp64_svd_on_a_decaying_spectrum():
    """Snapshots with the decay of elastic solutions (sigma_10 / sigma_1 ~ 1e-4): the int8 Gram
    keeps sigma_1..sigma_10 at FP64-Gram accuracy, where bf16x3 loses sigma_3 on."""
    from feab200.pod import PodBasis
    rng = np.random.default_rng(9)
    n = 120_000
    U, _ = np.linalg.qr(rng.standard_normal((n, 16)))
    s = np.logspace(0, -5, 16)
    X = ((U * s) @ np.linalg.qr(rng.standard_normal((16, 16)))[0]).astype(np.float32)
    ref = np.linalg.svd(X.astype(np.float64), compute_uv=False)[:10]
    got = {g: PodBasis().fit(torch.as_tensor(X).cuda(), n_modes=10, gram=g).singular_values[:10]
           for g in ("int8", "fp64")}
    err = {g: np.abs(v - ref) / ref for g, v in got.items()}
    assert err["int8"].max() < 1e-7, err
    assert err["int8"].max() <= 10 * err["fp64"].max() + 1e-12


def test_pod_auto_gram_picks_by_input_precision():
    """FP32 snapshots go to the exact-product tensor-core Gram, FP64 snapshots to the FP64 Gram
    (their values carry more bits than the seven 7-bit digits keep); both agree with the FP64
    SVD of their own input."""
    from feab200.pod import PodBasis
    rng = np.random.default_rng(12)
    n = 50_000
    U, _ = np.linalg.qr(rng.standard_normal((n, 12)))
    X = (U * np.logspace(0, -4, 12)) @ np.linalg.qr(rng.standard_normal((12, 12)))[0]
    for dt in (np.float32, np.float64):
        Xd = X.astype(dt)
        ref = np.linalg.svd(Xd.astype(np.float64), compute_uv=False)[:8]
        s_auto = PodBasis().fit(torch.as_tensor(Xd).cuda(), n_modes=8).singular_values[:8]
        s_same = PodBasis().fit(torch.as_tensor(Xd).cuda(), n_modes=8,
                                gram="int8" if dt == np.float32 else "fp64").singular_values[:8]
        assert np.array_equal(s_auto, s_same)
        assert (np.abs(s_auto - ref) / ref).max() < 1e-7
