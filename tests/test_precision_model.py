"""The value width of the mixed-precision operator, on the NumPy model of the kernels'
arithmetic (tests/precision_model.py).  CG on the 36-bit difference-form operator K~ converges
as fast as on K; what decides the mixed iteration count is the FP64 residual floor of the K~
solution, |(K - K~) x~| / |b|.  Below the tolerance the mixed solve takes FP64's iterations;
above it, one FP64 refinement cycle is needed and costs about half as many iterations again.
44 mantissa bits push the floor far below 1e-9."""
import numpy as np
import pytest

from precision_model import difference_operator, pcg_iterations, round_mantissa, tip_loaded_cantilever

TOL = 1e-9


def k_tilde_floor(Kff, b, dinv, apply):
    """FP64 relative residual b - K x of the CG solution of K~ x = b (recursive residual 1e-12)."""
    x, r = np.zeros_like(b), b.copy()
    z = dinv * r
    p, rz, bn = z.copy(), r @ z, np.linalg.norm(b)
    for _ in range(20 * len(b)):
        Ap = apply(p)
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        if np.linalg.norm(r) / bn < 1e-12:
            break
        z = dinv * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return np.linalg.norm(b - Kff @ x) / bn


def test_round_mantissa_keeps_36_bits():
    v = np.array([1.0 + 2.0 ** -36, 1.0 + 2.0 ** -37, 1.0 + 2.0 ** -38, -3.25, 0.0])
    r = round_mantissa(v, 36)
    assert r[0] == 1.0 + 2.0 ** -36            # representable: unchanged
    assert r[1] == 1.0 + 2.0 ** -36            # half way: rounded up on the bit pattern
    assert r[2] == 1.0                          # below half: rounded down
    assert r[3] == -3.25 and r[4] == 0.0
    x = np.random.default_rng(0).standard_normal(1000)
    assert np.max(np.abs(round_mantissa(x) - x) / np.abs(x)) <= 2.0 ** -37


def test_difference_operator_matches_K_up_to_value_rounding():
    Kff, b, dinv, free = tip_loaded_cantilever(6, 3, 3)
    x = np.random.default_rng(1).standard_normal(Kff.shape[0])
    y64 = Kff @ x
    assert np.linalg.norm(difference_operator(Kff, free)(x) - y64) / np.linalg.norm(y64) < 1e-10
    assert np.linalg.norm(difference_operator(Kff, free, 50)(x) - y64) / np.linalg.norm(y64) < 1e-14
    # translations are exact in the difference form: K~ 1_c = K 1_c for every component c
    for c in range(3):
        t = (free % 3 == c).astype(float)
        assert np.allclose(difference_operator(Kff, free)(t), Kff @ t, rtol=0, atol=1e-12 * abs(Kff).max())


@pytest.mark.parametrize("shape,E", [((20, 4, 4), 210e9), ((48, 4, 4), 200e9)])
def test_floor_below_tol_keeps_fp64_iterations(shape, E):
    Kff, b, dinv, free = tip_loaded_cantilever(*shape, E=E)
    op = difference_operator(Kff, free)
    assert k_tilde_floor(Kff, b, dinv, op) < TOL
    x64, k64, _ = pcg_iterations(Kff, b, dinv, TOL)
    xm, km, reps = pcg_iterations(Kff, b, dinv, TOL, apply=op)
    assert abs(km - k64) <= 2, (shape, k64, km)
    assert reps >= 1
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-8


def test_floor_above_tol_costs_one_refinement_cycle():
    Kff, b, dinv, free = tip_loaded_cantilever(48, 4, 4, E=210e9)     # same mesh, other rounding
    op = difference_operator(Kff, free)
    assert k_tilde_floor(Kff, b, dinv, op) > TOL
    _, k64, _ = pcg_iterations(Kff, b, dinv, TOL)
    _, k36, _ = pcg_iterations(Kff, b, dinv, TOL, apply=op)
    _, k44, _ = pcg_iterations(Kff, b, dinv, TOL, apply=difference_operator(Kff, free, 44))
    _, kex, _ = pcg_iterations(Kff, b, dinv, TOL, apply=lambda v: Kff @ v)   # exact values, same schedule
    assert k36 > 1.3 * k64, (k64, k36)
    assert abs(k44 - k64) <= 2 and abs(kex - k64) <= 2, (k64, k44, kex)
