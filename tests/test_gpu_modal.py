"""Consistent mass (feab_hex8_element_mass) and the modal solve (GPU block subspace iteration)
against the reference's own outputs (tests/golden/modal_20x4x4.npz: Hex8Solid3D.mass and
FESystem.solve_modal's shift-invert eigsh) and the oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _relnorm(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope="module")
def system(golden):
    import feab200
    g = golden("modal_20x4x4")
    mesh = feab200.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab200.FESystem(mesh, feab200.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(g["D"])
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    fs.assemble_mass(g["R"])
    return fs, g


def test_element_mass_matches_reference(golden):
    from feab200 import _lib as L
    from feab200.device import DeviceMesh
    g = golden("modal_20x4x4")
    X = g["coords"].reshape(-1, 3)
    dm = DeviceMesh(X, np.arange(len(X)).reshape(-1, 8))
    me = dm.element_mass(g["R"], layout=L.KE_FULL).cpu().numpy()
    assert _relnorm(me, g["me"]) < 1e-13
    assert np.array_equal(me, np.transpose(me, (0, 2, 1)))
    # total mass of each element: 7850 x volume in every direction
    for e in range(len(me)):
        tot = me[e][0::3, 0::3].sum()
        assert np.isclose(tot, g["me"][e][0::3, 0::3].sum(), rtol=1e-13)


def test_assembled_mass_matches_oracle(system):
    fs, g = system
    X, el = g["nodes"], g["elements"]
    M_ref = O.structural_csr(O.hex8_element_mass(X[el], g["R"]), el, 3 * len(X))
    M = fs.M
    assert abs(M - M_ref).max() <= 1e-12 * abs(M_ref).max()
    with pytest.raises(ValueError):
        fs.assemble_mass(7850.0)           # solids need a density matrix, as in the reference


def test_solve_modal_matches_reference(system):
    fs, g = system
    f, modes = fs.solve_modal(n_modes=6)
    assert np.max(np.abs(f - g["freq"]) / g["freq"]) < 1e-8
    free = np.setdiff1d(np.arange(fs.n_dof), g["fixed"])
    Phi, Vr = np.asarray(modes)[free], g["modes"][free]
    Mff = fs.M.tocsr()[np.ix_(free, free)]
    Kff = fs.reduced_operator(want32=False).to_scipy()
    assert np.allclose(Phi.T @ (Mff @ Phi), np.eye(6), atol=1e-8)              # M-orthonormal
    # the same 6-dimensional subspace as the reference (the bending pairs are degenerate to 1e-4,
    # so individual vectors may rotate within a pair)
    assert np.linalg.norm(Vr - Phi @ (Phi.T @ (Mff @ Vr))) / np.linalg.norm(Vr) < 1e-6
    lam = (2 * np.pi * f) ** 2
    R = Kff @ Phi - (Mff @ Phi) * lam[None, :]
    assert np.linalg.norm(R) / np.linalg.norm(Kff @ Phi) < 1e-7
    assert np.all(np.asarray(modes)[g["fixed"]] == 0.0)
    assert fs.last_modal_iterations < 60


def test_solve_modal_requires_mass():
    import feab200
    g_mesh = feab200.box_mesh(1.0, 0.2, 0.2, 4, 2, 2)
    fs = feab200.FESystem(g_mesh, feab200.Hex8Solid3D())
    fs.assemble_stiffness(O.D_solid3d(70e9, 0.33))
    fs.fix_dofs(g_mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    with pytest.raises(RuntimeError):
        fs.solve_modal(2)


def test_solve_modal_rejects_bad_mode_counts(system):
    fs, g = system
    with pytest.raises(ValueError):
        fs.solve_modal(0)
    with pytest.raises(ValueError):
        fs.solve_modal(len(fs.free_dofs))
