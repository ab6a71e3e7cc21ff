"""Strain / stress / von Mises / reaction recovery on the GPU (feab_hex8_recover, feab_hex8_apply)
against the reference's own outputs (tests/golden/recovery_20x4x4.npz) and the oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12      # normwise relative, FP64 kernel against the reference's FP64 NumPy


def _relnorm(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope="module")
def system(golden):
    import feab200
    g = golden("recovery_20x4x4")
    mesh = feab200.Mesh(nodes=g["nodes"], elements=g["elements"])
    fs = feab200.FESystem(mesh, feab200.Hex8Solid3D(), sparse=True)
    fs.assemble_stiffness(g["D"])
    fs.fix_dofs(mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    fs.F[:] = g["F"]
    return fs, g


def test_stress_and_strain_match_reference(system):
    fs, g = system
    U = g["U"]
    S = fs.stress(U)
    assert S.dof_names == ("sxx", "syy", "szz", "sxy", "syz", "sxz") and S.shape == (6 * len(g["nodes"]),)
    assert _relnorm(S.nodal, g["stress_nodes"]) < TOL
    assert _relnorm(fs.stress(U, at="elements"), g["stress_elements"]) < TOL
    assert _relnorm(fs.strain(U).nodal, g["strain_nodes"]) < TOL
    assert _relnorm(fs.strain(U, at="elements"), g["strain_elements"]) < TOL
    assert _relnorm(fs.von_mises(U), g["von_mises_nodes"]) < TOL
    assert _relnorm(fs.von_mises(U, at="elements"), g["von_mises_elements"]) < TOL
    assert np.allclose(fs.stress(U).component("sxx"), g["stress_nodes"][:, 0], rtol=0,
                       atol=TOL * np.abs(g["stress_nodes"]).max())


def test_reactions_match_reference_and_balance(system):
    fs, g = system
    R = fs.reactions(g["U"])
    assert _relnorm(R, g["reactions"]) < 1e-9
    assert abs(np.asarray(R)[2::3].sum() - 1.6e5) < 1e-6 * 1.6e5
    free = np.setdiff1d(np.arange(fs.n_dof), g["fixed"])
    assert not np.any(np.asarray(R)[free])


def test_recovery_after_solve_on_distorted_mesh():
    """A distorted mesh solved on the GPU, then recovered: against the oracle on the same U;
    the recovery is deterministic run to run."""
    import feab200
    from feab200.device import DeviceMesh
    nodes, el = O.box_mesh(1.0, 0.3, 0.2, 9, 4, 3)
    X = O.perturb_interior(nodes, (1 / 9, 0.3 / 4, 0.2 / 3), 0.3, 7)
    D = O.D_solid3d(70e9, 0.33)
    U = np.random.default_rng(3).standard_normal(3 * len(X)) * 1e-4
    dm = DeviceMesh(X, el)
    out = dm.recover(U, D, nodal=True, elements=True, von_mises=True)
    s_nodes, s_elem = O.recover(X, el, U, D)
    assert _relnorm(out["nodal"].cpu().numpy(), s_nodes) < TOL
    assert _relnorm(out["elements"].cpu().numpy(), s_elem) < TOL
    assert _relnorm(out["nodal_vm"].cpu().numpy(), O.von_mises(s_nodes)) < TOL
    assert _relnorm(out["elements_vm"].cpu().numpy(), O.von_mises(s_elem)) < TOL
    again = dm.recover(U, D, nodal=True, elements=True, von_mises=True)
    for k in out:
        assert np.array_equal(out[k].cpu().numpy(), again[k].cpu().numpy()), k
    e_nodes, _ = O.recover(X, el, U)
    assert _relnorm(dm.recover(U)["nodal"].cpu().numpy(), e_nodes) < TOL
    # a rigid translation has no strain
    t = np.tile([1e-3, -2e-3, 5e-4], len(X))
    assert np.abs(dm.recover(t, elements=True)["elements"].cpu().numpy()).max() < 1e-13
    del feab200


def test_recovery_error_paths(system):
    fs, g = system
    with pytest.raises(ValueError):
        fs.stress(g["U"][:-3])
    with pytest.raises(ValueError):
        fs.stress(g["U"], at="centroid")
    with pytest.raises(ValueError):
        fs.von_mises(g["U"], plane="strain")
    with pytest.raises(ValueError):
        fs.device_mesh.recover(g["U"], None, von_mises=True)


def test_recovery_rejects_bad_inputs():
    import ctypes as C
    import torch
    from feab200 import _lib as L
    from feab200.device import DeviceMesh
    nodes, el = O.box_mesh(1.0, 1.0, 1.0, 2, 2, 2)
    dm = DeviceMesh(nodes, el)
    topo = dm.topology()
    u = torch.zeros(3 * len(nodes), dtype=torch.float64, device=dm.device)
    sb = int(L.lib.feab_hex8_recover_scratch_bytes(dm.n_elem))
    scratch = torch.empty(sb, dtype=torch.uint8, device=dm.device)
    out = torch.empty((len(nodes), 6), dtype=torch.float64, device=dm.device)
    args = lambda n_elem, sbytes, nodal: (L.dptr(dm.coords), L.dptr(dm.conn), n_elem, len(nodes),  # noqa: E731
                                           L.dptr(topo.inc_ptr), L.dptr(topo.inc_elem), None, L.dptr(u), nodal, None,
                                           None, None, L.dptr(scratch), sbytes, None, dm.stream)
    assert L.lib.feab_hex8_recover(*args(0, sb, L.dptr(out))) == L.FEAB_BAD_ARG          # no elements
    assert L.lib.feab_hex8_recover(*args(dm.n_elem, sb - 8, L.dptr(out))) == L.FEAB_BAD_ARG   # scratch too small
    assert L.lib.feab_hex8_recover(*args(dm.n_elem, sb, None)) == L.FEAB_BAD_ARG          # no output asked for
    assert L.lib.feab_hex8_recover(*args(dm.n_elem, sb, C.c_void_p(out.data_ptr() + 8))) == L.FEAB_BAD_ARG  # misaligned
    assert L.lib.feab_hex8_recover(*args(dm.n_elem, sb, L.dptr(out))) == L.FEAB_OK
    torch.cuda.synchronize()
    assert float(out.abs().max()) == 0.0                                                   # u = 0 -> no strain
