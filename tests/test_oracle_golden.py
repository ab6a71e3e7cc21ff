"""The CPU oracle against vectors produced by the reference itself (tests/golden)."""
import numpy as np

import oracle as O


def test_box_mesh_and_jitter_match_reference(golden):
    g = golden("cantilever_20x4x4")
    nodes, el = O.box_mesh(2.0, 0.4, 0.4, 20, 4, 4)
    X = O.perturb_interior(nodes, (0.1, 0.1, 0.1), 0.1, 1234)
    assert np.array_equal(X, g["nodes"])
    assert np.array_equal(el, g["elements"])
    assert np.array_equal(O.fixed_dofs_on_plane(X, 0, 0.0), g["fixed"])


def test_stiffness_pattern_and_values_match_reference(golden):
    g = golden("cantilever_20x4x4")
    X, el = g["nodes"], g["elements"]
    ke = O.hex8_element_stiffness(X[el], g["D"])
    K = O.structural_csr(ke, el, 3 * len(X))
    assert K.nnz == int(g["nnz_full"])
    Kff = O.reduce_free(K, g["free"])
    assert np.array_equal(Kff.indptr, g["row_ptr"]) and np.array_equal(Kff.indices, g["col_idx"])
    assert np.abs(Kff.data - g["vals"]).max() / np.abs(g["vals"]).max() < 1e-14


def test_undistorted_pattern_is_structural(golden):
    g = golden("pattern_4x3x2")
    ke = O.hex8_element_stiffness(g["nodes"][g["elements"]], g["D"])
    K = O.structural_csr(ke, g["elements"], 3 * len(g["nodes"]))
    assert np.array_equal(K.indptr, g["K_row_ptr"]) and np.array_equal(K.indices, g["K_col_idx"])
    Kff = O.reduce_free(K, g["free"])
    assert np.array_equal(Kff.indptr, g["Kff_row_ptr"]) and np.array_equal(Kff.indices, g["Kff_col_idx"])
    # the reference's LIL storage drops exact-zero cancellations on an undistorted grid
    assert g["lil_col_idx"].size < K.nnz


def test_element_stiffness_matches_reference(golden):
    g = golden("ke_distorted")
    for D, ref in ((g["D"], g["ke"]), (g["D_aniso"], g["ke_aniso"])):
        ke = O.hex8_element_stiffness(g["coords"], D)
        assert np.abs(ke - ref).max() / np.abs(ref).max() < 1e-14


def test_facet_integrals_match_reference(golden):
    g = golden("facets")
    sh = O.facet_load_shares(g["coords"], float(g["traction"]))
    assert np.abs(sh - g["shares"]).max() / np.abs(g["shares"]).max() < 1e-13
    assert np.abs(O.facet_mass(g["coords"]) - g["mass"]).max() / np.abs(g["mass"]).max() < 1e-13


def test_pcg_matches_reference_iterations_and_solution(golden):
    g = golden("cantilever_20x4x4")
    import scipy.sparse as sp
    Kff = sp.csr_matrix((g["vals"], g["col_idx"], g["row_ptr"]))
    x, it, rel = O.preconditioned_cg(Kff, g["Ff"], O.jacobi_inverse_diagonal(Kff), tol=1e-10)
    assert it == int(g["pcg_iters"])
    assert np.linalg.norm(x - g["uf_pcg"]) / np.linalg.norm(g["uf_pcg"]) < 1e-12
    assert np.linalg.norm(x - g["U_lu"][g["free"]]) / np.linalg.norm(g["U_lu"]) < 1e-10


def test_pcg_error_paths():
    import scipy.sparse as sp
    A = sp.diags([1.0, -2.0, 3.0]).tocsr()
    try:
        O.preconditioned_cg(A, np.array([1.0, 1.0, 1.0]), None, tol=1e-12)
        raise AssertionError("expected LinAlgError")
    except np.linalg.LinAlgError:
        pass
    B = sp.csr_matrix(np.array([[4.0, 1.0, 0.0], [1.0, 3.0, 1.0], [0.0, 1.0, 2.0]]))
    try:
        O.preconditioned_cg(B, np.array([1.0, 2.0, 3.0]), None, tol=1e-30, maxiter=1)
        raise AssertionError("expected RuntimeError")
    except RuntimeError:
        pass
    try:
        O.jacobi_inverse_diagonal(sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 2.0]])))
        raise AssertionError("expected ValueError")
    except ValueError:
        pass


def test_simp_sensitivity_matches_reference(golden):
    g = golden("simp_6x3x3")
    ke = O.hex8_element_stiffness(g["nodes"][g["elements"]], g["D"])
    dc = O.compliance_sensitivity_closed_form(ke, g["elements"], g["u"], g["rho"], float(g["p"]), float(g["rho_min"]))
    assert np.abs(dc - g["dc"]).max() / np.abs(g["dc"]).max() < 1e-12
    # quadratic form through strains equals u^T ke u
    u_e = g["u"][O.global_dofs(g["elements"])]
    q = O.element_strain_energy_density(g["nodes"][g["elements"]], g["D"], u_e)
    ref = np.einsum("ei,eij,ej->e", u_e, ke, u_e)
    assert np.abs(q - ref).max() / np.abs(ref).max() < 1e-13
    # the reference's own FD and adjoint agree with its closed form
    sel = g["fd_elems"]
    assert np.allclose(g["dc"][sel], g["dc_fd"], rtol=1e-5)
    assert np.allclose(g["dc_adjoint"], g["dc"], rtol=1e-9)


def test_pod_singular_values_match_reference(golden):
    g = golden("pod_small")
    s = O.pod_singular_values(g["X"])
    assert np.abs(s - g["singular_values"]).max() / g["singular_values"][0] < 1e-14


def _relnorm(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def test_recovery_matches_reference(golden):
    g = golden("recovery_20x4x4")
    X, el, U, D = g["nodes"], g["elements"], g["U"], g["D"]
    s_nodes, s_elem = O.recover(X, el, U, D)
    e_nodes, e_elem = O.recover(X, el, U)
    assert _relnorm(s_nodes, g["stress_nodes"]) < 1e-13 and _relnorm(s_elem, g["stress_elements"]) < 1e-13
    assert _relnorm(e_nodes, g["strain_nodes"]) < 1e-13 and _relnorm(e_elem, g["strain_elements"]) < 1e-13
    assert _relnorm(O.von_mises(s_nodes), g["von_mises_nodes"]) < 1e-13
    assert _relnorm(O.von_mises(s_elem), g["von_mises_elements"]) < 1e-13
    K = O.structural_csr(O.hex8_element_stiffness(X[el], D), el, 3 * len(X))
    R = O.reactions(K, U, g["F"], g["fixed"])
    assert _relnorm(R, g["reactions"]) < 1e-9
    # the reactions balance the applied load (z: the -1e6 Pa traction on the 0.16 m^2 tip face)
    assert abs(R[2::3].sum() - 1.6e5) < 1e-6 * 1.6e5


def test_simp_loop_matches_reference(golden):
    g = golden("topopt_8x4x4")
    X, el = g["nodes"], g["elements"]
    H = O.build_filter_weights(X[el].mean(axis=1), float(g["radius"]))
    assert np.array_equal(H, g["H"])
    assert _relnorm(O.apply_sensitivity_filter(H, g["rho_s"], g["dc_s"]), g["dc_filtered"]) < 1e-14
    assert np.array_equal(O.oc_update(g["rho_s"], g["dc_s"], 0.4, move=0.2, rho_min_bound=1e-2), g["rho_oc"])
    rho, hist, u = O.topology_optimize_compliance(X, el, g["D"], g["fixed"], g["F"], 0.4, p=3.0, rho_min=1e-2,
                                                  move=0.2, n_iter=12, filter_radius=float(g["radius"]), tol=1e-3)
    assert len(hist) == len(g["compliance_history"])
    assert np.max(np.abs(np.array(hist) - g["compliance_history"]) / g["compliance_history"]) < 1e-9
    assert np.max(np.abs(rho - g["rho_final"])) < 1e-8
    assert _relnorm(u, g["u_final"]) < 1e-8


def test_bbar_element_stiffness_matches_reference(golden):
    g = golden("bbar_hex8")
    for tag in ("03", "04999"):
        ke = O.hex8_bbar_element_stiffness(g["coords"], g["D_" + tag])
        assert _relnorm(ke, g["ke_" + tag]) < 1e-14


def test_mass_and_modal_match_reference(golden):
    g = golden("modal_20x4x4")
    assert _relnorm(O.hex8_element_mass(g["coords"], g["R"]), g["me"]) < 1e-14
    X, el = g["nodes"], g["elements"]
    free = O.free_dofs(3 * len(X), g["fixed"])
    Kff = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(X[el], g["D"]), el, 3 * len(X)), free)
    Mff = O.reduce_free(O.structural_csr(O.hex8_element_mass(X[el], g["R"]), el, 3 * len(X)), free)
    f, V = O.modal(Kff, Mff, 6)
    assert np.max(np.abs(f - g["freq"]) / g["freq"]) < 1e-10
    # M-orthonormal modes spanning the reference's subspace
    Vr = g["modes"][free]
    assert np.allclose(V.T @ (Mff @ V), np.eye(6), atol=1e-8)
    assert np.linalg.norm(Vr - V @ (V.T @ (Mff @ Vr))) / np.linalg.norm(Vr) < 1e-6
