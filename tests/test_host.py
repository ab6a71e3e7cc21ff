"""Host-side logic (no GPU): mesh numbering, loads, boundary-condition bookkeeping."""
import os
import numpy as np
import pytest

import oracle as O
from feab200 import cantilever as cl
from feab200 import facet_loads as fl
from feab200.mesh import box_mesh
from feab200.solver import FESystem
from feab200.elements import Hex8Solid3D


@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 2, 5), (20, 4, 4), (7, 3, 2)])
def test_box_mesh_matches_oracle(shape):
    m = box_mesh(2.0, 0.4, 0.3, *shape)
    nodes, el = O.box_mesh(2.0, 0.4, 0.3, *shape)
    assert np.array_equal(m.nodes, nodes) and np.array_equal(m.elements, el)


def test_cantilever_20x4x4_inputs_match_reference(golden):
    g = golden("cantilever_20x4x4")
    c = cl.plain_cantilever()
    assert np.array_equal(c.mesh.nodes, g["nodes"])
    assert np.array_equal(c.mesh.elements, g["elements"])
    assert np.array_equal(c.fixed, g["fixed"])
    assert np.abs(c.F - g["F"]).max() <= 1e-12 * np.abs(g["F"]).max()
    assert np.isclose(c.F.sum(), -1.0e6 * 0.4 * 0.4)
    faces = fl.boundary_faces_on_plane(c.mesh.nodes, c.mesh.elements, 0, 2.0)
    assert np.array_equal(faces, g["facets"])


def test_facet_batch_matches_reference(golden):
    g = golden("facets")
    sh = np.stack([fl.consistent_facet_load_shares(3, c, float(g["traction"])) for c in g["coords"]])
    assert np.abs(sh - g["shares"]).max() / np.abs(g["shares"]).max() < 1e-13
    M = np.stack([fl.consistent_facet_mass(3, c, 1.0) for c in g["coords"]])
    assert np.abs(M - g["mass"]).max() < 1e-15


def test_nodal_tip_load_is_consistent():
    m = box_mesh(2.0, 0.4, 0.4, 4, 3, 3)
    tip = m.nodes_on_plane(0, 2.0)
    t = np.zeros(len(m.nodes))
    t[tip] = 1.0
    F = cl.nodal_tip_load(m, 2.0, t)
    assert np.isclose(F.sum(), 0.4 * 0.4)           # unit traction integrates to the face area
    assert np.allclose(F, cl.uniform_tip_load(m, 2.0, 1.0))


def test_fesystem_bookkeeping_without_gpu(golden):
    g = golden("cantilever_20x4x4")
    c = cl.plain_cantilever()
    fs = FESystem(c.mesh, Hex8Solid3D(), sparse=True)
    fs.fix_dofs(c.mesh.nodes_on_plane(0, 0.0), [0, 1, 2])
    assert np.array_equal(fs.fixed_dofs_array, g["fixed"])
    assert np.array_equal(fs.free_dofs, g["free"])
    fs.add_consistent_facet_load(Hex8Solid3D(), [tuple(f) for f in g["facets"]], 2, -1.0e6)
    assert np.abs(fs.F - g["F"]).max() <= 1e-12 * np.abs(g["F"]).max()
    fs.add_nodal_force([0, 1], "uy", 10.0)
    assert fs.F[1] == 5.0 and fs.F[4] == 5.0


def test_fesystem_argument_errors_match_reference():
    m = box_mesh(1.0, 1.0, 1.0, 2, 2, 2)
    with pytest.raises(ValueError):
        FESystem(m, Hex8Solid3D(), backend="jax")
    fs = FESystem(m, Hex8Solid3D())
    with pytest.raises(ValueError):
        fs.fix_dofs([], [0])
    with pytest.raises(ValueError):
        fs.fix_dofs([0], [3])
    with pytest.raises(ValueError):
        fs.fix_dofs([10_000], [0])
    with pytest.raises(ValueError):
        fs.add_nodal_force([0], "rx", 1.0)
    with pytest.raises(RuntimeError):
        fs.solve_static(method="pcg")     # K never assembled


def test_batch_and_snapshot_builders_are_seeded():
    a = cl.batch_cantilevers(n_problems=3, seed=9)
    b = cl.batch_cantilevers(n_problems=3, seed=9)
    for p, q in zip(a, b):
        assert p.meta["shape"] == q.meta["shape"] and np.array_equal(p.F, q.F)
        assert 4 <= p.F.shape[1] <= 16
    s = cl.fourier_snapshot_cantilever(nx=4, ny=3, nz=3, n_rhs=5)
    tip_t = s.F[2::3]
    assert s.F.shape == (3 * len(s.mesh.nodes), 5) and np.abs(tip_t).max() > 0


def test_fixed_dof_bookkeeping_is_cached_and_follows_direct_edits():
    """fix_dofs records DOFs node-major like the reference's loop (solver.py:1109-1176), and the
    cached free / fixed arrays follow every change of the fixed set, including direct edits."""
    m = box_mesh(1.0, 0.5, 0.5, 4, 2, 2)
    fs = FESystem(m, Hex8Solid3D())
    nodes = m.nodes_on_plane(0, 0.0)
    fs.fix_dofs(nodes, [2, 0], value=0.25)
    expected = [3 * int(n) + k for n in nodes for k in (2, 0)]
    assert list(fs.fixed_dof_values) == expected
    assert set(fs.fixed_dof_values.values()) == {0.25}
    fixed = fs.fixed_dofs_array
    assert np.array_equal(fixed, np.sort(expected))
    assert np.array_equal(fs.free_dofs, np.setdiff1d(np.arange(fs.n_dof), expected))
    assert np.array_equal(fs._fixed_dof_values_array(fixed), np.full(len(fixed), 0.25))
    # the returned arrays are copies: editing them does not touch the cache
    f = fs.free_dofs
    f[:] = -1
    assert fs.free_dofs.min() >= 0
    # a direct edit of the set is seen; a DOF without a recorded value counts as 0
    fs.fixed_dofs.add(1)
    assert 1 not in fs.free_dofs and 1 in fs.fixed_dofs_array
    assert fs._fixed_dof_values_array(np.array([1]))[0] == 0.0
    fs.fixed_dofs.discard(1)
    assert 1 in fs.free_dofs
    with pytest.raises(ValueError):
        fs.fix_dofs([len(m.nodes)], [0])
    with pytest.raises(ValueError):
        fs.fix_dofs(nodes, [3])


def test_bench_byte_counts():
    """The algorithmic byte formulas the bench's rooflines divide by."""
    import bench
    assert bench.recovery_bytes(10, 4) == 4 * (32 + 448 + 56 + 32 + 32 + 448) + 10 * (48 + 4 + 56)


@pytest.mark.parametrize("shape", [(8, 4, 4), (12, 3, 5)])
def test_oracle_workloads_match_product_workloads(shape):
    """The oracle's builders (used where the CUDA library must not load: the CPU reference arm and
    the full-size oracle job) give bit-identical inputs to the product's benchmark problems."""
    from oracle import workloads as W
    a, b = W.random_tip_cantilever(*shape), cl.random_tip_cantilever(*shape)
    for x, y in ((a["nodes"], b.mesh.nodes), (a["elements"], b.mesh.elements), (a["fixed"], b.fixed),
                 (a["free"], b.free), (a["F"], b.F), (a["D"], b.D)):
        assert np.array_equal(x, y)
    a, b = W.simp_cantilever(*shape), cl.simp_cantilever(*shape)
    assert np.array_equal(a["F"], b.F) and np.array_equal(a["rho"], b.meta["rho"])
    assert a["load_node"] == b.meta["load_node"] and np.array_equal(a["D"], b.D)


def test_oracle_pattern_only_matches_assembled_pattern():
    nodes, el = O.box_mesh(2.0, 0.4, 0.4, 6, 3, 2)
    nodes = O.perturb_interior(nodes, (0.3, 0.13, 0.2), 0.1, 3)
    fixed = O.fixed_dofs_on_plane(nodes)
    free = O.free_dofs(3 * len(nodes), fixed)
    K = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(nodes[el], O.D_solid3d(210e9, 0.3)), el,
                                       3 * len(nodes)), free)
    ip, ix = O.structural_pattern(el, 3 * len(nodes), free)
    assert np.array_equal(ip, K.indptr) and np.array_equal(ix, K.indices)


def test_reference_arm_runs_whole_steps_without_the_cuda_library():
    """bench.py --impl reference times whole oracle steps and never imports feab200 (so
    libfeab200.so is never mapped into that process)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import runpy, sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--shape', '8', '2', '2', "
            "'--steps', '2', '--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'feab200': any(m.startswith('feab200') for m in sys.modules), "
            "'so': 'libfeab200' in maps}))")
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    line, probe = lines[0], lines[1]
    assert probe == {"feab200": False, "so": False}
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 0
    assert len(line["step_ms"]) == 2 and line["value"] > 0
    assert set(line["config"]) == {"workload", "n_free", "nnz", "tol", "l2", "parallelism"}


def test_block_tuning_cache_round_trip(tmp_path):
    from feab200 import batched as bt
    path = str(tmp_path / "sub" / "tuning.json")
    k1 = bt.tuning_key("NVIDIA B200", 418176, 32348142, 1, 64, "fp64")
    k2 = bt.tuning_key("NVIDIA B200", 418176, 32348142, 1, 64, "mixed")
    assert k1 != k2
    bt.save_tuning(k1, bt.BlockShape(32, 64, 512.5), path)
    bt.save_tuning(k2, bt.BlockShape(128, 32, 480.0, True), path)
    got = bt.load_tuning(path)
    assert got == {k1: bt.BlockShape(32, 64, 512.5), k2: bt.BlockShape(128, 32, 480.0, True)}
    # malformed entries are ignored, a missing or corrupt file reads as empty
    import json
    raw = json.load(open(path))
    raw["bad"] = {"item_groups": 0, "tile_width": 64}
    raw["worse"] = {"tile_width": 3}
    raw["tiles_on_ragged_items"] = {"item_groups": 6, "tile_width": 64, "node_tiles": True}
    json.dump(raw, open(path, "w"))
    assert set(bt.load_tuning(path)) == {k1, k2}
    open(path, "w").write("{not json")
    assert bt.load_tuning(path) == {}
    assert bt.load_tuning(str(tmp_path / "missing.json")) == {}


def test_direct_solve_orderings_on_the_host():
    """The direct solve's host-side ordering (feab200.direct): on CPU tensors built from the
    oracle's K_ff, the DOF permutation is a bijection that keeps each node's rows together and in
    component order, and the ordering along the longest axis gives a band of about one
    cross-section of nodes (the bandwidth the GPU kernels then size their tiles for)."""
    import scipy.sparse as sp
    import torch
    import oracle as O
    from feab200.device import Pattern
    from feab200.direct import coordinate_order, dof_permutation, node_order

    X, el = O.box_mesh(2.0, 0.4, 0.4, 16, 3, 2)
    fixed = O.fixed_dofs_on_plane(X, 0, 0.0)
    free = O.free_dofs(3 * len(X), fixed)
    K = O.reduce_free(O.structural_csr(O.hex8_element_stiffness(X[el], O.D_solid3d(1.0, 0.3)), el, 3 * len(X)),
                      free).tocsr()
    node = free // 3
    starts = np.flatnonzero(np.r_[True, node[1:] != node[:-1]])
    fm = -np.ones(3 * len(X), np.int32)
    fm[free] = np.arange(len(free), dtype=np.int32)

    class Op:  # the fields of a ReducedOperator that the ordering reads, on the CPU
        pattern = Pattern(K.shape[0], K.nnz, len(starts), torch.as_tensor(K.indptr.astype(np.int32)),
                          torch.as_tensor(K.indices.astype(np.int32)),
                          torch.as_tensor(np.r_[starts, len(free)].astype(np.int32)), torch.as_tensor(fm))
        vals64 = torch.as_tensor(K.data)
        n = K.shape[0]

    op = Op()
    cross = (3 + 1) * (2 + 1)                        # nodes in one x = const cross-section
    for order in (node_order(op), coordinate_order(op, X)):
        assert sorted(order.tolist()) == list(range(len(starts)))
        iperm = dof_permutation(op, order).numpy()
        assert sorted(iperm.tolist()) == list(range(op.n))
        # a node's rows stay consecutive and in component order
        assert np.all(np.diff(iperm[starts[0]:starts[1]]) == 1)
        P = sp.csr_matrix((np.ones(op.n), (iperm, np.arange(op.n))), shape=K.shape)
        Kp = (P @ K @ P.T).tocoo()
        assert np.allclose(np.sort(np.linalg.eigvalsh(Kp.toarray()))[:3], np.sort(np.linalg.eigvalsh(K.toarray()))[:3])
    # along the longest axis: within two cross-sections of nodes (3 DOFs each)
    iperm = dof_permutation(op, coordinate_order(op, X)).numpy()
    P = sp.csr_matrix((np.ones(op.n), (iperm, np.arange(op.n))), shape=K.shape)
    Kp = (P @ K @ P.T).tocoo()
    assert int(np.abs(Kp.row - Kp.col).max()) < 3 * 2 * cross + 3
