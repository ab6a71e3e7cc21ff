"""Node tiles of the block SpMM (feab_tile_operator_build): the tile layout against a NumPy
construction from the same CSR, the tiled SpMM and block-PCG against the single-group ones.

A tile is FEAB_TILE_GROUPS consecutive node row groups of one problem; its union column list
is the union of the groups' column lists, each column with the mask of the groups that have it,
grouped by mask (ascending mask, ascending columns within a mask); the values follow in
(union column, group, row) order with rows past a group's free DOFs set to 0.  The meshes below have partially fixed nodes (groups of 1-2 rows), several
problems with group counts that are not multiples of 4 (a short last tile) and perturbed
coordinates.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

T = 4


def _batch(shapes=((5, 3, 2), (4, 3, 3), (7, 2, 2)), extra_fixed=True):
    from feab200.batched import ProblemBatch
    rng = np.random.default_rng(23)
    probs = []
    for i, sh in enumerate(shapes):
        X, el = O.box_mesh(1.0 + i, 0.5, 0.3, *sh)
        X = O.perturb_interior(X, np.array([1.0 / sh[0], 0.5 / sh[1], 0.3 / sh[2]]), 0.1, 3 + i)
        fixed = O.fixed_dofs_on_plane(X, 0, 0.0)
        if extra_fixed:
            n_dof = 3 * len(X)
            fixed = np.unique(np.concatenate([fixed, rng.choice(n_dof, n_dof // 9, replace=False)]))
        F = rng.standard_normal((3 * len(X), 3))
        probs.append((X, el, O.D_solid3d(5.0 * (1 + i), 0.3), fixed, F))
    b = ProblemBatch(probs)
    b.assemble()
    return b


def _dev(storage, ptr, count, dtype):
    """count elements of dtype at device address ptr inside storage, copied to the host."""
    itemsize = torch.empty((), dtype=dtype).element_size()
    off = ptr - storage.data_ptr()
    assert 0 <= off and off + count * itemsize <= storage.numel()
    return storage[off:off + count * itemsize].view(dtype).cpu().numpy()


def _expected_tiles(op, pgroups, precision):
    """(tile_g0, ucol, umask, values per tile) built in NumPy from the CSR (and the difference
    form's off-node column lists for mixed)."""
    rp = op.pattern.row_ptr.cpu().numpy()
    ci = op.pattern.col_idx.cpu().numpy()
    gp = op.pattern.group_ptr.cpu().numpy()
    v = op.vals64.cpu().numpy()
    tile_g0 = []
    for p in range(len(pgroups) - 1):
        tile_g0.extend(range(pgroups[p], pgroups[p + 1], T))
    tile_g0.append(pgroups[-1])
    tiles = []
    for t in range(len(tile_g0) - 1):
        lists, rows = [], []
        for g in range(tile_g0[t], tile_g0[t + 1]):
            r0, f = gp[g], gp[g + 1] - gp[g]
            cols = ci[rp[r0]:rp[r0 + 1]]
            vals = np.stack([v[rp[r0 + k]:rp[r0 + k + 1]] for k in range(f)])
            if precision == "mixed":   # off-node columns only
                keep = (cols < r0) | (cols >= r0 + f)
                cols, vals = cols[keep], vals[:, keep]
            lists.append(cols)
            rows.append(vals)
        union = np.unique(np.concatenate(lists)) if lists else np.zeros(0, np.int64)
        mask = np.zeros(len(union), np.int64)
        for j, cols in enumerate(lists):
            mask[np.searchsorted(union, cols)] |= 1 << j
        order = np.lexsort((union, mask))            # grouped by mask, ascending columns within one
        union, mask = union[order], mask[order]
        vals = []
        for u, c in enumerate(union):
            for j, cols in enumerate(lists):
                if (mask[u] >> j) & 1:
                    i = int(np.searchsorted(cols, c))
                    trip = np.zeros(3)
                    trip[:rows[j].shape[0]] = rows[j][:, i]
                    vals.append(trip)
        tiles.append((union, mask, np.array(vals).reshape(-1)))
    return np.array(tile_g0), tiles


def _round44(x):
    b = np.asarray(x, np.float64).view(np.uint64) + np.uint64(0x80)
    return (b & ~np.uint64(0xff)).view(np.float64)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tile_layout_matches_numpy_construction(precision):
    from feab200.batched import _problem_groups
    b = _batch()
    op = b.op
    pg = _problem_groups(op.pattern.group_ptr.cpu().numpy(), b.row_bounds)
    t = op.tile_operator(precision, pg)
    storage = op._tiles[(precision, np.asarray(pg, np.int32).tobytes())][0]
    tile_g0, tiles = _expected_tiles(op, pg, precision)
    assert t.n_tiles == len(tiles) and t.n_groups == op.pattern.n_groups
    assert np.array_equal(_dev(storage, t.tile_g0, t.n_tiles + 1, torch.int32), tile_g0)
    gt = _dev(storage, t.group_tile, t.n_groups, torch.int32)
    assert np.array_equal(gt, np.repeat(np.arange(t.n_tiles), np.diff(tile_g0)))
    uoff = _dev(storage, t.uoff, t.n_tiles + 1, torch.int32)
    poff = _dev(storage, t.poff, t.n_tiles + 1, torch.int32)
    ucol = _dev(storage, t.ucol, int(uoff[-1]), torch.int32)
    umask = _dev(storage, t.umask, int(uoff[-1]), torch.uint8)
    nv = 3 * int(poff[-1])
    if precision == "fp64":
        vals = _dev(storage, t.v64, nv, torch.float64)
    else:
        hi = _dev(storage, t.vhi, nv, torch.int32).view(np.uint32).astype(np.uint64)
        lo = _dev(storage, t.vlo, nv, torch.int16).view(np.uint16).astype(np.uint64)
        lo2 = _dev(storage, t.vlo2, nv, torch.uint8).astype(np.uint64)
        vals = ((hi << np.uint64(32)) | (lo << np.uint64(16)) | (lo2 << np.uint64(8))).view(np.float64)
    cptr = _dev(storage, t.cptr, t.n_tiles + 1, torch.int32)
    chunks = _dev(storage, t.chunk, 4 * int(cptr[-1]), torch.int32).reshape(-1, 4)
    for i in range(t.n_tiles):   # chunk descriptors: FEAB_TILE_CHUNK columns, contiguous values
        ch = chunks[cptr[i]:cptr[i + 1]]
        n_cols = uoff[i + 1] - uoff[i]
        assert len(ch) == (n_cols + 63) // 64
        if len(ch):
            assert np.array_equal(ch[:, 0], uoff[i] + 64 * np.arange(len(ch)))
            assert np.array_equal(ch[:, 1], np.minimum(64, n_cols - 64 * np.arange(len(ch))))
            assert ch[0, 2] == 3 * poff[i] and ch[:, 3].sum() == 3 * (poff[i + 1] - poff[i])
            assert np.array_equal(ch[1:, 2], ch[:-1, 2] + ch[:-1, 3])
            pop = np.array([bin(x).count("1") for x in umask[uoff[i]:uoff[i + 1]]])
            assert np.array_equal(ch[:, 3], [3 * pop[64 * c:64 * c + 64].sum() for c in range(len(ch))])
    for i, (union, mask, v) in enumerate(tiles):
        a, e = uoff[i], uoff[i + 1]
        assert (e - a) % 4 == 0 and e - a == (len(union) + 3) // 4 * 4
        assert np.array_equal(ucol[a:a + len(union)], union)
        assert np.array_equal(umask[a:a + len(union)], mask)
        assert not umask[a + len(union):e].any()
        assert poff[i + 1] - poff[i] == len(v) // 3
        got = vals[3 * poff[i]:3 * poff[i + 1]]
        want = v if precision == "fp64" else _round44(v)
        assert np.array_equal(got, want), i


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tiled_block_pcg_matches_single_group_spmm(precision):
    from feab200.batched import block_pcg
    b = _batch()
    op = b.op
    B = b.rhs_panel()
    res = {}
    for tiles in (True, False):
        X, r = block_pcg(op, b.row_bounds, B, b.cols, tol=1e-10, precision=precision, max_groups=8, tile_width=4,
                         tune=False, node_tiles=tiles)
        assert (r.status == 0).all()
        res[tiles] = (X, r)
    (Xt, rt), (Xg, rg) = res[True], res[False]
    assert float(torch.linalg.norm(Xt - Xg) / torch.linalg.norm(Xg)) < 1e-8
    assert np.abs(rt.iters.astype(int) - rg.iters.astype(int)).max() <= 2


def test_items_must_be_whole_tiles():
    from feab200 import _lib as L
    from feab200.batched import _block_pcg_call, _problem_groups, _work_items
    b = _batch()
    op = b.op
    gp = op.pattern.group_ptr.cpu().numpy()
    pg = _problem_groups(gp, b.row_bounds)
    B = b.rhs_panel()
    items = _work_items(gp, b.row_bounds, 6)          # 6 groups per item: not whole 4-group tiles
    with pytest.raises(ValueError):
        _block_pcg_call(op, *items, B, b.cols, 1e-8, 10, "fp64", 0.1, 4, pg)
    bad = L.TileOperator()
    bad.n_groups = op.pattern.n_groups + 1              # a tile operator of another operator
    csr = op.csr_struct()
    X = torch.empty_like(B)
    assert L.lib.feab_block_spmm(C.byref(csr), C.byref(bad), L.dptr(B), L.dptr(X), B.shape[1],
                                 L.stream_ptr(B.device)) == L.FEAB_BAD_ARG


def test_tile_operator_rejects_bad_problem_boundaries():
    b = _batch()
    op = b.op
    G = op.pattern.n_groups
    for pg in ([0, G // 2, G // 2, G], [1, G], [0, G - 1]):
        with pytest.raises(ValueError):
            op.tile_operator("fp64", pg)
