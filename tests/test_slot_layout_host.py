"""Room of a 3x3 solve slot in the sliced-ELL layout (no GPU).

The slice sizes follow k_sell_rank: each window of 256 block rows is sorted
by stored length (+1 when the diagonal is absent; longest first, ties in
row order) and cut into slices of RS = 32 / L rows, a slice taking
32 x ceil(longest / L) entries. The library reserves, per slot,
nnzb + rows + windows x (RS x 96 + 256 x (L - 1)) entries; these tests
restate the sizing, check the bound on Tet10 box patterns and on random
rows of up to 96 blocks, and reproduce the layout size the library reported
for the refused system of tests/test_gpu_slots.py (rows of 1,000 blocks)."""

import numpy as np
import scipy.sparse as sp

ROWS, SLOT_ROW = 256, 96


def sliced_entries(lengths, lanes=4, sort=True):
    rs = 32 // lanes
    total = 0
    for w0 in range(0, len(lengths), ROWS):
        win = np.asarray(lengths[w0:w0 + ROWS])
        if sort:
            win = win[np.lexsort((np.arange(len(win)), -win))]
        for s0 in range(0, len(win), rs):
            total += 32 * -(-int(win[s0:s0 + rs].max()) // lanes)
    return total


def room(nnzb, rows, lanes=4):
    rs = 32 // lanes
    return nnzb + rows + -(-rows // ROWS) * (rs * SLOT_ROW + ROWS * (lanes - 1))


def _tet10_lengths(shape):
    from cloudfem_b200.mesh import box_mesh_tet10
    m = box_mesh_tet10(*shape)
    e = np.asarray(m.elements)
    inc = sp.csr_matrix((np.ones(e.size), (np.repeat(np.arange(len(e)), 10), e.ravel())),
                        shape=(len(e), m.n_nodes))
    pat = (inc.T @ inc).tocsr()
    return np.diff(pat.indptr), pat.nnz, m.n_nodes   # the diagonal is in the pattern


def test_tet10_box_patterns_fit_the_room():
    for shape in [(4, 4, 4), (24, 3, 3), (10, 10, 2), (16, 2, 2)]:
        lengths, nnzb, n = _tet10_lengths(shape)
        assert lengths.max() <= 65
        need = sliced_entries(lengths)
        assert nnzb <= need <= room(nnzb, n), shape
        # rows sorted per window keep the padding to a few per cent
        assert need <= 1.15 * nnzb + 4 * n


def test_rows_up_to_the_slot_row_fit_for_every_lane_count():
    rng = np.random.default_rng(2)
    for lanes in (1, 2, 4):
        for n in (1, 255, 257, 3000):
            lengths = rng.integers(1, SLOT_ROW + 1, n)
            assert sliced_entries(lengths, lanes) <= room(int(lengths.sum()), n, lanes)


def test_refused_system_size_matches_the_library():
    n = 2560
    lengths = np.ones(n, dtype=int)
    lengths[::256] = 1000
    assert sliced_entries(lengths) == 89920
    assert room(5 * n, n) == 30720
