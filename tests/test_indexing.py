"""CFSimpleIndexer (reference src/hpg_indexing.hpp:67-181), with the
reference's own cases restated (tests/CFIndexerUnitTests.cc)."""
import itertools

import numpy as np

from hpg_b200.indexing import CFCellIndex, CFSimpleIndexer


def test_mixed_radix_known_values():
    ix = CFSimpleIndexer((3, False), (2, True), (4, False), (5, True), 2)
    # cube over (baseline class, w plane), group over (time, frequency)
    assert ix.cf_index(CFCellIndex(2, 1, 3, 4, 1)) == (1, 2 * 4 + 3, 1 * 5 + 4)
    assert ix.cf_extents() == (2, 12, 10)
    assert ix.cell_extents() == (3, 2, 4, 5, 2)


def test_round_trip_every_cell():
    ix = CFSimpleIndexer((2, True), (3, False), (4, True), (2, False), 3)
    seen = set()
    for bc, t, w, f, m in itertools.product(range(2), range(3), range(4),
                                            range(2), range(3)):
        cell = CFCellIndex(bc, t, w, f, m)
        idx = ix.cf_index(cell)
        assert ix.cell_index(idx) == cell
        m_ext, c_ext, g_ext = ix.cf_extents()
        assert idx[0] < m_ext and idx[1] < c_ext and idx[2] < g_ext
        seen.add(idx)
    assert len(seen) == 2 * 3 * 4 * 2 * 3


def test_vectorised_matches_scalar():
    ix = CFSimpleIndexer((3, False), (2, True), (4, False), (5, True), 1)
    rng = np.random.default_rng(0)
    bc, t, w, f = (rng.integers(0, n, 100) for n in (3, 2, 4, 5))
    cube, grp = ix.cf_index_arrays(bc, t, w, f)
    for k in range(100):
        _, c, g = ix.cf_index(CFCellIndex(bc[k], t[k], w[k], f[k], 0))
        assert (cube[k], grp[k]) == (c, g)


def test_reference_extents_every_variability():
    """CFSimpleIndexer.Extents (tests/CFIndexerUnitTests.cc:19-48)."""
    nb, nt, nw, nf, nm = 1, 2, 3, 4, 5
    for bv, tv, wv, fv in itertools.product((False, True), repeat=4):
        cube = grp = 1
        for n, v in ((nb, bv), (nt, tv), (nw, wv), (nf, fv)):
            if v:
                grp *= n
            else:
                cube *= n
        ix = CFSimpleIndexer((nb, bv), (nt, tv), (nw, wv), (nf, fv), nm)
        assert ix.cf_extents() == (nm, cube, grp)


def test_reference_examples():
    """CFSimpleIndexer.Examples (tests/CFIndexerUnitTests.cc:50-102)."""
    nb, nt, nw, nf, nm = 2, 2, 3, 4, 8
    ix = CFSimpleIndexer((nb, True), (nt, False), (nw, True), (nf, True), nm)
    cases = [((0, 0, 0, 0, 0), (0, 0, 0)),
             ((1, 0, 0, 0, 0), (0, 0, nw * nf)),
             ((1, 0, 2, 0, 0), (0, 0, nw * nf + 2 * nf)),
             ((1, 0, 2, 0, 1), (1, 0, nw * nf + 2 * nf)),
             ((1, 1, 2, 0, 0), (0, 1, nw * nf + 2 * nf)),
             ((1, 1, 2, 0, 1), (1, 1, nw * nf + 2 * nf)),
             ((1, 1, 2, 3, 1), (1, 1, nw * nf + 2 * nf + 3))]
    for cell, idx in cases:
        assert ix.cf_index(CFCellIndex(*cell)) == idx
        assert ix.cell_index(idx) == CFCellIndex(*cell)
