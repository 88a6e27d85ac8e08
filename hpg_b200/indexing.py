"""CF index bookkeeping: the reference's CFSimpleIndexer
(src/hpg_indexing.hpp:67-181).

A CF cell is addressed by (baseline class, time, w plane, frequency, Mueller
element).  The indexer maps it to the (mueller, cube, group) triple that
VisData.cf_index and the CF arrays use: the axes whose CF size may vary from
cell to cell ("variable" axes) are linearised, in the order baseline class,
time, w plane, frequency (first = most significant), into the group index;
the other axes, in the same order, into the cube index.
"""
from collections import namedtuple

import numpy as np

CFCellIndex = namedtuple(
    "CFCellIndex", ["baseline_class", "time", "w_plane", "frequency", "mueller"])

_AXES = ("baseline_class", "time", "w_plane", "frequency")


class CFSimpleIndexer:
    """Each axis is (length, variable); mueller is the Mueller axis length."""

    def __init__(self, baseline_class, time, w_plane, frequency, mueller):
        self.axes = [tuple(baseline_class), tuple(time), tuple(w_plane),
                     tuple(frequency)]
        for length, _ in self.axes:
            if length < 1:
                raise ValueError("axis lengths must be >= 1")
        self.mueller = int(mueller)

    def cf_index(self, cell):
        """CFCellIndex -> (mueller, cube, group)."""
        cube = grp = 0
        for (length, variable), i in zip(self.axes,
                                         (cell.baseline_class, cell.time,
                                          cell.w_plane, cell.frequency)):
            if variable:
                grp = grp * length + i
            else:
                cube = cube * length + i
        return (cell.mueller, cube, grp)

    def cell_index(self, index):
        """(mueller, cube, group) -> CFCellIndex."""
        mueller, cube, grp = index
        parts = {}
        for name, (length, variable) in reversed(list(zip(_AXES, self.axes))):
            if variable:
                parts[name] = grp % length
                grp //= length
            else:
                parts[name] = cube % length
                cube //= length
        return CFCellIndex(mueller=mueller, **parts)

    def cf_extents(self):
        """(mueller, number of cubes, number of groups)."""
        cube = grp = 1
        for length, variable in self.axes:
            if variable:
                grp *= length
            else:
                cube *= length
        return (self.mueller, cube, grp)

    def cell_extents(self):
        return tuple(length for length, _ in self.axes) + (self.mueller,)

    def cf_index_arrays(self, baseline_class, time, w_plane, frequency):
        """Vectorised cf_index for many visibilities: integer arrays of the
        four axes -> (cube, group) arrays, as VisData.cf_index takes them."""
        cube = np.zeros(np.shape(baseline_class), np.int64)
        grp = np.zeros_like(cube)
        for (length, variable), i in zip(self.axes,
                                         (baseline_class, time, w_plane,
                                          frequency)):
            i = np.asarray(i, np.int64)
            if variable:
                grp = grp * length + i
            else:
                cube = cube * length + i
        return cube.astype(np.uint32), grp.astype(np.uint32)
