"""Regenerate tests/golden/gridone.npy from the reference's HDF5 golden grid.

The reference's GridderState.GridOne test (tests/GridderStateUnitTests.cc
:1343-1463) compares a gridded single visibility, bit for bit, with the
91x91 complex128 dataset "grid" in tests/gridone.h5.  HDF5 is not installed
here; the file stores the dataset as one deflate-compressed chunk, so zlib
alone recovers it.  The chunk starts at byte 4080 and inflates to
91*91*16 bytes, row-major [x - 9523][y - 8522] (the test's indexing at
GridderStateUnitTests.cc:1433-1438).

    python tests/golden/make_gridone.py path/to/hpg/tests/gridone.h5
"""
import json
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CHUNK_OFFSET = 4080
SHAPE = (91, 91)


def main(src):
    raw = open(src, "rb").read()
    data = zlib.decompressobj().decompress(raw[CHUNK_OFFSET:])
    assert len(data) == SHAPE[0] * SHAPE[1] * 16, len(data)
    grid = np.frombuffer(data, dtype="<c16").reshape(SHAPE)
    np.save(os.path.join(HERE, "gridone.npy"), grid)
    meta = {
        "source": "tests/gridone.h5 of hannajonathan/hpg (dataset 'grid')",
        "test": "tests/GridderStateUnitTests.cc:1343-1463 (GridderState.GridOne)",
        "grid_size": [16384, 16384, 1, 1],
        "grid_scale": [0.0476591, 0.0476591],
        "cf_radius": 45,
        "cf_oversampling": 20,
        "freq": 3.693e9,
        "vis": [1.0, -1.0],
        "weight": 1.0,
        "uvw": [2344.1, 638.066, -1826.55],
        "footprint_ll": [9523, 8522],
        "footprint_ur": [9613, 8612],
        "index": "golden[x - 9523, y - 8522]",
    }
    with open(os.path.join(HERE, "gridone.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", os.path.join(HERE, "gridone.npy"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_gridone.py path/to/hpg/tests/gridone.h5")
    main(sys.argv[1])
