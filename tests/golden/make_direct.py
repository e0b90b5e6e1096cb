"""Writes tests/golden/direct_c1.npz: the exact discrete solution of C1 (the
FP64 sparse direct solve of the global system, oracle/direct.py) on every
edge.  bench.py states the error of its C1 solves against it; the tests
compute the direct solve afresh.

    python tests/golden/make_direct.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from adventure_fullwave_b200 import meshgen  # noqa: E402
from oracle import direct  # noqa: E402

if __name__ == "__main__":
    model = meshgen.make_model("c1")
    meshgen.round_trip_material(model)
    x = direct.solve(model, 0)
    path = os.path.join(HERE, "direct_c1.npz")
    np.savez_compressed(path, x=x, n_edges=np.array([model.n_edges]))
    print(path, os.path.getsize(path))
