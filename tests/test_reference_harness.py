"""Runs the reference itself (oracle/_ref/fw_ref_harness, built from the
reference's sources) on a fresh synthetic model and checks the oracle
restatement against it bit for bit.  Skipped where the harness is not built."""
import os

import numpy as np
import pytest

import refdump
from adventure_fullwave_b200 import meshgen
from oracle import oracle

pytestmark = pytest.mark.skipif(not os.path.exists(refdump.HARNESS), reason="reference harness not built")


def test_fresh_model_bitwise():
    m = meshgen.make_model("x", n=6, size=1.5, npml=1, layers=3, nleaves=None, leaf_cap=150, jitter=(0.3, 0.7),
                           seed=11)
    meshgen.round_trip_material(m)
    ref = refdump.run_harness(m, 1e-8, 3000, dump=1)
    part = oracle.partition(m)
    assert part.tfree == ref["infree"]
    xe, per_sub, hist, norm0 = oracle.hddm(m, part, 1e-8, 3000)
    assert len(hist) == ref["json"]["iterations"]
    assert np.array_equal(xe, ref["x"])
