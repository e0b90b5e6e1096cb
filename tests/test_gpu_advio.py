"""A model directory in the reference's layout, read back with
adventure_fullwave_b200.advio and solved through the C ABI: the same solution
as the model it was written from, and the reference's own (delta-gap model)."""
import os
import tempfile

import numpy as np
import pytest

from adventure_fullwave_b200 import advio, hddm, meshgen
from helpers import golden, rel_l2

pytestmark = pytest.mark.gpu


def test_model_directory_round_trip_solves_the_same():
    z, params, model = golden("gap")
    with tempfile.TemporaryDirectory() as d:
        meshgen.write_hddm_model(model, d)
        loaded = advio.load_model(d)
        with hddm.HddmSolver(loaded.model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
            r = s.solve(None)
            x = s.edge_solution()
            B, E, Je = s.post_em_E()
        out = os.path.join(d, "out.adv")
        advio.write_result(out, loaded, 0, x, B=B, E=E, Je=Je)
        res = advio.read_result(out)
    with hddm.HddmSolver(model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
        s.solve(None)
        x0 = s.edge_solution()
    assert r.converged
    assert np.array_equal(x, x0)
    assert rel_l2(x, z["x"]) <= 1e-8
    p = loaded.parts[0]
    for s_, ge in enumerate(p.seid2geid):
        assert np.array_equal(res["ElectricFieldReal"][s_], E[ge].real)
        assert np.array_equal(res["CurrentDensityImaginary"][s_], Je[ge].imag)
