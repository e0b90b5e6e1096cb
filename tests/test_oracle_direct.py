"""The FP64 sparse direct solve of the global system (oracle/direct.py)
against the reference's own HDDM solution of C1 at hddm_eps 1e-10: the
HDDM's error against the exact discrete solution is of the order of its
stopping tolerance (the oracle's: 3.9e-6 at 1e-6, 3.5e-10 at 1e-10), so at
1e-10 the two agree to 1e-9 relative L2.  This pins the direct solve
(assembly, PEC elimination, source) to the reference's discrete problem."""
import numpy as np

from helpers import golden, rel_l2
from oracle import direct


def test_direct_solve_vs_reference_c1():
    z, params, model = golden("c1")
    assert params["eps"] == 1e-10
    xd = direct.solve(model, 0)
    assert rel_l2(z["x"], xd) <= 1e-9
    # the PEC wall holds zero in both
    assert np.all(xd[model.pec_edge.astype(bool)] == 0)
