"""The drop-in table (adventure_fullwave_b200/dropin/set_hddm_func_gpu.c)
compiled against the reference and run by the reference's own driver:
main()'s flow with hddm_solver_CS (lib/hddm/hddm_solver.h:25-183) walking
set_hddm_func_fullwave_gpu instead of set_hddm_func_fullwave, on C1 to
hddm_eps 1e-10.  Its solution equals the plain reference run's to 1e-8
relative L2 over every edge, the same bar as the library's own C1 test."""
import os

import numpy as np
import pytest

import refdump
from helpers import golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(refdump.HARNESS_GPU), reason="oracle/_ref/fw_ref_gpu is not built")
def test_reference_driver_through_the_gpu_table():
    z, params, model = golden("c1")
    out = refdump.run_harness(model, params["eps"], params["max_loop"], dump=0, binary=refdump.HARNESS_GPU,
                              timeout=600)
    n_ref = int(z["iterations"][0])
    n = int(out["json"]["iterations"])
    err = rel_l2(out["x"], z["x"])
    print(f"C1 through the GPU table: {n} iterations (reference {n_ref}), rel L2 vs the reference run {err:.2e}")
    assert np.isfinite(out["x"]).all()
    assert abs(n - n_ref) <= 0.05 * n_ref
    assert err <= 1e-8
    # the reference's own log of the GPU run: the DOF count line of hddm_solver_CS
    assert out["norm0"] is None or out["norm0"] > 0
