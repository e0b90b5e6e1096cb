"""The reference's shipped sample model (main/fullwave/MODEL, read by
adventure_fullwave_b200.advio: 6 parts x 73 subdomains, 43,587 elements, one
antenna) solved through the C ABI with the antenna currents of the
reference's correction-Jo pre-solve, against the reference's own run to the
same hddm_eps (fixture tests/golden/ref_sample.npz, made by
tests/golden/make_sample.py)."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm

pytestmark = pytest.mark.gpu


def sample_model():
    import bench

    m, z = bench.sample_model()
    return z, m


def test_shipped_sample_vs_reference():
    z, m = sample_model()
    with hddm.HddmSolver(m, hddm_eps=float(z["eps"][0]), hddm_max_loop=40000) as s:
        r = s.solve(None)
        x = s.edge_solution()
    assert r.converged
    assert r.initial_norm == pytest.approx(float(z["norm0"][0]), rel=1e-6)
    ref_it = int(z["iterations"][0])
    assert abs(r.iterations - ref_it) <= 0.15 * ref_it
    stride = int(z["x_sample_stride"][0])
    xs = x[::stride]
    ref = z["x_sample"]
    # both runs stop at a max-norm relative residual of 1e-6
    assert np.linalg.norm(xs - ref) <= 1e-5 * np.linalg.norm(ref)
    assert np.linalg.norm(x) == pytest.approx(float(z["x_norm"][0]), rel=1e-5)
