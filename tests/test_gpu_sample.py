"""The reference's shipped sample model (main/fullwave/MODEL, read by
adventure_fullwave_b200.advio: 6 parts x 73 subdomains, 43,587 elements, one
antenna) solved through the C ABI with the antenna currents of the
reference's correction-Jo pre-solve, against the reference's own run to the
same hddm_eps (fixture tests/golden/ref_sample.npz, made by
tests/golden/make_sample.py).  Every subdomain keeps the part file's node
order, so the skyline profiles are the reference's bit for bit and the
factors agree to rounding."""
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
    err = np.linalg.norm(xs - ref) / np.linalg.norm(ref)
    print(f"sample: {r.iterations} iterations (reference {ref_it}), rel L2 vs the reference's solution {err:.2e}")
    assert err <= 1e-5
    assert np.linalg.norm(x) == pytest.approx(float(z["x_norm"][0]), rel=1e-5)


def test_shipped_sample_profiles_and_factors_vs_reference():
    """Skyline profiles (idx1, idx2, nlen) of all 438 subdomains bit-exact,
    and two subdomains' LDL^T factors to 1e-12, against the reference's own
    dump of its run on the sample."""
    z, m = sample_model()
    ptr = z["ref_dof_ptr"]
    with hddm.HddmSolver(m, hddm_eps=float(z["eps"][0]), hddm_max_loop=1) as s:
        s.make_tmp_aij(None)
        s.solve_dom_1st()
        for k in range(m.nsub):
            idx1, idx2, nlen = s.skyline_profile(k)
            assert np.array_equal(idx1, z["ref_idx1"][ptr[k]:ptr[k + 1]]), k
            assert np.array_equal(idx2, z["ref_idx2"][ptr[k]:ptr[k + 1]]), k
            assert nlen == int(z["ref_nlen"][k]), k
        for k in z["factor_subs"].tolist():
            ref = z[f"ref_factor_{k}"]
            fac = s.factor(k)
            assert fac.shape == ref.shape
            assert np.max(np.abs(fac - ref)) <= 1e-12 * np.max(np.abs(ref)), k
