"""The adjoint (backward) of the C ABI against the FP64 reference gradient of
the oracle and against central finite differences of GPU forward solves."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm
from test_oracle_adjoint import perturbed, small_design_model
from oracle import oracle

pytestmark = pytest.mark.gpu


def gpu_objective(model):
    with hddm.HddmSolver(model, hddm_eps=1e-12, hddm_max_loop=20000) as s:
        s.solve(0)
        x = s.edge_solution()
    return float(np.sum(np.abs(x[model.probe_edges]) ** 2))


def test_adjoint_vs_reference_gradient_and_fd():
    m = small_design_model()
    with hddm.HddmSolver(m, hddm_eps=1e-12, hddm_max_loop=20000) as s:
        r = s.solve(0)
        x_fwd = s.edge_solution()
        J, ge, gs, ra = s.adjoint_gradient()
        x_after = s.edge_solution()
    assert r.converged and ra.converged
    assert np.array_equal(x_fwd, x_after)
    Jo, geo, gso, xo = oracle.adjoint_gradient(m, m.probe_edges, m.design_tets)
    assert J == pytest.approx(Jo, rel=1e-9)
    assert np.max(np.abs(ge - geo)) <= 1e-7 * np.max(np.abs(geo))
    assert np.max(np.abs(gs - gso)) <= 1e-7 * np.max(np.abs(gso))
    for k in (0, 23, 47):
        t = m.design_tets[k]
        i = int(np.searchsorted(m.mat_flag, m.flag[t]))
        he = 1e-5 * m.mat_eps[i]
        fd = (gpu_objective(perturbed(m, t, d_eps=he)) - gpu_objective(perturbed(m, t, d_eps=-he))) / (2 * he)
        assert abs(fd - ge[k]) <= 1e-4 * np.max(np.abs(ge))


def test_adjoint_requires_a_forward_solve():
    from adventure_fullwave_b200 import _lib

    m = small_design_model()
    with hddm.HddmSolver(m) as s:
        with pytest.raises(_lib.FwgpuError) as e:
            s.adjoint_gradient()
        assert e.value.code == _lib.ERR_STATE
