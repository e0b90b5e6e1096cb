"""Several sources on one set of factors (``fwgpu_hddm_solve_multi``): each
source's solution against the one-source solve of the same model, on a C5-
style model in miniature (random layers, 5 % high-permittivity inclusions,
16 seeded dipoles)."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm, meshgen
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _model(nsources):
    m = meshgen.make_model("c5", n=12, size=1.0, npml=2, leaf_cap=200, seed=7, nsources=nsources)
    meshgen.round_trip_material(m)
    return m


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_sixteen_sources_match_one_at_a_time(precision):
    m = _model(16)
    assert len(m.sources) == 16 and m.nsub > 4
    opts = dict(hddm_eps=1e-10, hddm_max_loop=20000, precision=precision, ir_max_steps=2)
    with hddm.HddmSolver(m, **opts) as s:
        res = s.solve_multi(list(range(16)))
        xs = [s.edge_solution_multi(k) for k in range(16)]
    with hddm.HddmSolver(m, hddm_eps=1e-10, hddm_max_loop=20000) as s1:
        for k in (0, 5, 15):
            r1 = s1.solve(k) if k == 0 else s1.resolve(k)
            x1 = s1.edge_solution()
            assert res[k].converged
            assert rel_l2(xs[k], x1) <= (1e-8 if precision == "fp64" else 1e-6)
            assert abs(res[k].iterations - r1.iterations) <= max(3, r1.iterations // 10)
    # the sources are different problems
    assert rel_l2(xs[0], xs[1]) > 1e-2


def test_fewer_sources_and_a_zero_source():
    m = _model(3)
    with hddm.HddmSolver(m, hddm_eps=1e-10, hddm_max_loop=20000) as s:
        res = s.solve_multi([0, None, 2])
        x0, xz, x2 = (s.edge_solution_multi(k) for k in range(3))
        assert res[1].iterations == 0 and np.all(xz == 0)
        s.resolve(2)
        assert rel_l2(x2, s.edge_solution()) <= 1e-8
        s.resolve(0)
        assert rel_l2(x0, s.edge_solution()) <= 1e-8
        with pytest.raises(Exception):
            s.edge_solution_multi(3)


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_batched_adjoint_matches_one_source_at_a_time(precision):
    """fwgpu_adjoint_gradient_multi: the adjoint of 4 sources in one batched
    solve on the forward factors gives each source's J and gradient as the
    one-source forward/backward pair does (FP64: 1e-8 of max |g|; FP32
    factors with FP64 refinement: 1e-5)."""
    m = meshgen.make_model("adj", n=10, size=1.5, npml=2, layers=2, nleaves=8, design=2, nprobes=4, seed=2,
                           nsources=4)
    meshgen.round_trip_material(m)
    opts = dict(hddm_eps=1e-12, hddm_max_loop=20000, precision=precision, ir_max_steps=2)
    with hddm.HddmSolver(m, **opts) as s:
        s.solve_multi([0, 1, 2, 3])
        J, ge, gs, res = s.adjoint_gradient_multi()
        assert all(r.converged for r in res)
    tol = 1e-8 if precision == "fp64" else 1e-5
    for k in range(4):
        with hddm.HddmSolver(m, **opts) as s1:
            s1.solve(k)
            J1, ge1, gs1, _ = s1.adjoint_gradient()
        assert J[k] == pytest.approx(J1, rel=tol)
        assert np.max(np.abs(ge[k] - ge1)) <= tol * np.max(np.abs(ge1))
        assert np.max(np.abs(gs[k] - gs1)) <= tol * np.max(np.abs(gs1))
