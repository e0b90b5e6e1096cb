"""Delta-gap voltages and antenna currents (fwgpu_set_element_source: the
right-hand side of tet_MakeElement_EM_E, lib/fem/make_elem_em.c:66-330) on
the GPU against the reference's own runs: the assembled right-hand sides bit
for bit, the solutions to the solve tolerance."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm
from helpers import golden, rel_l2
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["gap", "antenna"])
def test_element_source_vs_reference(name):
    z, params, model = golden(name)
    with hddm.HddmSolver(model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
        s.make_tmp_aij(None)
        for k in range(model.nsub):
            rp, col, val, b = s.tmp_aij(k)
            assert np.array_equal(val, z[f"s{k}_aij_val"])
            assert np.array_equal(b, z[f"s{k}_aij_b"]), "element right-hand side must be bit-identical"
        r = s.solve(None)
        x = s.edge_solution()
        # the element source stays in place for a second solve
        r2 = s.solve(None)
        x2 = s.edge_solution()
    assert r.converged
    assert abs(r.iterations - int(z["iterations"][0])) <= max(2, int(0.05 * int(z["iterations"][0])))
    assert r.initial_norm == pytest.approx(float(z["norm0"][0]), rel=1e-6)
    assert rel_l2(x, z["x"]) <= 1e-8
    assert np.array_equal(x, x2) and r2.iterations == r.iterations


def test_element_source_plus_edge_source_and_clearing():
    """An edge source adds to the element source; clearing the element
    source leaves the edge source alone."""
    z, params, model = golden("antenna")
    rng = np.random.default_rng(3)
    edges = np.sort(rng.choice(model.n_edges, 5, replace=False)).astype(np.int32)
    vals = rng.standard_normal(5) + 1j * rng.standard_normal(5)
    part_both = oracle.partition(model, (edges, vals))
    xo_both, _, _, _ = oracle.hddm(model, part_both, 1e-11, 5000)
    es = model.element_source
    model.element_source = None
    part_edge = oracle.partition(model, (edges, vals))
    xo_edge, _, _, _ = oracle.hddm(model, part_edge, 1e-11, 5000)
    model.element_source = es
    with hddm.HddmSolver(model, hddm_eps=1e-11, hddm_max_loop=5000) as s:
        s.solve((edges, vals))
        x_both = s.edge_solution()
        s.set_element_source(None)
        s.solve((edges, vals))
        x_edge = s.edge_solution()
    assert rel_l2(x_both, xo_both) <= 1e-8
    assert rel_l2(x_edge, xo_edge) <= 1e-8
    assert rel_l2(x_both, x_edge) > 1e-3


def test_element_source_in_every_source_of_a_batched_solve():
    """The element source is added to each source of fwgpu_hddm_solve_multi,
    as it is to a one-source solve."""
    z, params, model = golden("antenna")
    rng = np.random.default_rng(11)
    srcs = []
    for _ in range(3):
        e = np.sort(rng.choice(model.n_edges, 4, replace=False)).astype(np.int32)
        srcs.append((e, rng.standard_normal(4) + 1j * rng.standard_normal(4)))
    with hddm.HddmSolver(model, hddm_eps=1e-11, hddm_max_loop=5000) as s:
        res = s.solve_multi(srcs)
        xs = [s.edge_solution_multi(k) for k in range(3)]
        singles = []
        for k in range(3):
            s.solve(srcs[k])
            singles.append(s.edge_solution())
    for k in range(3):
        assert res[k].converged
        assert rel_l2(xs[k], singles[k]) <= 1e-8
    assert rel_l2(xs[0], xs[1]) > 1e-3


def test_element_source_argument_errors():
    import ctypes

    from adventure_fullwave_b200 import _lib

    z, params, model = golden("gap")
    with hddm.HddmSolver(model) as s:
        lib = _lib.load()
        bad = _lib.FwElementSource(2, None, None, 0, None, None, None)
        assert lib.fwgpu_set_element_source(s._h, ctypes.byref(bad)) == _lib.ERR_ARG
        bad = _lib.FwElementSource(0, None, None, 1, None, None, None)
        assert lib.fwgpu_set_element_source(s._h, ctypes.byref(bad)) == _lib.ERR_ARG
        bad = _lib.FwElementSource(-1, None, None, 0, None, None, None)
        assert lib.fwgpu_set_element_source(s._h, ctypes.byref(bad)) == _lib.ERR_ARG
        # the source set at creation is still in place
        r = s.solve(None)
        assert r.converged and r.initial_norm == pytest.approx(float(z["norm0"][0]), rel=1e-6)
