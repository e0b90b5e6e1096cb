"""Failure paths of the C ABI on the GPU, each made on the host from bad
input (no GPU fault is involved): a negatively oriented element, a
subdomain whose matrix is not finite, and a non-finite right-hand side.

The reference has no error handling for any of these: emessage() exits on
a negative volume (lib/fem/tetrahedral.c tet_Volume6 users), a zero pivot
gives inf silently (lib/hddm/advlas_skyline.c:122), and a NaN residual
runs COCG on to hddm_max_loop (lib/hddm/hddm_solver_s.h:318-379).  The
library returns status codes instead."""
import numpy as np
import pytest

from adventure_fullwave_b200 import _lib, hddm, meshgen

pytestmark = pytest.mark.gpu


def _model(**kw):
    m = meshgen.make_model("x", n=6, size=1.0, npml=1, nleaves=6, seed=1, **kw)
    meshgen.round_trip_material(m)
    return m


def test_inverted_element_is_a_mesh_error():
    m = _model()
    # the same tet with vertices 1 and 2 swapped: edges relabelled to match
    # (01,02,03,12,23,13 -> 02,01,03,12,13,23), orientation negative
    t = 5
    m.tets = m.tets.copy()
    m.tet_edges = m.tet_edges.copy()
    m.tets[t] = m.tets[t][[0, 2, 1, 3]]
    m.tet_edges[t] = m.tet_edges[t][[1, 0, 2, 3, 5, 4]]
    with hddm.HddmSolver(m, hddm_eps=1e-6) as s:
        with pytest.raises(_lib.FwgpuError) as e:
            s.make_tmp_aij(0)
        assert e.value.code == _lib.ERR_MESH


def test_non_finite_subdomain_matrix_is_a_breakdown():
    """A NaN permittivity on the elements of subdomain 0: its assembled
    matrix, and with it the first pivot that meets a NaN entry, is not
    finite.  (No material table gives an exactly singular subdomain: the
    element matrix always holds the (nu/omega) curl-curl term,
    make_elem_em.c:227-232, whose null space rounding turns into tiny but
    finite pivots.)"""
    m = _model()
    f = int(m.mat_flag.max()) + 1
    m.mat_flag = np.append(m.mat_flag, f).astype(np.int32)
    m.mat_eps = np.append(m.mat_eps, np.nan)
    m.mat_sigma = np.append(m.mat_sigma, 0.0)
    m.flag = np.where(m.sub_of_tet == 0, f, m.flag).astype(np.int32)
    with hddm.HddmSolver(m, hddm_eps=1e-6) as s:
        s.make_tmp_aij(0)
        with pytest.raises(_lib.FwgpuError) as e:
            s.solve_dom_1st()
        assert e.value.code == _lib.ERR_BREAKDOWN


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_nan_source_stops_the_loop(precision):
    m = _model()
    edges, vals = m.sources[0]
    bad = (edges, np.where(np.arange(vals.shape[0]) == 0, complex(np.nan, 0.0), vals))
    with hddm.HddmSolver(m, hddm_eps=1e-10, hddm_max_loop=3000, precision=precision) as s:
        with pytest.raises(_lib.FwgpuError) as e:
            s.solve(bad)
        assert e.value.code == _lib.ERR_NONFINITE
        # the context stays usable: a finite source solves normally
        r = s.resolve(0)
        assert r.converged and np.isfinite(s.edge_solution()).all()


def test_nan_source_in_a_batch_stops_that_source_only():
    m = _model(nsources=2)
    edges, vals = m.sources[0]
    bad = (edges, np.full(vals.shape[0], complex(np.inf, 0.0)))
    with hddm.HddmSolver(m, hddm_eps=1e-8, hddm_max_loop=3000) as s:
        with pytest.raises(_lib.FwgpuError) as e:
            s.solve_multi([m.sources[1], bad])
        assert e.value.code == _lib.ERR_NONFINITE


def test_copy_wait_timeout_is_reported():
    """The staged solves' bounded wait for a copy: with the test hook the
    first wait polls an mbarrier that nothing completes, gives up after a
    few polls, raises the error word, and the kernel still waits for its
    copies in flight before it exits.  The host reports FWGPU_ERR_TIMEOUT;
    the device stays usable (a context without the hook solves normally)."""
    m = _model()
    with hddm.HddmSolver(m, hddm_eps=1e-8, hddm_max_loop=3000, solve_kernel="warp", stall_copy_test=1) as s:
        s.make_tmp_aij(0)
        with pytest.raises(_lib.FwgpuError) as e:
            s.solve_dom_1st()
        assert e.value.code == _lib.ERR_TIMEOUT
    x, r = hddm.hddm_solver_CS(m, 0, hddm_eps=1e-8, hddm_max_loop=3000, solve_kernel="warp")
    assert r.converged and np.isfinite(x).all()
