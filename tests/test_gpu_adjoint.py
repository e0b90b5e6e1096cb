"""The adjoint (backward) of the C ABI against the FP64 reference gradient of
the oracle and against central finite differences of GPU forward solves."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm, meshgen
from test_oracle_adjoint import perturbed, small_design_model
from oracle import oracle

pytestmark = pytest.mark.gpu


def gpu_objective(model, hddm_eps=1e-12, hddm_max_loop=20000):
    with hddm.HddmSolver(model, hddm_eps=hddm_eps, hddm_max_loop=hddm_max_loop) as s:
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


def test_c4_gradient_vs_central_differences():
    """C4 (the C2 mesh, 663,552 tets, with 10,368 design tets of their own
    complex eps_r): the adjoint gradient against central differences of
    forward solves at 16 seeded design tets, for the real and the imaginary
    part of eps_r (eps = eps0 eps', sigma = omega eps0 eps'', the
    reference's convention).

    One tet moves J very little: with a step of 1e-6 |eps_r| the change of J
    is about 1e-10 of J, the size of the solves' own error.  The 16 tets are
    therefore drawn (seeded) from the 5 % of the design region with the
    largest gradient, the step is 1e-4 |eps_r| (the central difference's
    truncation error is then about 1e-8 relative) and every solve runs to
    hddm_eps 1e-12; each tet's difference quotient must agree with its
    gradient to 1e-3."""
    eps0 = meshgen.EPS0
    m = meshgen.make_model("c4")
    meshgen.round_trip_material(m)
    assert m.design_tets.shape[0] == 10368
    tol = dict(hddm_eps=1e-12, hddm_max_loop=100000)
    with hddm.HddmSolver(m, **tol) as s:
        s.solve(0)
        J, ge, gs, ra = s.adjoint_gradient()
    assert ra.converged
    d_re, d_im = hddm.relative_permittivity_gradient(ge, gs, m.omega, eps0)
    rng = np.random.default_rng(2024)
    worst = 0.0
    for part, d in (("re", d_re), ("im", d_im)):
        top = np.argsort(-np.abs(d))[: d.shape[0] // 20]
        for k in rng.choice(top, 8, replace=False):
            t = int(m.design_tets[k])
            i = int(np.searchsorted(m.mat_flag, m.flag[t]))
            er = complex(m.mat_eps[i] / eps0, m.mat_sigma[i] / (m.omega * eps0))
            h = 1e-4 * abs(er)
            if part == "re":
                plus, minus = perturbed(m, t, d_eps=eps0 * h), perturbed(m, t, d_eps=-eps0 * h)
            else:
                plus, minus = perturbed(m, t, d_sigma=m.omega * eps0 * h), perturbed(m, t, d_sigma=-m.omega * eps0 * h)
            fd = (gpu_objective(plus, **tol) - gpu_objective(minus, **tol)) / (2 * h)
            dev = abs(fd - d[k]) / abs(d[k])
            worst = max(worst, dev)
            print(f"C4 tet {t} eps_r {part}: adjoint {d[k]:+.6e}, central difference {fd:+.6e}, rel dev {dev:.1e}")
            assert dev <= 1e-3
    print(f"C4 FD vs adjoint, 16 tets (8 eps', 8 eps''): worst rel dev {worst:.1e}")
