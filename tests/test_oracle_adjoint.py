"""The FP64 reference gradient of the oracle against central finite
differences of the oracle's own solves (CPU)."""
import copy

import numpy as np

from adventure_fullwave_b200 import meshgen
from oracle import oracle


def small_design_model():
    m = meshgen.make_model("adj", n=10, size=1.5, npml=2, layers=2, nleaves=8, design=2, nprobes=4, seed=2)
    meshgen.round_trip_material(m)
    return m


def perturbed(model, t, d_eps=0.0, d_sigma=0.0):
    m = copy.copy(model)
    m.mat_eps = model.mat_eps.copy()
    m.mat_sigma = model.mat_sigma.copy()
    i = int(np.searchsorted(m.mat_flag, m.flag[t]))
    m.mat_eps[i] += d_eps
    m.mat_sigma[i] += d_sigma
    return m


def test_oracle_gradient_matches_finite_differences():
    m = small_design_model()
    assert m.design_tets.shape[0] == 48 and m.probe_edges.shape[0] == 4
    picks = m.design_tets[[0, 23, 47]]
    J, ge, gs, _ = oracle.adjoint_gradient(m, m.probe_edges, picks)
    assert J > 0
    for k, t in enumerate(picks):
        i = int(np.searchsorted(m.mat_flag, m.flag[t]))
        he = 1e-5 * m.mat_eps[i]
        fd = (oracle.objective(perturbed(m, t, d_eps=he), m.probe_edges)
              - oracle.objective(perturbed(m, t, d_eps=-he), m.probe_edges)) / (2 * he)
        assert abs(fd - ge[k]) <= 1e-4 * np.max(np.abs(ge)), (k, fd, ge[k])
        hs = 1e-5 * m.omega * meshgen.EPS0
        fd = (oracle.objective(perturbed(m, t, d_sigma=hs), m.probe_edges)
              - oracle.objective(perturbed(m, t, d_sigma=-hs), m.probe_edges)) / (2 * hs)
        assert abs(fd - gs[k]) <= 1e-4 * np.max(np.abs(gs)), (k, fd, gs[k])
