"""The reference's shipped sample model (main/fullwave/MODEL, read by
adventure_fullwave_b200.advio: 6 parts x 73 subdomains, 43,587 elements, one
antenna) solved through the C ABI with the antenna currents of the
reference's correction-Jo pre-solve, against the reference's own run to the
same hddm_eps (fixture tests/golden/ref_sample.npz, made by
tests/golden/make_sample.py)."""
import os

import numpy as np
import pytest

from adventure_fullwave_b200 import advio, hddm, meshgen
from helpers import GOLDEN

pytestmark = pytest.mark.gpu


def sample_model():
    z = np.load(os.path.join(GOLDEN, "ref_sample.npz"))
    tets = z["tets"]
    tet_edges = z["tet_edges"]
    ne = int(tet_edges.max()) + 1
    edges = np.zeros((ne, 2), np.int32)
    for q, (a, b) in enumerate(advio._MID_PAIRS):
        edges[tet_edges[:, q], 0] = np.minimum(tets[:, a], tets[:, b])
        edges[tet_edges[:, q], 1] = np.maximum(tets[:, a], tets[:, b])
    m = meshgen.Model(name="sample", n=0, size=0.0, vertex_crd=z["vertex_crd"], tets=tets, tet_edges=tet_edges,
                      edges=edges, flag=z["flag"].astype(np.int32), mat_flag=z["mat_flag"], mat_eps=z["mat_eps"],
                      mat_sigma=z["mat_sigma"], omega=float(z["omega"][0]), pec_edge=np.zeros(ne, bool),
                      sub_of_tet=z["sub_of_tet"].astype(np.int32), nsub=int(z["nsub"][0]), sources=[])
    nv = m.n_vertices
    jo = np.zeros((1, nv, 3))
    jor = np.zeros((1, nv, 3))
    jo[0, z["antenna_vertices"]] = z["antenna_Jo"]
    jor[0, z["antenna_vertices"]] = z["antenna_Jor"]
    meshgen.antenna_source(m, z["antenna_flag"], jo, jor)
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
