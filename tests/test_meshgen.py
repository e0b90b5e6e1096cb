"""Synthetic model generator: sizes, orientation, PEC wall, partition."""
import numpy as np

from adventure_fullwave_b200 import meshgen


def test_c1_counts():
    m = meshgen.make_model("c1")
    n = 16
    assert m.n_tets == 6 * n ** 3 == 24576
    assert m.n_edges == 3 * n * (n + 1) ** 2 + 3 * n * n * (n + 1) + n ** 3 == 31024
    assert int(m.pec_edge.sum()) == 4608
    assert m.nsub == 64
    assert np.all(np.bincount(m.sub_of_tet) == 384)


def test_positive_orientation():
    m = meshgen.make_model("tiny", n=3, npml=1, nleaves=2)
    vol = meshgen._volume6(m.vertex_crd[m.tets])
    assert np.all(vol > 0)


def test_pml_profile():
    s = meshgen.pml_sigma(4, 1.0 / 16)
    assert s[0] == 0.0
    smax = -3.0 * np.log(1e-6) / (2 * 376.73 * 0.25)
    assert np.isclose(s[4], smax * (3.5 / 4) ** 2)


def test_jittered_partition_leaf_cap():
    m = meshgen.make_model("x", n=8, size=1.5, npml=2, layers=2, nleaves=None, leaf_cap=120, jitter=(0.3, 0.7),
                           seed=5)
    counts = np.bincount(m.sub_of_tet)
    assert counts.max() <= 120 and counts.min() >= 1
    m2 = meshgen.make_model("x", n=8, size=1.5, npml=2, layers=2, nleaves=None, leaf_cap=120, jitter=(0.3, 0.7),
                            seed=5)
    assert np.array_equal(m.sub_of_tet, m2.sub_of_tet)


def test_source_is_z_directed_near_centre():
    m = meshgen.make_model("c1")
    e, v = m.sources[0]
    assert e.shape[0] == 4 and np.allclose(v, -1j)
    d = m.vertex_crd[m.edges[e, 1]] - m.vertex_crd[m.edges[e, 0]]
    assert np.allclose(d[:, :2], 0.0)


def test_material_round_trip_is_stable():
    m = meshgen.make_model("x", n=6, size=1.5, npml=1, layers=3, nleaves=4)
    meshgen.round_trip_material(m)
    eps, sig, om = m.mat_eps.copy(), m.mat_sigma.copy(), m.omega
    meshgen.round_trip_material(m)
    assert np.array_equal(eps, m.mat_eps) and np.array_equal(sig, m.mat_sigma) and om == m.omega
