"""The reader and writer of the reference's model and result files
(adventure_fullwave_b200.advio): round trips through the part-file writer,
and the reference's shipped sample model and results where present."""
import os
import tempfile

import numpy as np
import pytest

from adventure_fullwave_b200 import advio, meshgen
from helpers import golden

SAMPLE = os.path.join(os.environ.get("FW_REFERENCE", "/root/reference"), "main", "fullwave", "MODEL")


@pytest.mark.parametrize("name", ["layered", "gap"])
def test_part_file_round_trip(name):
    z, params, model = golden(name)
    with tempfile.TemporaryDirectory() as d:
        meshgen.write_hddm_model(model, d)
        got = advio.load_model(d).model
    assert np.array_equal(got.vertex_crd, model.vertex_crd)
    assert np.array_equal(got.tets, model.tets)
    assert np.array_equal(got.tet_edges, model.tet_edges)
    assert np.array_equal(got.edges, model.edges)
    assert np.array_equal(got.flag, model.flag)
    assert np.array_equal(got.pec_edge, model.pec_edge)
    assert np.array_equal(got.sub_of_tet, model.sub_of_tet) and got.nsub == model.nsub
    assert np.array_equal(got.mat_flag, model.mat_flag)
    assert np.array_equal(got.mat_eps, model.mat_eps) and np.array_equal(got.mat_sigma, model.mat_sigma)
    assert got.omega == model.omega
    if model.element_source is not None:
        assert np.array_equal(got.element_source.gap_box, model.element_source.gap_box)
        assert np.array_equal(got.element_source.gap_volt, model.element_source.gap_volt)
    else:
        assert got.element_source is None


def test_result_round_trip():
    z, params, model = golden("layered")
    rng = np.random.default_rng(1)
    x = rng.standard_normal(model.n_edges) + 1j * rng.standard_normal(model.n_edges)
    B = rng.standard_normal((model.n_tets, 3)) + 1j * rng.standard_normal((model.n_tets, 3))
    with tempfile.TemporaryDirectory() as d:
        meshgen.write_hddm_model(model, d)
        loaded = advio.load_model(d)
        path = os.path.join(d, "out.adv")
        advio.write_result(path, loaded, 0, x, B=B)
        r = advio.read_result(path)
    p = loaded.parts[0]
    eidx = {int(g): k for k, g in enumerate(loaded.edge_gnid.tolist())}
    for s, rec in enumerate(r["MagneticVectorPotential"]):
        gn = p.pnid2gnid[p.snid2pnid[s]]
        assert np.all(np.diff(rec["snid"]) > 0)
        k = np.array([eidx[int(g)] for g in gn[rec["snid"]]])
        assert np.array_equal(rec["re"] + 1j * rec["im"], x[k])
        ge = p.seid2geid[s]
        assert np.array_equal(r["MagneticFieldReal"][s], B[ge].real)
        assert np.array_equal(r["MagneticFieldImaginary"][s], B[ge].imag)


@pytest.mark.skipif(not os.path.isdir(SAMPLE), reason="the reference's sample model is not on this machine")
def test_shipped_sample_model_and_results():
    loaded = advio.load_model(SAMPLE)
    m = loaded.model
    assert len(loaded.parts) == 6 and m.nsub == 6 * 73
    v = m.vertex_crd[m.tets]
    d6 = np.einsum("ij,ij->i", np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), v[:, 3] - v[:, 0])
    assert np.all(d6 > 0)
    # every edge joins two vertices of each element holding it
    assert np.all(m.edges[:, 0] < m.edges[:, 1])
    assert loaded.material.antennas == [(1, "md", "antenna.dat")]
    # the shipped results: one value per edge, the same in every subdomain holding it
    x = np.full(m.n_edges, np.nan + 0j)
    eidx = {int(g): k for k, g in enumerate(loaded.edge_gnid.tolist())}
    for q, p in enumerate(loaded.parts):
        r = advio.read_result(os.path.join(SAMPLE, "result", f"advhddm_out_{q}.adv"))
        for s, rec in enumerate(r["MagneticVectorPotential"]):
            gn = p.pnid2gnid[p.snid2pnid[s]]
            k = np.array([eidx[int(g)] for g in gn[rec["snid"]]])
            vals = rec["re"] + 1j * rec["im"]
            have = ~np.isnan(x[k].real)
            assert np.array_equal(x[k][have], vals[have])
            x[k] = vals
        assert len(r["ElectricFieldReal"]) == len(p.nop)
        # the writer gives the same layout: node ids per subdomain, element arrays per subdomain
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "out.adv")
            z3 = np.zeros((m.n_tets, 3), complex)
            advio.write_result(out, loaded, q, np.zeros(m.n_edges, complex), B=z3, E=z3, Je=z3)
            w = advio.read_result(out)
        assert set(w) == set(r)
        for label in r:
            for a, b in zip(w[label], r[label]):
                if label == "MagneticVectorPotential":
                    assert np.array_equal(a["snid"], b["snid"])
                else:
                    assert a.shape == b.shape
    assert not np.isnan(x.real).any()


def test_sample_fixture_matches_the_reader():
    """tests/golden/ref_sample.npz holds the shipped sample as this reader
    gives it; where the reference is present, read it again and compare."""
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_sample.npz"))
    assert int(z["nsub"][0]) == 438 and z["tets"].shape == (43587, 4)
    assert int(z["iterations"][0]) > 0 and z["antenna_vertices"].shape[0] > 0
    if not os.path.isdir(SAMPLE):
        return
    m = advio.load_model(SAMPLE).model
    assert np.array_equal(m.vertex_crd, z["vertex_crd"])
    assert np.array_equal(m.tets, z["tets"]) and np.array_equal(m.tet_edges, z["tet_edges"])
    assert np.array_equal(m.flag, z["flag"]) and np.array_equal(m.sub_of_tet, z["sub_of_tet"])
    assert m.omega == float(z["omega"][0])
    # the antenna currents built from the definition file equal those the
    # reference's own run left (the fixture's)
    es = m.element_source
    assert es is not None and list(es.antenna_flag) == list(z["antenna_flag"])
    jo = np.zeros((m.n_vertices, 3))
    jor = np.zeros((m.n_vertices, 3))
    jo[z["antenna_vertices"]] = z["antenna_Jo"]
    jor[z["antenna_vertices"]] = z["antenna_Jor"]
    assert np.array_equal(es.antenna_Jo[0], jo) and np.array_equal(es.antenna_Jor[0], jor)


def test_sample_maps_match_the_reference():
    """The shipped sample's integer setup with every subdomain in the part
    file's node order: nop, Dirichlet list, interface DOFs and the edge of
    every local DOF equal the reference's own (make_PartMesh_FW on the six
    parts, dumped by oracle/ref_harness.c), for all 438 subdomains."""
    import bench
    from adventure_fullwave_b200 import hddm

    m, z = bench.sample_model()
    part = hddm.Partition(m)
    assert part.n_subdomains == 438
    for k in range(m.nsub):
        got = part.maps(k)
        for key, name in (("nop", "nop"), ("ibc", "ibc"), ("inbc_nfid", "inbc_nfid")):
            p = z[f"ref_{key}_ptr"]
            assert np.array_equal(np.asarray(got[name]).ravel(), z[f"ref_{key}"][p[k]:p[k + 1]]), (k, key)
        d = z["ref_dof_ptr"]
        assert np.array_equal(got["edge_gid"], z["ref_edge"][d[k]:d[k + 1]]), k


def test_antenna_definition_shapes():
    """Parallelepiped and double sectorial cylinder definitions on a small
    model: currents only on vertices of the antenna's elements inside the
    shape; the cylinder's current is tangential with the given magnitude."""
    z, params, model = golden("antenna")
    flag = int(model.element_source.antenna_flag[0])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "a.dat")
        with open(path, "w") as f:
            f.write("Full-Wave\nParallelpiped\n0.5 0.5 0.5\n0.75 0.5 0.5\n0.5 0.75 0.5\n0.5 0.5 0.75\n"
                    "1.0 2.0 3.0  0.5 0.25 0.125\n")
        jo, jor = advio.antenna_currents(model, flag, advio.read_jodefine(path))
        c = model.vertex_crd
        inside = np.all((c >= 0.5 - 1e-12) & (c <= 0.75 + 1e-12), axis=1)
        held = np.zeros(model.n_vertices, bool)
        held[np.unique(model.tets[model.flag == flag])] = True
        assert np.array_equal(np.any(jor != 0, axis=1), inside & held)
        assert np.all(jor[inside & held] == [1.0, 2.0, 3.0]) and np.all(jo[inside & held] == [0.5, 0.25, 0.125])
        with open(path, "w") as f:
            f.write("Full-Wave\nDoubleSectorialCylinder\n0.75 0.75 0.5 z 0.5\ndeg 0 360\n0.1 0.3\n2.0 -1.0\n")
        jo, jor = advio.antenna_currents(model, flag, advio.read_jodefine(path))
    r = np.hypot(c[:, 0] - 0.75, c[:, 1] - 0.75)
    on = np.any(jor != 0, axis=1)
    assert on.any() and np.all(held[on])
    assert np.allclose(np.linalg.norm(jor[on], axis=1), 2.0) and np.allclose(np.linalg.norm(jo[on], axis=1), 1.0)
    radial = np.stack([c[on, 0] - 0.75, c[on, 1] - 0.75], axis=1)
    assert np.allclose(np.einsum("ij,ij->i", radial, jor[on, :2]), 0.0) and np.all(jor[on, 2] == 0.0)
    assert np.all((r[on] ** 2 >= 0.01 - 1e-15) & (r[on] ** 2 <= 0.09 + 1e-15))
