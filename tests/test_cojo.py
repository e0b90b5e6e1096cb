"""The correction-Jo pre-solve of an antenna (main/fullwave/main.c:92-98),
on the CPU: the library's integer setup (fwgpu_cojo_partition_build, no GPU)
and the oracle (oracle/cojo.py) against the reference's own run of the
pre-solve (fixture tests/golden/ref_cojo.npz, made by
tests/golden/make_cojo.py) on the shipped sample model and on a synthetic
single-part model with a cylinder antenna, also with vertex nodes in its
Dirichlet lists (which advio reads into model.pec_vertex and the pre-solve
holds at zero)."""
import os
import sys

import numpy as np
import pytest

from adventure_fullwave_b200 import _lib, hddm
from oracle import cojo

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_cojo  # noqa: E402
import refdump  # noqa: E402

FIX = os.path.join(HERE, "golden", "ref_cojo.npz")


def fixture():
    return np.load(FIX)


def models():
    import bench

    m, _ = bench.sample_model()
    return {"sample": m, "cyl": make_cojo.cylinder_model().model,
            "cylp": make_cojo.cylinder_model(with_pec_vertices=True).model}


def ref_subs(z, key):
    """Per subdomain of the reference's antenna problem: (id, vertices, ibc,
    inbc_nfid, inbc_ln, Ihr, Ihi)."""
    out = []
    p = z[f"{key}_ptr"]
    for k, s in enumerate(z[f"{key}_sub"].tolist()):
        row = [s, z[f"{key}_vertex"][p[k]:p[k + 1]]]
        for name in ("ibc", "inbc_nfid", "inbc_ln"):
            q = z[f"{key}_{name}_ptr"]
            row.append(z[f"{key}_{name}"][q[k]:q[k + 1]])
        row += [z[f"{key}_ihr"][p[k]:p[k + 1]], z[f"{key}_ihi"][p[k]:p[k + 1]]]
        out.append(row)
    return out


@pytest.mark.parametrize("key", ["sample", "cyl", "cylp"])
def test_integer_setup_matches_the_reference(key):
    """Subdomains, antenna DOFs in enf order, Dirichlet lists and interface
    DOFs bit-exact; interface numbers too on the single-part model (the
    multi-part sample numbers its interface per part in the reference, in one
    numbering here), and one global vertex per interface number."""
    z = fixture()
    m = models()[key]
    flag = int(z[f"{key}_flag"][0])
    part = hddm.CorrectJoPartition(m, flag)
    ref = ref_subs(z, key)
    assert part.total_free == int(z[f"{key}_tfree"][0])
    assert part.subdomain_ids.tolist() == [r[0] for r in ref]
    gid_of_ln = {}
    for k, (s, verts, ibc, nfid, ln, _, _) in enumerate(ref):
        mp = part.maps(k)
        assert np.array_equal(mp["edge_gid"], verts), s
        assert np.array_equal(mp["ibc"], ibc), s
        assert np.array_equal(mp["inbc_nfid"], nfid), s
        if key != "sample":
            assert np.array_equal(mp["inbc_ln_part"], ln), s
        for n, g in zip(mp["inbc_ln_part"].tolist(), mp["edge_gid"][mp["inbc_nfid"]].tolist()):
            assert gid_of_ln.setdefault(n, g) == g
    # the oracle's restatement gives the same maps
    op = cojo.partition(m, flag)
    assert op.tfree == part.total_free and [s.sub for s in op.subs] == [r[0] for r in ref]
    for sb, r in zip(op.subs, ref):
        assert np.array_equal(sb.gid, r[1]) and np.array_equal(sb.ibc, r[2]) and np.array_equal(sb.inbc_nfid, r[3])


@pytest.mark.parametrize("key", ["sample", "cyl", "cylp"])
def test_oracle_matches_the_reference(key):
    """Both passes (currents Jor, then Jo): the same iteration count, the
    residual history to the 7 printed digits (the first 15 above 1e-12), and
    the potentials of every subdomain to 1e-9 relative L2 (the reference's
    subdomain CG stops at a relative residual of 1e-12, the oracle solves
    directly)."""
    z = fixture()
    m = models()[key]
    es = m.element_source
    flag = int(z[f"{key}_flag"][0])
    op = cojo.partition(m, flag)
    ref = ref_subs(z, key)
    for tag, cur, col in (("r", es.antenna_Jor[0], 5), ("i", es.antenna_Jo[0], 6)):
        phi, per_sub, hist, norm0 = cojo.hddm(m, op, cur, 1e-10, 4000)
        rh = z[f"{key}_hist_{tag}"]
        assert hist.shape == rh.shape
        assert norm0 == pytest.approx(float(z[f"{key}_norm0_{tag}"][0]), rel=6e-7, abs=1e-300)
        # residuals above rounding level (the last step of a converged
        # Krylov run can land at 1e-16 in either)
        keep = rh > 1e-12
        assert np.allclose(hist[keep][:15], rh[keep][:15], rtol=1e-6, atol=0)
        got = np.concatenate(per_sub)
        want = np.concatenate([r[col] for r in ref])
        if np.any(want):
            assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-9
        else:
            assert not np.any(got)
        # the potential per vertex is each subdomain's value there
        for sb, x in zip(op.subs, per_sub):
            assert np.allclose(phi[sb.gid], x, rtol=0, atol=1e-12 * max(1.0, np.abs(want).max()))


def one_subdomain_model():
    """The cylinder model as one subdomain: no interface, the first antenna
    DOF held at zero."""
    m = models()["cyl"]
    m.sub_of_tet = np.zeros(m.n_tets, np.int32)
    m.nsub = 1
    m.sub_order = None
    return m


def test_pinned_dof_without_interface():
    m = one_subdomain_model()
    flag = int(m.element_source.antenna_flag[0])
    part = hddm.CorrectJoPartition(m, flag)
    assert part.n_subdomains == 1 and part.total_free == 0
    mp = part.maps(0)
    assert mp["ibc"].tolist() == [0] and mp["inbc_nfid"].shape[0] == 0
    op = cojo.partition(m, flag)
    assert op.subs[0].pinned and op.subs[0].ibc.tolist() == [0]
    phi, per_sub, hist, _ = cojo.hddm(m, op, m.element_source.antenna_Jor[0])
    assert hist.shape[0] == 0 and per_sub[0][0] == 0.0 and np.any(per_sub[0])


def test_dirichlet_vertices_are_read_and_held():
    """advio reads the vertex nodes of the Dirichlet lists.  In the
    reference's pre-solve they lead each subdomain's Dirichlet list and stay
    out of the interface, shared ones too (make_PartMesh.c:393-421)."""
    ms = models()
    assert ms["cyl"].pec_vertex is None
    pv = ms["cylp"].pec_vertex
    assert pv is not None and pv.any()
    z = fixture()
    ref = ref_subs(z, "cylp")
    seen = np.zeros_like(pv)
    shared = 0
    for r in ref:
        k = int(pv[r[1]].sum())
        assert np.array_equal(r[2][:k], np.nonzero(pv[r[1]])[0])
        assert not pv[r[1][r[3]]].any()  # no interface DOF on a Dirichlet list
        shared += int(seen[r[1]][pv[r[1]]].sum())
        seen[r[1][pv[r[1]]]] = True
    assert np.array_equal(seen, pv) and shared > 0
    assert int(z["cylp_tfree"][0]) < int(z["cyl_tfree"][0])


def test_no_antenna_element_is_an_error():
    m = models()["cyl"]
    with pytest.raises(_lib.FwgpuError):
        hddm.CorrectJoPartition(m, 12345)


@pytest.mark.skipif(not os.path.exists(refdump.HARNESS), reason="reference harness not built")
def test_fixture_is_the_reference_run():
    """The cylinder model's fixture entries are what the reference gives when
    run again here."""
    import tempfile

    z = fixture()
    with tempfile.TemporaryDirectory() as wd:
        mdir = os.path.join(wd, "MODEL")
        make_cojo.write_cylinder_model(mdir)
        ld = make_cojo.advio.load_model(mdir)
        cj, secs = refdump.run_cojo(mdir, wd)
    vidx = {int(g): k for k, g in enumerate(np.asarray(ld.vertex_gnid).tolist())}
    got = make_cojo.pack("cyl", cj, secs, vidx)
    for k, v in got.items():
        assert np.array_equal(v, z[k]), k


def test_entry_points_refuse_bad_arguments_before_any_device_work():
    """The C ABI's argument checks of the pre-solve's entry points, which run
    before any CUDA call: FP32 factors and shard ranges are refused, null
    handles and currents too, and a context that is not a pre-solve's is
    turned away by the pre-solve's calls."""
    import ctypes

    lib = _lib.load()
    m = models()["cyl"]
    mesh, keep = hddm._mesh_struct(m)
    flag = int(m.element_source.antenna_flag[0])
    out = ctypes.c_void_p()
    fp32 = _lib.FwOptions(1e-10, 4000, _lib.PREC_FP32_IR, 1, 0.0, 16, 0, 0, 0, 0.0, 0, 0, 0, 0)
    assert lib.fwgpu_cojo_create(ctypes.byref(mesh), flag, None, ctypes.byref(fp32), ctypes.byref(out)) == _lib.ERR_ARG
    assert not out.value
    shard = _lib.FwOptions(1e-10, 4000, _lib.PREC_FP64, 1, 0.0, 16, 0, 0, 0, 0.0, 0, 2, 0, 0)
    assert lib.fwgpu_cojo_create(ctypes.byref(mesh), flag, None, ctypes.byref(shard), ctypes.byref(out)) == _lib.ERR_ARG
    cur = np.zeros(3 * m.n_vertices)
    p = cur.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.fwgpu_cojo_solve(None, p, None, None) == _lib.ERR_ARG
    assert lib.fwgpu_cojo_set_current(None, p) == _lib.ERR_ARG
    n = ctypes.c_int32()
    assert lib.fwgpu_cojo_subdomains(None, ctypes.byref(n), None) == _lib.ERR_ARG
    with pytest.raises(ValueError):
        hddm.CorrectJoPartition(m, flag, pec_vertex=np.zeros(3, bool))


@pytest.mark.skipif(__import__("conftest").has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    with pytest.raises(_lib.FwgpuError) as e:
        hddm.CorrectJoSolver(models()["cyl"], 4)
    assert e.value.code == _lib.ERR_CUDA
