"""The oracle restatement (oracle/fw_oracle.c) against the reference's own
outputs (golden fixtures made by tests/golden/make_golden.py from the
reference built from its sources): bit for bit."""
import numpy as np
import pytest

from helpers import golden
from oracle import oracle


@pytest.mark.parametrize("name", ["tiny", "layered"])
def test_assembly_and_factor_bitwise(name):
    z, params, model = golden(name)
    part = oracle.partition(model)
    for s, sub in enumerate(part.subs):
        rp, col, val, b = oracle.assemble_sub(model, sub)
        assert np.array_equal(rp, z[f"s{s}_aij_row_ptr"])
        assert np.array_equal(col, z[f"s{s}_aij_col"])
        assert np.array_equal(val, z[f"s{s}_aij_val"])
        idx1, idx2, nlen, mat = oracle.factor_sub(model, sub)
        assert np.array_equal(idx1, z[f"s{s}_idx1"]) and np.array_equal(idx2, z[f"s{s}_idx2"])
        assert nlen == z[f"s{s}_fac"].shape[0]
        assert np.array_equal(mat, z[f"s{s}_fac"])


@pytest.mark.parametrize("name", ["tiny", "layered"])
def test_hddm_bitwise(name):
    z, params, model = golden(name)
    part = oracle.partition(model)
    xe, per_sub, hist, norm0 = oracle.hddm(model, part, params["eps"], params["max_loop"])
    assert len(hist) == int(z["iterations"][0])
    assert norm0 == pytest.approx(float(z["norm0"][0]), rel=1e-6)
    # the reference prints the history with 7 digits
    assert np.allclose(hist, z["hist"], rtol=5e-7, atol=0)
    assert np.array_equal(xe, z["x"])


def test_c1_history_and_solution():
    """C1 to hddm_eps 1e-10: all 693 residuals (at full precision, as the
    harness records them) and every edge value equal the reference's."""
    z, params, model = golden("c1")
    part = oracle.partition(model)
    xe, per_sub, hist, norm0 = oracle.hddm(model, part, params["eps"], params["max_loop"])
    assert len(hist) == int(z["iterations"][0]) == 693
    assert norm0 == float(z["norm0_full"][0])
    assert np.array_equal(hist, z["hist_full"])
    assert np.array_equal(xe, z["x"])


@pytest.mark.parametrize("name", ["tiny", "layered", "gap", "antenna"])
@pytest.mark.parametrize("tag", ["post", "post_drop"])
def test_post_em_E_bitwise(name, tag):
    """HDDM_post_em_E on the reference's converged solution; ``post_drop``
    leaves the first Permittivity and Conductor flags out, which exercises the
    nu = 0 and sigma = 0 branches."""
    z, params, model = golden(name)
    B, E, Je = oracle.post_em_E(model, z["x"], drop_first=(tag == "post_drop"))
    assert np.array_equal(B, z[f"{tag}_B"])
    assert np.array_equal(E, z[f"{tag}_E"])
    assert np.array_equal(Je, z[f"{tag}_Je"])
    if tag == "post_drop":
        dropped = model.flag == model.mat_flag[0]
        assert not np.any(B[dropped]) and not np.any(Je[dropped])
        assert dropped.any() or name == "gap"  # the gap block takes every element of flag 0


@pytest.mark.parametrize("name", ["gap", "antenna"])
def test_element_source_bitwise(name):
    """Delta-gap voltages and antenna currents through the reference's own
    element routine (tet_MakeElement_EM_E): the assembled right-hand sides,
    the factors and the converged solution, bit for bit."""
    z, params, model = golden(name)
    part = oracle.partition(model, None)
    nonzero = 0
    for s, sub in enumerate(part.subs):
        rp, col, val, b = oracle.assemble_sub(model, sub)
        assert np.array_equal(val, z[f"s{s}_aij_val"])
        assert np.array_equal(b, z[f"s{s}_aij_b"])
        nonzero += np.count_nonzero(b)
        idx1, idx2, nlen, mat = oracle.factor_sub(model, sub)
        assert np.array_equal(mat, z[f"s{s}_fac"])
    assert nonzero > 0
    xe, per_sub, hist, norm0 = oracle.hddm(model, part, params["eps"], params["max_loop"])
    assert len(hist) == int(z["iterations"][0])
    assert np.array_equal(xe, z["x"])


def test_element_rhs_branches():
    """The element right-hand side restatement on single elements: zero
    outside the sources, the later gap box wins, antenna terms are linear in
    the currents."""
    import make_golden

    z, params, model = golden("gap")
    be = oracle.element_rhs(model)
    es = model.element_source
    inside = np.zeros(model.n_vertices, bool)
    for box in es.gap_box:
        c = model.vertex_crd
        inside |= np.all((c >= box[0::2]) & (c <= box[1::2]), axis=1)
    touched = inside[model.tets].any(axis=1)
    assert not np.any(be[~touched])
    _, sig = oracle.material_per_element(model)
    assert np.any(be[touched & (sig > 0)])
    assert not np.any(be[touched & (sig == 0)])
    za, pa, ma = golden("antenna")
    b1 = oracle.element_rhs(ma)
    ma.element_source.antenna_Jo = 2.0 * ma.element_source.antenna_Jo
    ma.element_source.antenna_Jor = 2.0 * ma.element_source.antenna_Jor
    b2 = oracle.element_rhs(ma)
    assert np.array_equal(b2, 2.0 * b1)
    assert not np.any(b1[ma.flag != ma.element_source.antenna_flag[0]])
