"""The correction-Jo pre-solve of an antenna (main/fullwave/main.c:92-98) on
the GPU through the C ABI (fwgpu_cojo_create / fwgpu_cojo_solve), against
the reference's own run (fixture tests/golden/ref_cojo.npz) and the oracle
(oracle/cojo.py): the shipped sample model and a synthetic cylinder antenna
(also with Dirichlet vertices), both passes, plus PEC vertices on interface
DOFs and a single subdomain checked against the oracle."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm
from oracle import cojo
from test_cojo import fixture, models, one_subdomain_model, ref_subs

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("key", ["sample", "cyl", "cylp"])
def test_gpu_matches_the_reference_and_the_oracle(key):
    z = fixture()
    m = models()[key]
    es = m.element_source
    flag = int(z[f"{key}_flag"][0])
    ref = ref_subs(z, key)
    op = cojo.partition(m, flag)
    with hddm.CorrectJoSolver(m, flag, hddm_eps=1e-10, hddm_max_loop=4000) as s:
        assert s.subdomain_ids().tolist() == [r[0] for r in ref]
        for k, r in enumerate(ref):
            mp = s.subdomain_maps(k)
            assert np.array_equal(mp["edge_gid"], r[1]) and np.array_equal(mp["ibc"], r[2])
        first = None
        for tag, cur, col in (("r", es.antenna_Jor[0], 5), ("i", es.antenna_Jo[0], 6)):
            phi, res = s.solve(cur)
            rh = z[f"{key}_hist_{tag}"]
            assert res.converged
            assert abs(res.iterations - rh.shape[0]) <= 1, (res.iterations, rh.shape[0])
            assert res.initial_norm == pytest.approx(float(z[f"{key}_norm0_{tag}"][0]), rel=6e-7, abs=1e-300)
            got = np.concatenate([phi[r[1]] for r in ref])
            want = np.concatenate([r[col] for r in ref])
            ophi, _, ohist, _ = cojo.hddm(m, op, cur, 1e-10, 4000)
            if np.any(want):
                err_ref, err_orc = rel(got, want), rel(phi, ophi)
                print(f"{key} pass {tag}: {res.iterations} iterations (reference {rh.shape[0]}), "
                      f"rel L2 vs reference {err_ref:.1e}, vs oracle {err_orc:.1e}")
                assert err_ref <= 1e-9
                assert err_orc <= 1e-10
                h = s.history()
                keep = ohist[: h.shape[0]] > 1e-12
                n = min(10, int(keep.sum()))
                assert np.allclose(h[: keep.shape[0]][keep][:n], ohist[: h.shape[0]][keep][:n], rtol=1e-6)
            else:
                assert res.iterations == 0 and not np.any(phi)
            if first is None:
                first = (cur, phi)
        # the factors are reused; the same current gives the same bits
        phi2, _ = s.solve(first[0])
        assert np.array_equal(phi2, first[1])


def test_gpu_pec_vertices_and_one_subdomain_vs_oracle():
    """Antenna vertices on a Dirichlet list (no reference model has any; the
    oracle is the check), and the whole antenna in one subdomain (no
    interface: the first DOF held at zero, the direct solve alone)."""
    m = models()["cyl"]
    es = m.element_source
    flag = int(es.antenna_flag[0])
    held = np.unique(m.tets[m.flag == flag])
    pec = np.zeros(m.n_vertices, np.uint8)
    pec[held[::5]] = 1
    op = cojo.partition(m, flag, pec.astype(bool))
    with hddm.CorrectJoSolver(m, flag, pec_vertex=pec) as s:
        for cur in (es.antenna_Jor[0], es.antenna_Jo[0]):
            phi, res = s.solve(cur)
            ophi, _, ohist, _ = cojo.hddm(m, op, cur, 1e-10, 4000)
            assert res.converged and abs(res.iterations - ohist.shape[0]) <= 1
            assert rel(phi, ophi) <= 1e-10
            # PEC vertices that are not interface DOFs stay at zero
            assert not np.any(phi[np.setdiff1d(held[::5], op.iface_gid)])
    m1 = one_subdomain_model()
    op1 = cojo.partition(m1, flag)
    with hddm.CorrectJoSolver(m1, flag) as s:
        phi, res = s.solve(es.antenna_Jor[0])
        ophi, _, _, _ = cojo.hddm(m1, op1, es.antenna_Jor[0])
        assert res.converged and res.iterations == 0
        assert rel(phi, ophi) <= 1e-11
