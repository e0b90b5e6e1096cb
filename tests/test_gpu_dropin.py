"""The drop-in tables (adventure_fullwave_b200/dropin/set_hddm_func_gpu.c)
compiled against the reference and run by the reference's own drivers:
  * main()'s flow with hddm_solver_CS (lib/hddm/hddm_solver.h:25-183)
    walking set_hddm_func_fullwave_gpu instead of set_hddm_func_fullwave, on
    C1 to hddm_eps 1e-10: the solution equals the plain reference run's to
    1e-8 relative L2 over every edge, the same bar as the library's own C1
    test;
  * main()'s correction-Jo pre-solve with hddm_solver_RS walking
    set_hddm_func_correct_Jor_gpu / _Joi_gpu, on a model with a cylinder
    antenna: every subdomain's potentials equal the reference's own
    pre-solve (tests/golden/ref_cojo.npz) to 1e-9 relative L2."""
import os

import numpy as np
import pytest

import refdump
from helpers import golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(refdump.HARNESS_GPU), reason="oracle/_ref/fw_ref_gpu is not built")
def test_reference_driver_through_the_gpu_table():
    z, params, model = golden("c1")
    out = refdump.run_harness(model, params["eps"], params["max_loop"], dump=0, binary=refdump.HARNESS_GPU,
                              timeout=600)
    n_ref = int(z["iterations"][0])
    n = int(out["json"]["iterations"])
    err = rel_l2(out["x"], z["x"])
    print(f"C1 through the GPU table: {n} iterations (reference {n_ref}), rel L2 vs the reference run {err:.2e}")
    assert np.isfinite(out["x"]).all()
    assert abs(n - n_ref) <= 0.05 * n_ref
    assert err <= 1e-8
    # the reference's own log of the GPU run: the DOF count line of hddm_solver_CS
    assert out["norm0"] is None or out["norm0"] > 0


@pytest.mark.skipif(not os.path.exists(refdump.HARNESS_GPU), reason="oracle/_ref/fw_ref_gpu is not built")
def test_reference_pre_solve_through_the_gpu_tables():
    import tempfile

    import make_cojo
    from adventure_fullwave_b200 import advio

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cojo.npz"))
    with tempfile.TemporaryDirectory() as wd:
        mdir = os.path.join(wd, "MODEL")
        make_cojo.write_cylinder_model(mdir)
        ld = advio.load_model(mdir)
        cj, secs = refdump.run_cojo(mdir, wd, binary=refdump.HARNESS_GPU)
    vidx = {int(g): k for k, g in enumerate(np.asarray(ld.vertex_gnid).tolist())}
    subs = [k for k, d in enumerate(cj[0]["subs"]) if d["nf"]]
    assert subs == z["cyl_sub"].tolist()
    verts = np.concatenate([[vidx[int(g)] for g in cj[0]["subs"][k]["gid"]] for k in subs])
    assert np.array_equal(verts, z["cyl_vertex"])
    for key in ("ihr", "ihi"):
        got = np.concatenate([cj[0]["subs"][k][key] for k in subs])
        err = rel_l2(got, z[f"cyl_{key}"])
        print(f"pre-solve through the GPU tables, {key}: rel L2 vs the reference {err:.1e}")
        assert err <= 1e-9
    # the reference's driver logged both passes with the antenna's interface size
    cs = [s for s in secs if s["title"].startswith("Correction Jo")]
    assert len(cs) == 2 and all(s["dof"] == int(z["cyl_tfree"][0]) for s in cs)
