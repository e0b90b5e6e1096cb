"""Runs the reference itself (oracle/_ref/fw_ref_harness, built from the
reference's sources) on a fresh synthetic model and checks the oracle
restatement against it bit for bit.  Skipped where the harness is not built."""
import os

import numpy as np
import pytest

import refdump
from adventure_fullwave_b200 import meshgen
from oracle import oracle

pytestmark = pytest.mark.skipif(not os.path.exists(refdump.HARNESS), reason="reference harness not built")


def test_fresh_model_bitwise():
    m = meshgen.make_model("x", n=6, size=1.5, npml=1, layers=3, nleaves=None, leaf_cap=150, jitter=(0.3, 0.7),
                           seed=11)
    meshgen.round_trip_material(m)
    ref = refdump.run_harness(m, 1e-8, 3000, dump=1)
    part = oracle.partition(m)
    assert part.tfree == ref["infree"]
    xe, per_sub, hist, norm0 = oracle.hddm(m, part, 1e-8, 3000)
    assert len(hist) == ref["json"]["iterations"]
    assert np.array_equal(xe, ref["x"])


def _run_main(model, write_antenna):
    """The model written in the reference's layout, its antenna files added by
    ``write_antenna(model_dir)``, run by the harness in main() mode; returns
    the loaded model, the reference's currents and solution and iteration
    count."""
    import json
    import subprocess
    import tempfile

    from adventure_fullwave_b200 import advio

    with tempfile.TemporaryDirectory() as wd:
        mdir = os.path.join(wd, "MODEL")
        meshgen.write_hddm_model(model, mdir)
        os.remove(os.path.join(mdir, "source.txt"))
        write_antenna(mdir)
        env = dict(os.environ, FW_HARNESS_MAIN="1", FW_HARNESS_OUT=os.path.join(mdir, "ref"))
        subprocess.run([refdump.HARNESS, "-memlimit", "60000", "-hddm-eps", "1e-10", "-hddm-max-loop", "4000",
                        "MODEL"], cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       timeout=600)
        loaded = advio.load_model(mdir)
        lines = open(os.path.join(mdir, "ref.jo")).read().split("\n")
        x_ref = refdump.read_sol(os.path.join(mdir, "ref.sol"), model.n_vertices, model.n_edges)
        iterations = int(json.load(open(os.path.join(mdir, "ref.json")))["iterations"])
    m2 = loaded.model
    jo = np.zeros((m2.n_vertices, 3))
    jor = np.zeros((m2.n_vertices, 3))
    vidx = {int(g): k for k, g in enumerate(loaded.vertex_gnid.tolist())}
    cnt = int(lines[1].split()[1])
    for ln in lines[2:2 + cnt]:
        t = ln.split()
        jo[vidx[int(t[0])]] = [float(u) for u in t[1:4]]
        jor[vidx[int(t[0])]] = [float(u) for u in t[4:7]]
    return m2, jo, jor, x_ref, iterations


def test_md_cylinder_antenna_as_main_runs_it():
    """An antenna defined by a double sectorial cylinder (md): the currents
    advio builds from the definition equal those main() leaves, and the
    oracle's solve equals the reference's bit for bit."""
    from helpers import golden

    z, params, model = golden("antenna")
    flag = int(model.element_source.antenna_flag[0])
    model.element_source = None

    def write(mdir):
        with open(os.path.join(mdir, "mtrl.dat"), "a") as f:
            f.write(f"\nAntenna 1\n{flag} md cyl.dat\n")
        with open(os.path.join(mdir, "cyl.dat"), "w") as f:
            f.write("Full-Wave\nDoubleSectorialCylinder\n0.75 0.75 0.5 z 0.5\ndeg 30 270\n0.1 0.3\n2.0 -1.0\n")

    m2, jo, jor, x_ref, iterations = _run_main(model, write)
    es = m2.element_source
    assert np.array_equal(es.antenna_Jo[0], jo) and np.array_equal(es.antenna_Jor[0], jor)
    assert np.any(jor)
    xe, _, hist, _ = oracle.hddm(m2, oracle.partition(m2, None), 1e-10, 4000)
    assert len(hist) == iterations
    assert np.array_equal(xe, x_ref)


def test_rf_antenna_model_directory_as_main_runs_it():
    """An antenna given by current data files (rf): advio.load_model builds
    the same vertex currents as main(), and the oracle's solve of the loaded
    model equals the reference's bit for bit."""
    from helpers import golden

    z, params, model = golden("antenna")
    flag = int(model.element_source.antenna_flag[0])
    model.element_source = None
    held = np.unique(model.tets[model.flag == flag])
    rng = np.random.default_rng(4)
    listed = held[rng.random(held.shape[0]) < 0.8]  # some antenna vertices left out
    extra = np.setdiff1d(np.arange(model.n_vertices), held)[:5]  # some off the antenna
    ids = np.concatenate([listed, extra])[::-1]  # not sorted

    def write(mdir):
        with open(os.path.join(mdir, "mtrl.dat"), "a") as f:
            f.write(f"\nAntenna 1\n{flag} rf jo.dat\n")
        for suffix, scale in (("r", 1.0), ("i", 0.5)):
            with open(os.path.join(mdir, "jo.dat" + suffix), "w") as f:
                f.write(f"{ids.shape[0]}\n")
                for v in ids:
                    c = model.vertex_crd[v]
                    f.write(f"{int(v)} {scale * (1 + c[0]):.17e} {scale * (0.3 - c[1]):.17e} {scale * c[2] * 2:.17e}\n")

    m2, jo, jor, x_ref, iterations = _run_main(model, write)
    es = m2.element_source
    assert es is not None and list(es.antenna_flag) == [flag]
    assert np.array_equal(es.antenna_Jo[0], jo) and np.array_equal(es.antenna_Jor[0], jor)
    assert np.any(jo) and np.any(jor)
    xe, _, hist, _ = oracle.hddm(m2, oracle.partition(m2, None), 1e-10, 4000)
    assert len(hist) == iterations
    assert np.array_equal(xe, x_ref)
