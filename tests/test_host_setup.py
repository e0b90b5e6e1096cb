"""The host setup's threaded builders (fw::global_rows, fw::envelope_layout
in adventure_fullwave_b200/csrc/fw_build.cpp) give exactly the arrays of
plain serial restatements (tests/host/host_setup_check.cpp, compiled here
with g++), on a jittered multi-subdomain model and on the same mesh cut into
a few large subdomains."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from adventure_fullwave_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "adventure_fullwave_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not present")
    out = str(tmp_path_factory.mktemp("host") / "host_setup_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, "-o", out,
                    os.path.join(HERE, "host", "host_setup_check.cpp"), os.path.join(CSRC, "fw_build.cpp")],
                   check=True)
    return out


def write_model(m, d, sub=None):
    m.vertex_crd.astype(np.float64).tofile(os.path.join(d, "crd.bin"))
    m.tets.astype(np.int32).tofile(os.path.join(d, "tv.bin"))
    m.tet_edges.astype(np.int32).tofile(os.path.join(d, "te.bin"))
    m.flag.astype(np.int32).tofile(os.path.join(d, "flag.bin"))
    m.pec_edge.astype(np.uint8).tofile(os.path.join(d, "pec.bin"))
    (m.sub_of_tet if sub is None else sub).astype(np.int32).tofile(os.path.join(d, "sub.bin"))


@pytest.mark.parametrize("cut", ["rcb", "few"])
def test_threaded_builders_match_serial(checker, tmp_path, cut):
    m = meshgen.make_model("hs", n=16, size=1.5, npml=2, layers=3, nleaves=None, leaf_cap=200, jitter=(0.3, 0.7),
                           seed=5)
    if cut == "rcb":
        write_model(m, str(tmp_path))
        nsub = m.nsub
    else:
        nsub = 3
        write_model(m, str(tmp_path), m.sub_of_tet % nsub)
    r = subprocess.run([checker, str(tmp_path), str(nsub)], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "identical" in r.stdout
