"""Integer setup (make_PartMesh_FW for one part): the product's host builder,
the oracle restatement and the reference itself agree bit for bit."""
import numpy as np
import pytest

from adventure_fullwave_b200 import hddm, meshgen
from helpers import golden
from oracle import oracle


def _same_maps(a, o):
    return (np.array_equal(a["nop"], o.nop) and np.array_equal(a["ibc"], o.ibc)
            and np.array_equal(a["inbc_nfid"], o.inbc_nfid) and np.array_equal(a["inbc_ln_part"], o.inbc_ln)
            and np.array_equal(a["edge_gid"], o.edge_gid))


@pytest.mark.parametrize("name", ["tiny", "layered"])
def test_oracle_partition_matches_reference(name):
    z, params, model = golden(name)
    part = oracle.partition(model)
    assert part.tfree == int(z["total_free"][0])
    for s, sub in enumerate(part.subs):
        assert np.array_equal(sub.nop, z[f"s{s}_nop"])
        assert np.array_equal(sub.ibc, z[f"s{s}_ibc"])
        assert np.array_equal(sub.inbc_nfid, z[f"s{s}_inbc_nfid"])
        assert np.array_equal(sub.inbc_ln, z[f"s{s}_inbc_ln"])
        assert np.array_equal(sub.edge_gid, z[f"s{s}_edge_gid"])


@pytest.mark.parametrize("kw", [
    dict(name="c1"),
    dict(name="c2"),
    dict(name="x", n=8, size=1.5, npml=2, layers=2, nleaves=None, leaf_cap=120, jitter=(0.3, 0.7), seed=1),
    dict(name="x", n=6, size=1.0, npml=1, layers=None, nleaves=1),
    dict(name="x", n=10, size=1.5, npml=2, layers=3, nleaves=None, leaf_cap=50, jitter=(0.3, 0.7), seed=9),
])
def test_product_builder_matches_oracle(kw):
    m = meshgen.make_model(**kw)
    prod = hddm.Partition(m)
    orc = oracle.partition(m)
    assert prod.n_subdomains == m.nsub
    assert prod.total_free == orc.tfree
    for s in range(m.nsub):
        assert _same_maps(prod.maps(s), orc.subs[s]), s


def test_builder_rejects_bad_input():
    from adventure_fullwave_b200 import _lib

    m = meshgen.make_model("x", n=3, npml=1, nleaves=2)
    m.sub_of_tet = m.sub_of_tet.copy()
    m.sub_of_tet[0] = 99
    with pytest.raises(_lib.FwgpuError):
        hddm.Partition(m)
    m2 = meshgen.make_model("x", n=3, npml=1, nleaves=2)
    m2.nsub = 3  # an empty subdomain
    with pytest.raises(_lib.FwgpuError):
        hddm.Partition(m2)
