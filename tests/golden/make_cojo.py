"""Generates tests/golden/ref_cojo.npz: the reference's own correction-Jo
pre-solve (main/fullwave/main.c:92-98) run here by oracle/_ref/fw_ref_harness
in main() mode (FW_HARNESS_MAIN=1, FW_HARNESS_COJO_ONLY=1):

    make -f oracle/Makefile.ref
    python tests/golden/make_cojo.py

Three models:
  * ``sample``: the reference's shipped model directory (main/fullwave/MODEL,
    6 parts x 73 subdomains, one parallelepiped antenna);
  * ``cyl``: the synthetic ``antenna`` golden model written in the
    reference's layout with a double sectorial cylinder antenna (md) whose
    currents have real and imaginary parts (``cylinder_model`` rebuilds it
    through the package's own writer and reader);
  * ``cylp``: the same with vertex nodes in its Dirichlet lists
    (``pec_vertices``: the antenna's vertices on its lowest plane, some of
    them shared by subdomains), which the pre-solve holds at zero and keeps
    out of its interface.
For each, per subdomain holding antenna elements: its id, the model vertex of
each antenna DOF (enf order), the Dirichlet list, the interface entries
(nfid, ln_part) and the potentials Ihr, Ihi the reference leaves; the
interface size; and each pass's initial norm and residuals from the
reference's calc_log (7 digits).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import refdump  # noqa: E402
from adventure_fullwave_b200 import advio, meshgen  # noqa: E402

SAMPLE = os.path.join(os.environ.get("FW_REFERENCE", "/root/reference"), "main", "fullwave", "MODEL")
CYLINDER = "Full-Wave\nDoubleSectorialCylinder\n0.75 0.75 0.5 z 0.5\ndeg 30 270\n0.1 0.3\n2.0 -1.0\n"


def pec_vertices(model, flag):
    """Dirichlet vertices for the ``cylp`` model: the antenna's vertices on
    its lowest plane (z = 0.5), some of them shared by subdomains."""
    on_antenna = np.zeros(model.n_vertices, bool)
    on_antenna[np.unique(model.tets[model.flag == flag])] = True
    return on_antenna & (model.vertex_crd[:, 2] == 0.5)


def write_cylinder_model(mdir: str, with_pec_vertices: bool = False):
    """The ``antenna`` golden model with an md cylinder antenna, in the
    reference's model-directory layout; with_pec_vertices adds vertex nodes
    to its Dirichlet lists (pec_vertices)."""
    from helpers import golden

    z, params, model = golden("antenna")
    flag = int(model.element_source.antenna_flag[0])
    model.element_source = None
    if with_pec_vertices:
        model.pec_vertex = pec_vertices(model, flag)
    meshgen.write_hddm_model(model, mdir)
    os.remove(os.path.join(mdir, "source.txt"))
    with open(os.path.join(mdir, "mtrl.dat"), "a") as f:
        f.write(f"\nAntenna 1\n{flag} md cyl.dat\n")
    with open(os.path.join(mdir, "cyl.dat"), "w") as f:
        f.write(CYLINDER)


def cylinder_model(with_pec_vertices: bool = False):
    """The cylinder model as the package reads it (advio.load_model)."""
    with tempfile.TemporaryDirectory() as wd:
        mdir = os.path.join(wd, "MODEL")
        write_cylinder_model(mdir, with_pec_vertices)
        return advio.load_model(mdir)


def pack(prefix: str, cj, secs, vidx) -> dict:
    a = cj[0]
    subs = [k for k, d in enumerate(a["subs"]) if d["nf"]]
    out = {f"{prefix}_flag": np.array([a["flag"]]), f"{prefix}_tfree": np.array([a["total_free"]]),
           f"{prefix}_sub": np.array(subs, np.int32)}
    ptr = [0]
    for k in subs:
        ptr.append(ptr[-1] + a["subs"][k]["nf"])
    out[f"{prefix}_ptr"] = np.array(ptr, np.int64)
    out[f"{prefix}_vertex"] = np.concatenate([[vidx[int(g)] for g in a["subs"][k]["gid"]] for k in subs]).astype(np.int32)
    for key in ("ibc", "inbc_nfid", "inbc_ln"):
        arrs = [a["subs"][k][key] for k in subs]
        out[f"{prefix}_{key}_ptr"] = np.concatenate([[0], np.cumsum([x.shape[0] for x in arrs])]).astype(np.int64)
        out[f"{prefix}_{key}"] = np.concatenate(arrs).astype(np.int32)
    out[f"{prefix}_ihr"] = np.concatenate([a["subs"][k]["ihr"] for k in subs])
    out[f"{prefix}_ihi"] = np.concatenate([a["subs"][k]["ihi"] for k in subs])
    cs = [s for s in secs if s["title"].startswith("Correction Jo")]
    assert len(cs) == 2 and cs[0]["dof"] == a["total_free"]
    for tag, s in zip(("r", "i"), cs):
        out[f"{prefix}_norm0_{tag}"] = np.array([s["norm0"]])
        out[f"{prefix}_hist_{tag}"] = s["hist"]
    return out


def main():
    out = {}
    with tempfile.TemporaryDirectory() as wd:
        cj, secs = refdump.run_cojo(SAMPLE, wd)
    ld = advio.load_model(SAMPLE)
    vidx = {int(g): k for k, g in enumerate(np.asarray(ld.vertex_gnid).tolist())}
    out.update(pack("sample", cj, secs, vidx))
    with tempfile.TemporaryDirectory() as wd:
        mdir = os.path.join(wd, "MODEL")
        write_cylinder_model(mdir)
        ld = advio.load_model(mdir)
        cj, secs = refdump.run_cojo(mdir, wd)
    vidx = {int(g): k for k, g in enumerate(np.asarray(ld.vertex_gnid).tolist())}
    out.update(pack("cyl", cj, secs, vidx))
    with tempfile.TemporaryDirectory() as wd:
        mdir = os.path.join(wd, "MODEL")
        write_cylinder_model(mdir, with_pec_vertices=True)
        ld = advio.load_model(mdir)
        cj, secs = refdump.run_cojo(mdir, wd)
    vidx = {int(g): k for k, g in enumerate(np.asarray(ld.vertex_gnid).tolist())}
    out.update(pack("cylp", cj, secs, vidx))
    path = os.path.join(HERE, "ref_cojo.npz")
    np.savez_compressed(path, **out)
    print(path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
