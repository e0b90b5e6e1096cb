"""Generates tests/golden/ref_sample.npz from the reference's shipped sample
model (main/fullwave/MODEL: 6 parts x 73 subdomains, one antenna), run here
by the reference itself:

    make -f oracle/Makefile.ref
    python tests/golden/make_sample.py

The model directory is copied to a scratch directory and run by
oracle/_ref/fw_ref_harness with FW_HARNESS_MAIN=1, which is the reference's
main() flow: hddm_Init, the correction-Jo pre-solve of the antenna, then the
full-wave HDDM solve to hddm_eps = 1e-6.  The fixture holds the mesh as
adventure_fullwave_b200.advio reads it (with every subdomain's local node
order), the antenna currents the pre-solve left (its output, which this
library takes as input), the reference's initial norm and iteration count,
a strided sample and norms of its converged edge solution, and the
reference's integer maps (nop, Dirichlet list, interface DOFs, edge of each
local DOF) and skyline profiles (idx1, idx2, nlen) of all 438 subdomains,
with the LDL^T factors of two of them.
"""
from __future__ import annotations

import os
import shutil
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from adventure_fullwave_b200 import advio  # noqa: E402

sys.path.insert(0, HERE)
import refdump  # noqa: E402

FACTOR_SUBS = (0, 219)

SAMPLE = os.path.join(os.environ.get("FW_REFERENCE", "/root/reference"), "main", "fullwave", "MODEL")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "fw_ref_harness")
EPS = 1e-6
STRIDE = 53


def read_jo(path, vidx, nv):
    lines = open(path).read().split("\n")
    nant = int(lines[0])
    i = 1
    flags, jo, jor = [], [], []
    for _ in range(nant):
        f, cnt = map(int, lines[i].split())
        i += 1
        a = np.zeros((nv, 3))
        b = np.zeros((nv, 3))
        for _ in range(cnt):
            t = lines[i].split()
            i += 1
            v = vidx[int(t[0])]
            a[v] = [float(u) for u in t[1:4]]
            b[v] = [float(u) for u in t[4:7]]
        flags.append(f)
        jo.append(a)
        jor.append(b)
    return np.array(flags, np.int32), np.array(jo), np.array(jor)


def read_solution(path, eidx, ne):
    buf = open(path, "rb").read()
    nsub = struct.unpack_from("<i", buf, 0)[0]
    o = 4
    x = np.full(ne, np.nan + 0j)
    for _ in range(nsub):
        n = struct.unpack_from("<i", buf, o)[0]
        o += 4
        g = np.frombuffer(buf, "<i4", n, o)
        o += 4 * n
        v = np.frombuffer(buf, "<c16", n, o)
        o += 16 * n
        x[[eidx[int(q)] for q in g.tolist()]] = v
    return x


def read_norm0(log):
    """Initial norm of the full-wave solve: the last '# Norm' line of the log
    (the correction-Jo solves come first)."""
    norm = None
    for line in open(log):
        t = line.split()
        if len(t) >= 5 and t[2] == "#" and t[3] == "Norm":
            norm = float(t[4])
    return norm


def main():
    loaded = advio.load_model(SAMPLE)
    m = loaded.model
    wd = tempfile.mkdtemp(prefix="fwsample_")
    shutil.copytree(SAMPLE, os.path.join(wd, "MODEL"), ignore=shutil.ignore_patterns("result", "calc_log"))
    for dp, dn, fn in os.walk(wd):
        for n in dn + fn:
            os.chmod(os.path.join(dp, n), 0o755)
    env = dict(os.environ, FW_HARNESS_MAIN="1", FW_HARNESS_OUT=os.path.join(wd, "ref"), FW_HARNESS_DUMP="2")
    subprocess.run([HARNESS, "-memlimit", "60000", "-hddm-eps", repr(EPS), "-hddm-max-loop", "40000", "MODEL"],
                   cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    vidx = {int(g): k for k, g in enumerate(loaded.vertex_gnid.tolist())}
    eidx = {int(g): k for k, g in enumerate(loaded.edge_gnid.tolist())}
    flags, jo, jor = read_jo(os.path.join(wd, "ref.jo"), vidx, m.n_vertices)
    x = read_solution(os.path.join(wd, "ref.sol"), eidx, m.n_edges)
    log = os.path.join(wd, "MODEL", "calc_log", "log_g_HDDM_Full_Wave")
    hist = [ln.split() for ln in open(log) if ln.strip() and not ln.startswith("#")]
    iterations = int(hist[-1][0])
    ant = np.nonzero(np.any(jo[0] != 0, axis=1) | np.any(jor[0] != 0, axis=1))[0].astype(np.int32)
    # the reference's maps and profiles, every part's subdomains in order
    _, ints = refdump.read_ints(os.path.join(wd, "ref.ints"), 0)
    fac = refdump.read_fac(os.path.join(wd, "ref.fac"))
    assert len(ints) == len(fac) == m.nsub
    maps = {}
    for key in ("nop", "ibc", "inbc_nfid"):
        arrs = [np.asarray(d[key]).ravel() for d in ints]
        maps[f"ref_{key}"] = np.concatenate(arrs).astype(np.int32)
        maps[f"ref_{key}_ptr"] = np.concatenate([[0], np.cumsum([a.shape[0] for a in arrs])]).astype(np.int32)
    maps["ref_edge"] = np.concatenate([[eidx[int(g)] for g in d["edge_gid"].tolist()] for d in ints]).astype(np.int32)
    maps["ref_idx1"] = np.concatenate([f["idx1"] for f in fac]).astype(np.int32)
    maps["ref_idx2"] = np.concatenate([f["idx2"] for f in fac]).astype(np.int32)
    maps["ref_nlen"] = np.array([f["nlen"] for f in fac], np.int32)
    maps["ref_dof_ptr"] = np.concatenate([[0], np.cumsum([f["idx1"].shape[0] for f in fac])]).astype(np.int32)
    maps["factor_subs"] = np.array(FACTOR_SUBS, np.int32)
    for s in FACTOR_SUBS:
        maps[f"ref_factor_{s}"] = fac[s]["mat"]
    so = m.sub_order
    path = os.path.join(HERE, "ref_sample.npz")
    np.savez_compressed(
        path, vertex_crd=m.vertex_crd, tets=m.tets, tet_edges=m.tet_edges, flag=m.flag.astype(np.int8),
        sub_of_tet=m.sub_of_tet.astype(np.int16), nsub=np.array([m.nsub]), mat_flag=m.mat_flag, mat_eps=m.mat_eps,
        mat_sigma=m.mat_sigma, omega=np.array([m.omega]), antenna_flag=flags, antenna_vertices=ant,
        antenna_Jo=jo[0][ant], antenna_Jor=jor[0][ant], eps=np.array([EPS]), iterations=np.array([iterations]),
        norm0=np.array([read_norm0(log)]), x_sample_stride=np.array([STRIDE]), x_sample=x[::STRIDE],
        x_sum=np.array([x.sum()]), x_norm=np.array([np.linalg.norm(x)]), sub_vertex_ptr=so[0],
        sub_vertex_order=so[1], sub_edge_ptr=so[2], sub_edge_order=so[3], **maps)
    shutil.rmtree(wd)
    print(path, os.path.getsize(path), "iterations", iterations)


if __name__ == "__main__":
    main()
