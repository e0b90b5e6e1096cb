"""Readers for the dump files the reference harness (oracle/ref_harness.c)
writes, and a runner for it.  Used by make_golden.py (run where the
reference is built) and by the tests that re-run the reference harness when
its binary is present."""
from __future__ import annotations

import json
import os
import struct
import subprocess
import tempfile

import numpy as np

REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
HARNESS = os.path.join(REPO, "oracle", "_ref", "fw_ref_harness")
# the same driver with the reference's table replaced by the GPU drop-in
HARNESS_GPU = os.path.join(REPO, "oracle", "_ref", "fw_ref_gpu")


def read_ints(path: str, nv: int):
    a = np.frombuffer(open(path, "rb").read(), dtype="<i4")
    nsub, infree = int(a[0]), int(a[1])
    o = 4
    subs = []
    for _ in range(nsub):
        nmp, nap, nel = (int(v) for v in a[o:o + 3])
        o += 3
        nop = a[o:o + 10 * nel].reshape(nel, 10).copy()
        o += 10 * nel
        nbc = int(a[o])
        o += 1
        ibc = a[o:o + nbc].copy()
        o += nbc
        nin = int(a[o])
        o += 1
        inb = a[o:o + 2 * nin].reshape(nin, 2).copy()
        o += 2 * nin
        gid = a[o:o + nmp] - nv
        o += nmp
        subs.append(dict(nop=nop, ibc=ibc, inbc_nfid=inb[:, 0].copy(), inbc_ln=inb[:, 1].copy(), edge_gid=gid))
    return infree, subs


def read_aij(path: str):
    b = open(path, "rb").read()
    o = 0
    out = []
    while o < len(b):
        nf = struct.unpack_from("<i", b, o)[0]
        o += 4
        rp = [0]
        cols, vals = [], []
        for _ in range(nf):
            n = struct.unpack_from("<i", b, o)[0]
            o += 4
            cols.append(np.frombuffer(b, "<i4", n, o))
            o += 4 * n
            vals.append(np.frombuffer(b, "<c16", n, o))
            o += 16 * n
            rp.append(rp[-1] + n)
        bb = np.frombuffer(b, "<c16", nf, o).copy()
        o += 16 * nf
        out.append(dict(row_ptr=np.array(rp, np.int32), col=np.concatenate(cols).astype(np.int32),
                        val=np.concatenate(vals), b=bb))
    return out


def read_fac(path: str):
    b = open(path, "rb").read()
    o = 0
    out = []
    while o < len(b):
        nd, nl = struct.unpack_from("<ii", b, o)
        o += 8
        i1 = np.frombuffer(b, "<i4", nd, o).copy()
        o += 4 * nd
        i2 = np.frombuffer(b, "<i4", nd, o).copy()
        o += 4 * nd
        mat = np.frombuffer(b, "<c16", nl, o).copy()
        o += 16 * nl
        out.append(dict(idx1=i1, idx2=i2, nlen=nl, mat=mat))
    return out


def read_sol(path: str, nv: int, n_edges: int):
    b = open(path, "rb").read()
    nsub = struct.unpack_from("<i", b, 0)[0]
    o = 4
    xe = np.zeros(n_edges, np.complex128)
    seen = np.zeros(n_edges, bool)
    for _ in range(nsub):
        n = struct.unpack_from("<i", b, o)[0]
        o += 4
        g = np.frombuffer(b, "<i4", n, o) - nv
        o += 4 * n
        x = np.frombuffer(b, "<c16", n, o)
        o += 16 * n
        new = ~seen[g]
        xe[g[new]] = x[new]
        seen[g] = True
    return xe


def read_post(path: str, n_tets: int):
    """Element results B, E, Je of the reference's post step as the harness
    dumps them per subdomain, put in global element order: three (n_tets, 3)
    complex arrays."""
    b = open(path, "rb").read()
    nsub = struct.unpack_from("<i", b, 0)[0]
    o = 4
    out = [np.zeros((n_tets, 3), np.complex128) for _ in range(3)]
    seen = np.zeros(n_tets, bool)
    for _ in range(nsub):
        n = struct.unpack_from("<i", b, o)[0]
        o += 4
        g = np.frombuffer(b, "<i4", n, o)
        o += 4 * n
        for a in out:
            a[g] = np.frombuffer(b, "<c16", 3 * n, o).reshape(n, 3)
            o += 48 * n
        seen[g] = True
    assert o == len(b) and seen.all()
    return tuple(out)


def read_log(path: str):
    """Residual history of the full-wave solve from the reference's calc_log
    (hddm_solver_s.h:203-207, :319-323): returns (norm0, resi per iteration)."""
    norm0 = None
    hist = []
    for line in open(path):
        t = line.split()
        if len(t) >= 4 and t[0] == "0" and t[2] == "#" and t[3] == "Norm":
            norm0 = float(t[4])
        elif len(t) == 2 and not line.startswith("#"):
            hist.append(float(t[1]))
    return norm0, np.array(hist)


def run_harness(model, hddm_eps: float, hddm_max_loop: int, dump: int = 2, workdir: str = None, timeout=3600,
                binary: str = HARNESS):
    """Write ``model`` in the reference's part-file layout and run the
    reference on it.  Returns a dict of the parsed outputs."""
    from adventure_fullwave_b200 import meshgen

    own = workdir is None
    wd = tempfile.mkdtemp(prefix="fwref_") if own else workdir
    mdir = os.path.join(wd, "MODEL")
    meshgen.write_hddm_model(model, mdir)
    env = dict(os.environ, FW_HARNESS_DUMP=str(dump), FW_HARNESS_OUT=os.path.join(mdir, "ref"))
    cmd = [binary, "-memlimit", "60000", "-hddm-eps", repr(hddm_eps), "-hddm-max-loop", str(hddm_max_loop), "MODEL"]
    subprocess.run(cmd, cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   timeout=timeout)
    nv = model.n_vertices
    out = dict(json=json.load(open(os.path.join(mdir, "ref.json"))))
    out["x"] = read_sol(os.path.join(mdir, "ref.sol"), nv, model.n_edges)
    out["norm0"], out["hist"] = read_log(os.path.join(mdir, "calc_log", "log_g_HDDM_Full_Wave"))
    # the same history at full precision, recorded by the harness (not by the
    # GPU table, whose interface vectors stay on the device)
    hp = os.path.join(mdir, "ref.hist")
    if os.path.exists(hp):
        h = np.fromfile(hp, dtype="<f8")
        out["norm0_full"], out["hist_full"] = float(h[0]), h[1:].copy()
    # seconds of each interface iteration after the first (subdomain solves + COCG step)
    out["iteration_s"] = np.fromfile(os.path.join(mdir, "ref.itimes"), dtype="<f8")
    if dump >= 1:
        out["infree"], out["ints"] = read_ints(os.path.join(mdir, "ref.ints"), nv)
        out["post"] = read_post(os.path.join(mdir, "ref.post"), model.n_tets)
        out["post_drop"] = read_post(os.path.join(mdir, "ref.post_drop"), model.n_tets)
    if dump >= 2:
        out["aij"] = read_aij(os.path.join(mdir, "ref.aij"))
        out["fac"] = read_fac(os.path.join(mdir, "ref.fac"))
    out["workdir"] = wd
    return out


def read_cojo(path: str):
    """The correction-Jo dump of the harness in main() mode (<prefix>.cojo):
    per antenna its flag, interface size and, per subdomain of every part in
    order, the global node id of each antenna DOF (enf order), the Dirichlet
    list, the interface entries (nfid, ln_part) and the potentials Ihr, Ihi."""
    lines = open(path).read().split("\n")
    pos = 0

    def nxt():
        nonlocal pos
        pos += 1
        return lines[pos - 1]

    nant, nsub = (int(t) for t in nxt().split())
    out = []
    for _ in range(nant):
        flag, tfree = (int(t) for t in nxt().split())
        subs = []
        for _ in range(nsub):
            nf, nbc, ninbc = (int(t) for t in nxt().split())
            d = dict(nf=nf)
            if nf:
                d["gid"] = np.array(nxt().split(), np.int64)
                d["ibc"] = np.array(nxt().split(), np.int64)
                ib = np.array(nxt().split(), np.int64).reshape(-1, 2)
                d["inbc_nfid"], d["inbc_ln"] = ib[:, 0], ib[:, 1]
                d["ihr"] = np.array(nxt().split(), np.float64)
                d["ihi"] = np.array(nxt().split(), np.float64)
                assert d["gid"].shape[0] == nf and d["ibc"].shape[0] == nbc and ib.shape[0] == ninbc
            subs.append(d)
        out.append(dict(flag=flag, total_free=tfree, subs=subs))
    return out


def read_log_sections(path: str):
    """Every section of a reference calc_log: title, interface DOFs, initial
    max-norm and the residual per iteration (7 digits)."""
    secs = []
    for line in open(path):
        t = line.split()
        if line.startswith("# ") and not line.startswith("# DOF") and not line.startswith("#   "):
            secs.append(dict(title=line[2:].strip(), dof=None, norm0=None, hist=[]))
        elif line.startswith("# DOF on interface"):
            secs[-1]["dof"] = int(t[-1])
        elif len(t) >= 5 and t[0] == "0" and t[2] == "#" and t[3] == "Norm":
            secs[-1]["norm0"] = float(t[4])
        elif len(t) == 2 and not line.startswith("#"):
            secs[-1]["hist"].append(float(t[1]))
    for sec in secs:
        sec["hist"] = np.array(sec["hist"])
    return secs


def run_cojo(model_dir: str, workdir: str, timeout=600, binary: str = HARNESS):
    """Run main()'s correction-Jo pre-solve of the reference on a model
    directory (copied into workdir/MODEL) and return the parsed dump and the
    log sections.  binary=HARNESS_GPU runs it through the GPU tables."""
    import shutil

    mdir = os.path.join(workdir, "MODEL")
    if os.path.abspath(model_dir) != os.path.abspath(mdir):
        shutil.copytree(model_dir, mdir, ignore=shutil.ignore_patterns("calc_log", "result"))
    env = dict(os.environ, FW_HARNESS_MAIN="1", FW_HARNESS_COJO_ONLY="1", FW_HARNESS_OUT=os.path.join(mdir, "ref"))
    subprocess.run([binary, "-memlimit", "60000", "MODEL"], cwd=workdir, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=timeout)
    return read_cojo(os.path.join(mdir, "ref.cojo")), read_log_sections(
        os.path.join(mdir, "calc_log", "log_g_HDDM_Full_Wave"))
