"""CPU oracle of the full-wave HDDM hot path.

TEST INFRASTRUCTURE ONLY: used by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker; the product never
imports it.  Two parts:

* ``partition`` restates, in numpy, the integer setup the reference's
  ``make_PartMesh_FW`` (``lib/hddm/make_PartMesh.c:1201-1241``) performs for
  one part: subdomain-local vertex and edge numbering in subdomain node order
  (``make_MESH_make_ap``/``change_ap``, ``lib/fem/make_MESH.c:237-272,539-552``),
  the slot-8/9 swap of ``nop`` (``make_MESH.c:556-585``), the interface DOFs
  (mid-nodes shared by subdomains, PEC ones excluded, part-interface order,
  ``make_PartMesh.c:158-748``) and the Dirichlet list with the interface DOFs
  last (``make_PartMesh.c:1068-1194``).
* ``hddm`` runs ``oracle/fw_oracle.c`` (built into ``oracle/liboracle.so``),
  the C restatement of the reference's assembly, skyline LDL^T and s-mode
  COCG, on those arrays.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
FILE_SLOT = np.array([0, 1, 2, 3, 5, 4])  # tet_n slot -> file mid-node


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "fw_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        # gcc -O2 as the reference's Makefile.in:33
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", LIB, src, "-lm"], check=True)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
    return _lib


@dataclass
class SubData:
    els: np.ndarray        # global element ids
    nop: np.ndarray        # (nel, 10) local ids after the slot swap
    crd: np.ndarray        # (nap, 3) local vertex coordinates
    eps: np.ndarray        # (nel,)
    sigma: np.ndarray      # (nel,)
    edge_gid: np.ndarray   # (nmp,) global edge id of each local edge
    ibc: np.ndarray        # Dirichlet list: PEC (sorted) then interface (sorted)
    inbc_nfid: np.ndarray  # sorted local ids of interface DOFs
    inbc_ln: np.ndarray    # their part-interface numbers
    b: np.ndarray          # (nmp,) complex assembled source right-hand side


@dataclass
class Partition:
    subs: List[SubData]
    tfree: int
    iface_gid: np.ndarray


def material_per_element(model) -> tuple:
    """First match of each element flag in the Permittivity and Conductor
    tables (``lib/fem/make_elem_em.c:98-109``)."""
    eps = np.zeros(model.n_tets)
    sig = np.zeros(model.n_tets)
    # the tables have unique flags, so a dictionary lookup is the first match
    emap = {}
    for f, e in zip(model.mat_flag.tolist(), model.mat_eps.tolist()):
        emap.setdefault(f, e)
    smap = {}
    for f, s in zip(model.mat_flag.tolist(), model.mat_sigma.tolist()):
        smap.setdefault(f, s)
    fl = model.flag.tolist()
    eps[:] = [emap.get(f, 0.0) for f in fl]
    sig[:] = [smap.get(f, 0.0) for f in fl]
    return eps, sig


def element_rhs(model) -> np.ndarray:
    """The element right-hand sides of ``model.element_source``
    (``tet_MakeElement_EM_E``, ``lib/fem/make_elem_em.c:66-330``): (n_tets, 6)
    complex in the edge-table order, zeros where an element has none."""
    nt = model.n_tets
    out = np.zeros((nt, 6), np.complex128)
    es = getattr(model, "element_source", None)
    if es is None:
        return out
    lib = load()
    lib.orc_element_rhs.restype = None
    _, sig = material_per_element(model)
    ng = es.n_gaps
    box = np.ascontiguousarray(es.gap_box, np.float64).reshape(-1)
    volt = np.ascontiguousarray(es.gap_volt, np.float64)
    if box.size == 0:
        box = np.zeros(6)
        volt = np.zeros(1)
    # first antenna whose flag matches (make_elem_em.c:110-115)
    ant = np.full(nt, -1, np.int64)
    if ng == 0:
        for k in range(es.n_antennas - 1, -1, -1):
            ant[model.flag == es.antenna_flag[k]] = k
    be = np.zeros(12, np.float64)
    joe = np.zeros(24, np.float64)
    for t in range(nt):
        if ng == 0 and ant[t] < 0:
            continue
        v = model.tets[t]
        xyz = np.ascontiguousarray(np.concatenate([model.vertex_crd[v, 0], model.vertex_crd[v, 1],
                                                   model.vertex_crd[v, 2]]), np.float64)
        if ant[t] >= 0:
            k = ant[t]
            joe[0::2] = -es.antenna_Jo[k][v].ravel()
            joe[1::2] = -es.antenna_Jor[k][v].ravel()
        lib.orc_element_rhs(_p(xyz, ctypes.c_double), ctypes.c_double(sig[t]), ctypes.c_double(model.omega),
                            ctypes.c_int(ng), _p(box, ctypes.c_double), _p(volt, ctypes.c_double),
                            ctypes.c_int(1 if ant[t] >= 0 else 0), _p(joe, ctypes.c_double), _p(be, ctypes.c_double))
        out[t] = be[0::2] + 1j * be[1::2]
    return out


def partition(model, source=0) -> Partition:
    nv = model.n_vertices
    ne = model.n_edges
    nsub = model.nsub
    order = np.argsort(model.sub_of_tet, kind="stable")
    counts = np.bincount(model.sub_of_tet, minlength=nsub)
    starts = np.concatenate([[0], np.cumsum(counts)])
    eps, sig = material_per_element(model)
    held = np.zeros(ne, dtype=np.int64)
    owner = np.full(ne, -1, dtype=np.int64)
    sub_edges = []
    for s in range(nsub):
        els = order[starts[s]:starts[s + 1]]
        e = np.unique(model.tet_edges[els])
        sub_edges.append(e)
        held[e] += 1
        new = owner[e] < 0
        owner[e[new]] = s
    iface = (held >= 2) & ~model.pec_edge
    iface_gid = np.nonzero(iface)[0]
    ln_of = np.full(ne, -1, dtype=np.int64)
    ln_of[iface_gid] = np.arange(iface_gid.shape[0])
    if source is None:
        src_e, src_v = np.zeros(0, np.int64), np.zeros(0, np.complex128)
    elif isinstance(source, int):
        src_e, src_v = model.sources[source]
    else:
        src_e, src_v = source
    ebe = element_rhs(model) if getattr(model, "element_source", None) is not None else None
    subs = []
    for s in range(nsub):
        els = order[starts[s]:starts[s + 1]]
        e = sub_edges[s]
        v = np.unique(model.tets[els])
        eloc = {int(g): i for i, g in enumerate(e.tolist())}
        vloc = np.full(nv, -1, dtype=np.int64)
        vloc[v] = np.arange(v.shape[0])
        nop = np.empty((els.shape[0], 10), dtype=np.int32)
        nop[:, :4] = vloc[model.tets[els]]
        te = model.tet_edges[els][:, FILE_SLOT]
        nop[:, 4:] = np.searchsorted(e, te)
        pec_l = np.nonzero(model.pec_edge[e])[0]
        if_l = np.nonzero(iface[e])[0]
        b = np.zeros(e.shape[0], dtype=np.complex128)
        if ebe is not None:
            # SetFe (aij_matrix_func.h:327-338): element by element, in element order
            for k in range(els.shape[0]):
                for i in range(6):
                    b[nop[k, 4 + i]] += ebe[els[k], i]
        for g, val in zip(np.asarray(src_e).tolist(), np.asarray(src_v).tolist()):
            if owner[g] == s:
                b[eloc[g]] += val
        subs.append(SubData(els=els, nop=nop, crd=model.vertex_crd[v], eps=eps[els], sigma=sig[els], edge_gid=e,
                            ibc=np.concatenate([pec_l, if_l]).astype(np.int32), inbc_nfid=if_l.astype(np.int32),
                            inbc_ln=ln_of[e[if_l]].astype(np.int32), b=b))
    return Partition(subs=subs, tfree=int(iface_gid.shape[0]), iface_gid=iface_gid)


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def hddm(model, part: Partition, hddm_eps: float = 1e-3, hddm_max_loop: int = 4000):
    """The reference's s-mode HDDM solve on ``part``.  Returns
    (per-edge solution (global edge ids, lowest subdomain's value),
    per-subdomain solutions, residual history, initial norm)."""
    lib = load()
    subs = part.subs
    nsub = len(subs)
    i32, f64 = ctypes.c_int32, ctypes.c_double
    nel = np.array([s.nop.shape[0] for s in subs], np.int32)
    nap = np.array([s.crd.shape[0] for s in subs], np.int32)
    nmp = np.array([s.edge_gid.shape[0] for s in subs], np.int32)
    nbc = np.array([s.ibc.shape[0] for s in subs], np.int32)
    nin = np.array([s.inbc_nfid.shape[0] for s in subs], np.int32)
    nop = np.ascontiguousarray(np.concatenate([s.nop for s in subs]), np.int32)
    crd = np.ascontiguousarray(np.concatenate([s.crd for s in subs]), np.float64)
    eps = np.ascontiguousarray(np.concatenate([s.eps for s in subs]), np.float64)
    sig = np.ascontiguousarray(np.concatenate([s.sigma for s in subs]), np.float64)
    ibc = np.ascontiguousarray(np.concatenate([s.ibc for s in subs]), np.int32)
    nf = np.ascontiguousarray(np.concatenate([s.inbc_nfid for s in subs]), np.int32)
    ln = np.ascontiguousarray(np.concatenate([s.inbc_ln for s in subs]), np.int32)
    bb = np.concatenate([s.b for s in subs])
    b = np.ascontiguousarray(np.stack([bb.real, bb.imag], 1).ravel(), np.float64)
    x = np.zeros(2 * int(nmp.sum()), np.float64)
    hist = np.zeros(max(1, hddm_max_loop) + 1, np.float64)
    norm0 = ctypes.c_double()
    lib.orc_hddm.restype = ctypes.c_int
    it = lib.orc_hddm(nsub, _p(nel, i32), _p(nop, i32), _p(nap, i32), _p(crd, f64), _p(eps, f64), _p(sig, f64),
                      _p(nmp, i32), _p(nbc, i32), _p(ibc, i32), _p(nin, i32), _p(nf, i32), _p(ln, i32), _p(b, f64),
                      int(part.tfree), ctypes.c_double(model.omega), ctypes.c_double(hddm_eps), int(hddm_max_loop),
                      _p(x, f64), _p(hist, f64), ctypes.byref(norm0))
    if it < 0:
        raise RuntimeError(f"oracle failed with {it}")
    xs = x[0::2] + 1j * x[1::2]
    per_sub = np.split(xs, np.cumsum(nmp)[:-1])
    xe = np.zeros(model.n_edges, dtype=np.complex128)
    seen = np.zeros(model.n_edges, dtype=bool)
    for s, xv in zip(subs, per_sub):
        new = ~seen[s.edge_gid]
        xe[s.edge_gid[new]] = xv[new]
        seen[s.edge_gid] = True
    return xe, per_sub, hist[:it], norm0.value


def assemble_sub(model, sub: SubData):
    lib = load()
    i32, f64 = ctypes.c_int32, ctypes.c_double
    nmp = sub.edge_gid.shape[0]
    nop = np.ascontiguousarray(sub.nop, np.int32)
    crd = np.ascontiguousarray(sub.crd, np.float64)
    eps = np.ascontiguousarray(sub.eps, np.float64)
    sig = np.ascontiguousarray(sub.sigma, np.float64)
    b = np.ascontiguousarray(np.stack([sub.b.real, sub.b.imag], 1).ravel(), np.float64)
    cap = 64 * nmp + 64
    rp = np.zeros(nmp + 1, np.int32)
    col = np.zeros(cap, np.int32)
    val = np.zeros(2 * cap, np.float64)
    bo = np.zeros(2 * nmp, np.float64)
    lib.orc_assemble_sub.restype = ctypes.c_int
    n = lib.orc_assemble_sub(int(nop.shape[0]), _p(nop, i32), _p(crd, f64), _p(eps, f64), _p(sig, f64), nmp,
                             _p(b, f64), ctypes.c_double(model.omega), cap, _p(rp, i32), _p(col, i32), _p(val, f64),
                             _p(bo, f64))
    if n < 0:
        raise RuntimeError("assembly buffer too small")
    return rp, col[:n], val[0:2 * n:2] + 1j * val[1:2 * n:2], bo[0::2] + 1j * bo[1::2]


def factor_sub(model, sub: SubData):
    lib = load()
    i32, f64 = ctypes.c_int32, ctypes.c_double
    nmp = sub.edge_gid.shape[0]
    nop = np.ascontiguousarray(sub.nop, np.int32)
    crd = np.ascontiguousarray(sub.crd, np.float64)
    eps = np.ascontiguousarray(sub.eps, np.float64)
    sig = np.ascontiguousarray(sub.sigma, np.float64)
    ibc = np.ascontiguousarray(sub.ibc, np.int32)
    idx1 = np.zeros(nmp, np.int32)
    idx2 = np.zeros(nmp, np.int32)
    lib.orc_factor_sub.restype = ctypes.c_int
    cap = nmp * (nmp + 1) // 2 + 1
    mat = np.zeros(2 * cap, np.float64)
    n = lib.orc_factor_sub(int(nop.shape[0]), _p(nop, i32), _p(crd, f64), _p(eps, f64), _p(sig, f64), nmp,
                           int(ibc.shape[0]), _p(ibc, i32), ctypes.c_double(model.omega), cap, _p(idx1, i32),
                           _p(idx2, i32), _p(mat, f64))
    if n < 0:
        raise RuntimeError("factor buffer too small")
    return idx1, idx2, n, mat[0:2 * n:2] + 1j * mat[1:2 * n:2]


def element_ss(model, t: int) -> np.ndarray:
    """Mass matrix SS_e (tetNedelec_sideside) of element t in the edge-table
    order, from the restated element routine: with eps = 0 and sigma = 1 its
    imaginary part is exactly SS_e (make_elem_em.c:254-265)."""
    lib = load()
    v = model.tets[t]
    xyz = np.ascontiguousarray(np.concatenate([model.vertex_crd[v, 0], model.vertex_crd[v, 1],
                                               model.vertex_crd[v, 2]]), np.float64)
    ae = np.zeros(72, np.float64)
    lib.orc_element_matrix.restype = ctypes.c_int
    lib.orc_element_matrix(_p(xyz, ctypes.c_double), ctypes.c_double(0.0), ctypes.c_double(1.0),
                           ctypes.c_double(model.omega), _p(ae, ctypes.c_double))
    return ae[1::2].reshape(6, 6)


def adjoint_gradient(model, probe_edges, design_tets, hddm_eps: float = 1e-12, hddm_max_loop: int = 20000):
    """FP64 reference gradient of J = sum_p |x_p|^2 with respect to eps [F/m]
    and sigma [S/m] of each design element: forward and adjoint HDDM solves
    with the restated reference solver, then dJ/deps = 2 omega Re(s),
    dJ/dsigma = 2 Im(s), s = lambda_e^T SS_e x_e."""
    part = partition(model, 0)
    x, _, _, _ = hddm(model, part, hddm_eps, hddm_max_loop)
    pe = np.asarray(probe_edges)
    J = float(np.sum(np.abs(x[pe]) ** 2))
    part_adj = partition(model, (pe, np.conj(x[pe])))
    lam, _, _, _ = hddm(model, part_adj, hddm_eps, hddm_max_loop)
    ge = np.zeros(len(design_tets))
    gs = np.zeros(len(design_tets))
    for k, t in enumerate(design_tets):
        edges = model.tet_edges[t][FILE_SLOT]
        s = lam[edges] @ element_ss(model, int(t)) @ x[edges]
        ge[k] = 2.0 * model.omega * s.real
        gs[k] = 2.0 * s.imag
    return J, ge, gs, x


def objective(model, probe_edges, hddm_eps: float = 1e-12, hddm_max_loop: int = 20000) -> float:
    part = partition(model, 0)
    x, _, _, _ = hddm(model, part, hddm_eps, hddm_max_loop)
    return float(np.sum(np.abs(x[np.asarray(probe_edges)]) ** 2))


def post_em_E(model, xedge, drop_first: bool = False):
    """Element results of the post step (``HDDM_post_em_E``,
    ``main/fullwave/fullwave.c:639-763``) from the edge solution ``xedge``:
    returns (B, E, Je), each (n_tets, 3) complex, in global element order.
    The Permittivity and Conductor lists are the model's material table;
    ``drop_first`` leaves out the first entry of each, so that the elements of
    that flag take the nu = 0 and sigma = 0 branches."""
    lib = load()
    flags = np.ascontiguousarray(model.mat_flag, np.int32)
    sig = np.ascontiguousarray(model.mat_sigma, np.float64)
    k = 1 if drop_first and flags.shape[0] > 0 else 0
    flags, sig = np.ascontiguousarray(flags[k:]), np.ascontiguousarray(sig[k:])
    nt = model.n_tets
    x = np.ascontiguousarray(np.stack([np.real(xedge), np.imag(xedge)], 1).ravel(), np.float64)
    out = [np.zeros(6 * nt, np.float64) for _ in range(3)]
    tv = np.ascontiguousarray(model.tets, np.int32)
    te = np.ascontiguousarray(model.tet_edges, np.int32)
    crd = np.ascontiguousarray(model.vertex_crd, np.float64)
    fl = np.ascontiguousarray(model.flag, np.int32)
    lib.orc_post_em_E.restype = ctypes.c_int
    bad = lib.orc_post_em_E(ctypes.c_int(nt), _p(tv, ctypes.c_int), _p(te, ctypes.c_int), _p(crd, ctypes.c_double),
                            _p(fl, ctypes.c_int), ctypes.c_int(flags.shape[0]), _p(flags, ctypes.c_int),
                            ctypes.c_int(flags.shape[0]), _p(flags, ctypes.c_int), _p(sig, ctypes.c_double),
                            ctypes.c_double(model.omega), _p(x, ctypes.c_double), *[_p(o, ctypes.c_double) for o in out])
    if bad:
        raise ValueError(f"{bad} elements with a zero-length edge")
    return tuple((o[0::2] + 1j * o[1::2]).reshape(nt, 3) for o in out)
