"""The reference's model and result files, read and written in Python.

A user of the reference keeps a model as a directory (``./MODEL``) holding:

- ``model/advhddm_in_<part>.adv``: one ADVENTURE HDDM part file per part,
  read by ``read_modeldata_file`` (``lib/std/fileio.c:760-991``);
- ``mtrl.dat``: the material table, read by ``read_mtrldat_file``
  (``fileio.c:3474-3572``);
- ``volt.dat``: the source selection of the element routine
  (``lib/fem/make_elem_em.c:74-96,332-346``).

``load_model`` turns such a directory into a ``meshgen.Model`` that
``hddm.HddmSolver`` solves. ``write_result`` writes a solution in the
layout of the reference's result file (``write_outdata_file_HDDM_FW``,
``fileio.c:2930-3160``).

The part files are AdvDoc containers. Each document is stored as:

    "AdvDoc\\0" | int64 payload length | payload |
    int64 header length | int32 len + document id | int32 property count |
    (int32 len + key, int32 len + value) ...

All values are little endian. A file is a concatenation of documents.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import meshgen

MAGIC = b"AdvDoc\0"


@dataclass
class AdvDoc:
    did: str
    props: Dict[str, str]
    payload: bytes


def read_advdoc(path: str) -> List[AdvDoc]:
    """Every document of an AdvDoc file, in file order."""
    data = open(path, "rb").read()
    docs = []
    o = 0
    while o < len(data):
        if data[o:o + 7] != MAGIC:
            raise ValueError(f"{path}: no AdvDoc document at byte {o}")
        o += 7
        (plen,) = struct.unpack_from("<q", data, o)
        o += 8
        payload = data[o:o + plen]
        o += plen
        (hlen,) = struct.unpack_from("<q", data, o)
        o += 8
        h = data[o:o + hlen]
        o += hlen
        k = 0
        (n,) = struct.unpack_from("<i", h, k)
        k += 4
        did = h[k:k + n].decode()
        k += n
        (np_,) = struct.unpack_from("<i", h, k)
        k += 4
        props = {}
        for _ in range(np_):
            (n,) = struct.unpack_from("<i", h, k)
            key = h[k + 4:k + 4 + n].decode()
            k += 4 + n
            (n,) = struct.unpack_from("<i", h, k)
            val = h[k + 4:k + 4 + n].decode()
            k += 4 + n
            props[key] = val
        docs.append(AdvDoc(did, props, payload))
    return docs


def write_advdoc(path: str, docs: List[AdvDoc]) -> None:
    with open(path, "wb") as f:
        for d in docs:
            h = bytearray()
            h += struct.pack("<i", len(d.did)) + d.did.encode()
            h += struct.pack("<i", len(d.props))
            for k, v in d.props.items():
                h += struct.pack("<i", len(k)) + k.encode()
                h += struct.pack("<i", len(v)) + v.encode()
            f.write(MAGIC + struct.pack("<q", len(d.payload)) + d.payload + struct.pack("<q", len(h)) + bytes(h))


def _find(docs: List[AdvDoc], key: str, value: str) -> AdvDoc:
    for d in docs:
        if d.props.get(key) == value:
            return d
    raise KeyError(f"no document with {key} = {value}")


def _per_subdomain(payload: bytes, nsub: int, width: int, dtype: str = "<i4") -> List[np.ndarray]:
    """Lists stored as (int32 count, count*width items) per subdomain."""
    out = []
    o = 0
    for _ in range(nsub):
        (n,) = struct.unpack_from("<i", payload, o)
        o += 4
        a = np.frombuffer(payload, dtype, n * width, o)
        o += a.nbytes
        out.append(a.reshape(n, width) if width > 1 else a)
    return out


@dataclass
class HddmPart:
    """One part file as read_modeldata_file keeps it in PartMesh/DomMesh."""

    part: int
    crd: np.ndarray                 # (nnd, 3) part node coordinates
    pnid2gnid: np.ndarray           # (nnd,) part node -> global node
    nd_elem: int
    nop: List[np.ndarray]           # per subdomain (nel, nd_elem) subdomain node ids
    snid2pnid: List[np.ndarray]     # per subdomain: subdomain node -> part node
    inbc: List[np.ndarray]          # per subdomain (ninbc, 5): snid, coordinate, charge_part, ln_chpar, ln_part
    dbc: Optional[List[np.ndarray]]  # per subdomain: Dirichlet (Axn0) subdomain node ids
    flag: List[np.ndarray]          # per subdomain (nel,)
    seid2geid: List[np.ndarray]     # per subdomain (nel,) global element ids
    props: Dict[str, Dict[str, str]] = field(default_factory=dict)


def read_hddm_part(path: str) -> HddmPart:
    """``read_modeldata_file`` (``lib/std/fileio.c:760-991``) for one part."""
    docs = read_advdoc(path)
    node = _find(docs, "content_type", "Node")
    nnd = int(node.props["num_items"])
    dim = int(node.props["dimension"])
    crd = np.frombuffer(node.payload, "<f8", nnd * dim).reshape(nnd, dim)
    p2g = np.frombuffer(_find(docs, "label", "NodeIndex_PartToGlobal").payload, "<i4", nnd)
    ifd = _find(docs, "content_type", "HDDM_InterfaceDOF")
    nsub = int(ifd.props["num_subdomains"])
    el = _find(docs, "content_type", "HDDM_Element")
    nd = int(el.props["num_nodes_per_element"])
    opts = _find(docs, "label", "Options")
    need_dbc = opts.props.get("DirichletBCs_Axn0") == "NEED"
    return HddmPart(
        part=int(ifd.props.get("part_number", 0)), crd=crd, pnid2gnid=p2g, nd_elem=nd,
        nop=_per_subdomain(el.payload, nsub, nd),
        snid2pnid=_per_subdomain(_find(docs, "label", "NodeIndex_SubdomainToPart").payload, nsub, 1),
        inbc=_per_subdomain(_find(docs, "label", "InterfaceDOF").payload, nsub, 5),
        dbc=_per_subdomain(_find(docs, "label", "DirichletBCs_Axn0").payload, nsub, 1) if need_dbc else None,
        flag=_per_subdomain(_find(docs, "label", "Flag").payload, nsub, 1),
        seid2geid=_per_subdomain(_find(docs, "label", "ElementIndex_SubdomainToGlobal").payload, nsub, 1),
        props={"Options": opts.props, "HDDM_InterfaceDOF": ifd.props, "HDDM_Element": el.props})


@dataclass
class Material:
    """``mtrl.dat`` as ``read_mtrldat_file`` keeps it in MTRL."""

    eps_flag: np.ndarray
    eps: np.ndarray
    sigma_flag: np.ndarray
    sigma: np.ndarray
    omega: float
    antennas: List[Tuple[int, str, str]]  # (flag, mode, file name)


def read_mtrl(path: str) -> Material:
    """The sections of ``mtrl.dat`` the full-wave path uses: Permittivity,
    Conductor, Antenna and AntennaOmega (``fileio.c:3474-3572``).  The
    reference sorts the Permittivity list by flag (``:3504``)."""
    toks = open(path).read().split()
    eps_f, eps_v, sig_f, sig_v, ants = [], [], [], [], []
    omega = None
    i = 0
    while i < len(toks):
        t = toks[i]
        if t == "Permittivity":
            n = int(toks[i + 1])
            for k in range(n):
                eps_f.append(int(toks[i + 2 + 2 * k]))
                eps_v.append(float(toks[i + 3 + 2 * k]))
            i += 2 + 2 * n
        elif t == "Conductor":
            n = int(toks[i + 1])
            for k in range(n):
                sig_f.append(int(toks[i + 2 + 2 * k]))
                sig_v.append(float(toks[i + 3 + 2 * k]))
            i += 2 + 2 * n
        elif t == "Antenna":
            n = int(toks[i + 1])
            for k in range(n):
                ants.append((int(toks[i + 2 + 3 * k]), toks[i + 3 + 3 * k], toks[i + 4 + 3 * k]))
            i += 2 + 3 * n
        elif t == "AntennaOmega":
            omega = float(toks[i + 1])
            i += 2
        else:
            i += 1
    if omega is None:
        raise ValueError(f"{path}: no AntennaOmega")
    order = np.argsort(np.asarray(eps_f, np.int64), kind="stable")
    return Material(np.asarray(eps_f, np.int32)[order], np.asarray(eps_v, np.float64)[order],
                    np.asarray(sig_f, np.int32), np.asarray(sig_v, np.float64), omega, ants)


def read_volt(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """``volt.dat``: dg, then per gap the x, y and z bounds and dV
    (``make_elem_em.c:96,332-346``).  Returns (boxes (dg, 6), volts (dg,))."""
    lines = [ln for ln in open(path).read().splitlines() if ln.strip()]
    dg = int(lines[0].split()[0])
    boxes = np.zeros((dg, 6))
    volts = np.zeros(dg)
    for k in range(dg):
        xb, yb, zb, dv = (lines[1 + 4 * k + q].split() for q in range(4))
        boxes[k] = [float(xb[0]), float(xb[1]), float(yb[0]), float(yb[1]), float(zb[0]), float(zb[1])]
        volts[k] = float(dv[0])
    return boxes, volts


@dataclass
class LoadedModel:
    model: meshgen.Model
    parts: List[HddmPart]
    material: Material
    vertex_gnid: np.ndarray   # global node id of each vertex
    edge_gnid: np.ndarray     # global node id (mid-node) of each edge
    sub_part: np.ndarray      # (nsub, 2): part and subdomain-in-part of each subdomain


# mid-node slots of a quadratic tetrahedron in file order: 01, 02, 03, 12, 23, 13
_MID_PAIRS = ((0, 1), (0, 2), (0, 3), (1, 2), (2, 3), (1, 3))


def load_model(model_dir: str, name: Optional[str] = None) -> LoadedModel:
    """Reads ``<model_dir>/model/advhddm_in_*.adv``, ``mtrl.dat`` and, if
    present, ``volt.dat`` into one model with global vertex and edge numbers.

    Subdomains are numbered part by part.  Vertices and edges are numbered
    in ascending global node id.  An edge is on the PEC wall when its
    mid-node is in a subdomain's DirichletBCs_Axn0 list.  A ``volt.dat``
    with gaps becomes the model's delta-gap source.  Antenna currents come
    from the reference's correction-Jo pre-solve and are not in these
    files, so a model driven by an antenna has no source after loading."""
    mdir = os.path.join(model_dir, "model")
    files = sorted((f for f in os.listdir(mdir) if f.startswith("advhddm_in_") and f.endswith(".adv")),
                   key=lambda f: int(f[len("advhddm_in_"):-4]))
    if not files:
        raise FileNotFoundError(f"no advhddm_in_*.adv under {mdir}")
    parts = [read_hddm_part(os.path.join(mdir, f)) for f in files]
    mat = read_mtrl(os.path.join(model_dir, "mtrl.dat"))

    n_el = sum(int(sum(a.shape[0] for a in p.nop)) for p in parts)
    el_nodes = np.zeros((n_el, 10), np.int64)
    el_flag = np.zeros(n_el, np.int32)
    el_sub = np.zeros(n_el, np.int32)
    seen = np.zeros(n_el, bool)
    gcrd: Dict[int, np.ndarray] = {}
    pec_gnid = []
    sub_part = []
    sub = 0
    max_g = 0
    for p in parts:
        if p.nd_elem != 10:
            raise ValueError("only quadratic tetrahedra (10 nodes) carry edge elements")
        max_g = max(max_g, int(p.pnid2gnid.max()) + 1)
    g_crd = np.full((max_g, 3), np.nan)
    for p in parts:
        g_crd[p.pnid2gnid] = p.crd
        for s in range(len(p.nop)):
            gn = p.pnid2gnid[p.snid2pnid[s]]
            ge = p.seid2geid[s]
            if ge.max() >= n_el or seen[ge].any():
                raise ValueError("element ids are not a permutation of 0..n-1")
            seen[ge] = True
            el_nodes[ge] = gn[p.nop[s]]
            el_flag[ge] = p.flag[s]
            el_sub[ge] = sub
            if p.dbc is not None:
                pec_gnid.append(gn[p.dbc[s]])
            sub_part.append((p.part, s))
            sub += 1
    if not seen.all():
        raise ValueError("element ids are not a permutation of 0..n-1")
    vert_g = np.unique(el_nodes[:, :4])
    mid_g = np.unique(el_nodes[:, 4:])
    vidx = np.full(max_g, -1, np.int64)
    vidx[vert_g] = np.arange(vert_g.shape[0])
    eidx = np.full(max_g, -1, np.int64)
    eidx[mid_g] = np.arange(mid_g.shape[0])
    tets = vidx[el_nodes[:, :4]].astype(np.int32)
    tet_edges = eidx[el_nodes[:, 4:]].astype(np.int32)
    edges = np.zeros((mid_g.shape[0], 2), np.int32)
    for q, (a, b) in enumerate(_MID_PAIRS):
        lo = np.minimum(tets[:, a], tets[:, b])
        hi = np.maximum(tets[:, a], tets[:, b])
        edges[tet_edges[:, q], 0] = lo
        edges[tet_edges[:, q], 1] = hi
    pec = np.zeros(mid_g.shape[0], bool)
    if pec_gnid:
        g = np.concatenate(pec_gnid)
        g = g[eidx[g] >= 0]
        pec[eidx[g]] = True
    crd = g_crd[vert_g]
    flags = np.union1d(mat.eps_flag, mat.sigma_flag).astype(np.int32)
    eps_of = dict(zip(mat.eps_flag.tolist(), mat.eps.tolist()))
    sig_of = dict(zip(mat.sigma_flag.tolist(), mat.sigma.tolist()))
    model = meshgen.Model(
        name=name or os.path.basename(os.path.abspath(model_dir)), n=0,
        size=float(np.max(crd.max(axis=0) - crd.min(axis=0))), vertex_crd=np.ascontiguousarray(crd),
        tets=tets, tet_edges=tet_edges, edges=edges, flag=el_flag,
        mat_flag=flags, mat_eps=np.array([eps_of.get(f, 0.0) for f in flags.tolist()]),
        mat_sigma=np.array([sig_of.get(f, 0.0) for f in flags.tolist()]), omega=mat.omega, pec_edge=pec,
        sub_of_tet=el_sub, nsub=sub, sources=[])
    vpath = os.path.join(model_dir, "volt.dat")
    if os.path.exists(vpath):
        boxes, volts = read_volt(vpath)
        if volts.shape[0] > 0:
            meshgen.delta_gap_source(model, boxes, volts)
    return LoadedModel(model, parts, mat, vert_g, mid_g, np.asarray(sub_part, np.int32))


def read_result(path: str) -> Dict[str, List[np.ndarray]]:
    """A result file of the reference (``advhddm_out_<part>.adv``,
    ``write_outdata_file_HDDM_FW``): per label the per-subdomain arrays.
    The edge solution ("MagneticVectorPotential", format i4f8f8) gives
    (snid, value) per local edge; element fields give (nel, 3) values."""
    docs = read_advdoc(path)
    out: Dict[str, List[np.ndarray]] = {}
    for d in docs:
        label = d.props.get("label")
        nsub = int(d.props.get("num_subdomains", "0"))
        if label is None or nsub == 0:
            continue
        fmt = d.props.get("format", "")
        if label == "MagneticVectorPotential":
            rec = np.dtype([("snid", "<i4"), ("re", "<f8"), ("im", "<f8")])
            subs = []
            o = 0
            for _ in range(nsub):
                (n,) = struct.unpack_from("<i", d.payload, o)
                o += 4
                a = np.frombuffer(d.payload, rec, n, o)
                o += a.nbytes
                subs.append(a)
            out[label] = subs
        elif fmt == "f8f8f8":
            out[label] = _per_subdomain(d.payload, nsub, 3, "<f8")
    return out


def write_result(path: str, loaded: LoadedModel, part: int, x: np.ndarray,
                 B: Optional[np.ndarray] = None, E: Optional[np.ndarray] = None) -> None:
    """The result file of one part in the reference's layout
    (``write_outdata_file_HDDM_FW``, ``fileio.c:2930-3160``): the edge
    solution per subdomain as (snid, re, im) records keyed by the
    subdomain's own node ids, and, when given, the element fields
    B = i (nu/omega) rot E and E (from ``HddmSolver.post_em_E``) as real and
    imaginary (nel, 3) documents in each subdomain's element order."""
    p = loaded.parts[part]
    eidx = {int(g): k for k, g in enumerate(loaded.edge_gnid.tolist())}
    vec = bytearray()
    el_docs = {}
    for s in range(len(p.nop)):
        gn = p.pnid2gnid[p.snid2pnid[s]]
        mids = np.unique(p.nop[s][:, 4:])  # subdomain node ids of the mid-nodes
        vec += struct.pack("<i", mids.shape[0])
        for snid in mids.tolist():
            v = x[eidx[int(gn[snid])]]
            vec += struct.pack("<idd", int(snid), float(v.real), float(v.imag))
        ge = p.seid2geid[s]
        for label, arr in (("MagneticField", B), ("ElectricField", E)):
            if arr is None:
                continue
            for suffix, f in (("Real", np.real), ("Imaginary", np.imag)):
                el_docs.setdefault(label + suffix, bytearray())
                el_docs[label + suffix] += struct.pack("<i", ge.shape[0]) + np.ascontiguousarray(
                    f(arr[ge]), "<f8").tobytes()
    nsub = str(len(p.nop))
    docs = [AdvDoc("MagneticVectorPotential", {"content_type": "HDDM_FEGenericAttribute", "num_subdomains": nsub,
                                              "fega_type": "NodeVariable", "format": "f8f8",
                                              "label": "MagneticVectorPotential", "index_byte": "4"}, bytes(vec))]
    for label, payload in el_docs.items():
        docs.append(AdvDoc(label, {"content_type": "HDDM_FEGenericAttribute", "num_subdomains": nsub,
                                   "num_items_orig": str(loaded.model.n_tets), "fega_type": "AllElementVariable",
                                   "format": "f8f8f8", "label": label, "index_byte": "4"}, bytes(payload)))
    write_advdoc(path, docs)
