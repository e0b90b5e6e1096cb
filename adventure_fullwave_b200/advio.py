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


PI = 3.14159265358979323846  # lib/std/defs.h:218


@dataclass
class AntennaDefinition:
    """One shape of a ``md`` antenna definition file (``read_Jodefine_file``,
    ``fileio.c:1170-1470``): a parallelepiped ("pp") with its face
    equations, or a double sectorial cylinder ("dsc"), each with the real and
    imaginary current of the Full-Wave analysis."""

    kind: str
    ap: np.ndarray = None          # pp: 5 corner points (ap[4] opposite ap[0]); dsc: x0 y0 z0 z1
    abc: np.ndarray = None         # pp: face normals (3, 3)
    d: np.ndarray = None           # pp: (2, 3) face constants through ap[0] and ap[4]
    tolerance: float = 0.0
    jo_re: np.ndarray = None       # pp: (3,), dsc: scalar in [0]
    jo_im: np.ndarray = None
    xyz: int = 2                   # dsc axis
    theta: Tuple[float, float] = (0.0, 0.0)
    r2: Tuple[float, float] = (0.0, 0.0)


def _outer(p, q):
    n = ((1, 2), (2, 0), (0, 1))
    return [p[a] * q[b] - p[b] * q[a] for a, b in n]


def _face_d(abc, ap):
    dd = 0.0
    for i in range(3):
        dd += abc[i] * ap[i]
    return -dd


def read_jodefine(path: str) -> List[AntennaDefinition]:
    """The shapes of an antenna definition file, in file order."""
    toks = open(path).read().split()
    if not toks or toks[0] != "Full-Wave":
        raise ValueError(f"{path}: only Full-Wave antenna definitions are read")
    defs = []
    i = 1
    while i < len(toks):
        t = toks[i]
        i += 1
        if t == "Parallelpiped":
            ap = [[float(toks[i + 3 * k + j]) for j in range(3)] for k in range(4)]
            i += 12
            jr = [float(toks[i + j]) for j in range(3)]
            ji = [float(toks[i + 3 + j]) for j in range(3)]
            i += 6
            vec = [[ap[k][j] - ap[0][j] for j in range(3)] for k in range(1, 4)]
            ap4 = list(ap[0])
            for k in range(3):
                for j in range(3):
                    ap4[j] += vec[k][j]
            abc = [_outer(vec[0], vec[1]), _outer(vec[0], vec[2]), _outer(vec[1], vec[2])]
            d = [[_face_d(abc[k], ap[0]) for k in range(3)], [_face_d(abc[k], ap4) for k in range(3)]]
            tol = 1.0e100
            for k in range(3):
                dd = 0.0
                for j in range(3):
                    dd += vec[k][j] * vec[k][j]
                dd = float(np.sqrt(dd))
                if dd < tol:
                    tol = dd
            defs.append(AntennaDefinition("pp", ap=np.array(ap + [ap4]), abc=np.array(abc), d=np.array(d),
                                          tolerance=tol * 1.0e-05, jo_re=np.array(jr), jo_im=np.array(ji)))
        elif t == "DoubleSectorialCylinder":
            ap = [float(toks[i + j]) for j in range(3)]
            axis = toks[i + 3]
            height = float(toks[i + 4])
            i += 5
            x, y, z = {"x": (1, 2, 0), "y": (2, 0, 1), "z": (0, 1, 2)}[axis]
            if height == 0.0:
                raise ValueError(f"{path}: cylinder height 0")
            if height > 0.0:
                zr = (ap[z], ap[z] + height)
            else:
                zr = (ap[z] + height, ap[z])
            unit, theta, angle = toks[i], float(toks[i + 1]), float(toks[i + 2])
            i += 3
            if unit == "deg":
                theta = theta * PI / 180.0
                angle = angle * PI / 180.0
            elif unit != "rad":
                raise ValueError(f"{path}: angle unit {unit}")
            dd = 2.0 * PI
            if angle == 0.0:
                raise ValueError(f"{path}: rotation angle 0")
            elif angle > dd or angle < -dd:
                th = [0.0, 0.0]
            elif angle > 0.0:
                th = [theta, theta + angle]
            else:
                th = [theta + angle, theta]
            while PI < th[0]:
                th[0] += -dd
                th[1] += -dd
            while th[0] < -PI:
                th[0] += dd
                th[1] += dd
            r0, r1 = float(toks[i]), float(toks[i + 1])
            i += 2
            if not (0 <= r0 < r1):
                raise ValueError(f"{path}: cylinder radii")
            jr, ji = float(toks[i]), float(toks[i + 1])
            i += 2
            if height < 0.0:
                jr, ji = -jr, -ji
            defs.append(AntennaDefinition("dsc", ap=np.array([ap[x], ap[y], zr[0], zr[1]]),
                                          jo_re=np.array([jr]), jo_im=np.array([ji]),
                                          xyz={"x": 0, "y": 1, "z": 2}[axis], theta=(th[0], th[1]),
                                          r2=(r0 * r0, r1 * r1)))
        else:
            raise ValueError(f"{path}: unknown antenna shape {t}")
    return defs


def _pp_side(ap, xyz, tol, abc, d):
    d0 = d
    d1 = d
    for i in range(3):
        d0 += abc[i] * ap[i]
        d1 += abc[i] * xyz[i]
    if abs(d0) < tol:
        d0 = 0.0
    if abs(d1) < tol:
        d1 = 0.0
    return d0 * d1 >= 0.0


def antenna_currents(model: meshgen.Model, flag: int, defs: List[AntennaDefinition]) -> Tuple[np.ndarray, np.ndarray]:
    """The vertex currents an ``md`` antenna leaves in the reference:
    ``make_Jo_from_definition`` (``fileio.c:1553-1700``) over the vertices of
    the antenna's elements (``make_MESH.c:470-495``), shapes applied last to
    first so the first shape holding a vertex wins.  The reference runs it
    twice (``make_MESH.c:679,735``): Jor keeps the real-part pass (each shape's
    first current triple), Jo gets the imaginary part (its second).
    Returns (Jo, Jor), each (n_vertices, 3)."""
    nv = model.n_vertices
    jo = np.zeros((nv, 3))
    jor = np.zeros((nv, 3))
    verts = np.unique(model.tets[model.flag == flag])
    crd = model.vertex_crd
    for dfn in reversed(defs):
        for v in verts.tolist():
            c = crd[v].tolist()
            if dfn.kind == "pp":
                ok = True
                for j in range(3):
                    ok = _pp_side(c, dfn.ap[0], dfn.tolerance, dfn.abc[j], dfn.d[1][j])
                    if not ok:
                        break
                    ok = _pp_side(c, dfn.ap[4], dfn.tolerance, dfn.abc[j], dfn.d[0][j])
                    if not ok:
                        break
                if ok:
                    jor[v] = dfn.jo_re
                    jo[v] = dfn.jo_im
            else:
                x, y, z = {0: (1, 2, 0), 1: (2, 0, 1), 2: (0, 1, 2)}[dfn.xyz]
                a0 = c[x] - dfn.ap[0]
                a1 = c[y] - dfn.ap[1]
                a2 = c[z]
                ll = 0.0
                ll += a0 * a0
                ll += a1 * a1
                if ll < dfn.r2[0] or dfn.r2[1] < ll:
                    continue
                if a2 < dfn.ap[2] or dfn.ap[3] < a2:
                    continue
                import math
                theta = math.atan2(a1, a0)
                if not (dfn.theta[0] == 0.0 and dfn.theta[1] == 0.0):
                    if dfn.theta[1] < theta:
                        continue
                    elif theta < dfn.theta[0]:
                        theta += 2.0 * PI
                        if dfn.theta[1] < theta:
                            continue
                for arr, cur in ((jor, float(dfn.jo_re[0])), (jo, float(dfn.jo_im[0]))):
                    arr[v, x] = -cur * math.sin(theta)
                    arr[v, y] = cur * math.cos(theta)
                    arr[v, z] = 0.0
    return jo, jor


def read_jodata(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """A current data file of an ``rf`` antenna (``read_Jodata_file_read``,
    ``fileio.c:1016-1050``): the count, then per node its global node id and
    three current components.  Returns (node ids, (n, 3) currents) sorted by
    node id."""
    toks = open(path).read().split()
    n = int(toks[0])
    ids = np.array([int(toks[1 + 4 * k]) for k in range(n)], np.int64)
    val = np.array([[float(toks[2 + 4 * k + j]) for j in range(3)] for k in range(n)])
    order = np.argsort(ids, kind="stable")
    return ids[order], val[order]


def antenna_currents_from_files(model: meshgen.Model, flag: int, vertex_gnid: np.ndarray, real_path: str,
                                imag_path: str) -> Tuple[np.ndarray, np.ndarray]:
    """The vertex currents of an ``rf`` antenna: the real-part file
    (``<name>r``) gives Jor and the imaginary-part file (``<name>i``) gives Jo
    (``make_MESH.c:674-676,729-733``, ``read_Jodata_file_decompose``,
    ``fileio.c:1053-1106``), on the vertices of the antenna's elements; a
    vertex the file does not list gets 0.  Returns (Jo, Jor)."""
    nv = model.n_vertices
    held = np.zeros(nv, bool)
    held[np.unique(model.tets[model.flag == flag])] = True
    vidx = {int(g): k for k, g in enumerate(np.asarray(vertex_gnid).tolist())}
    out = []
    for path in (imag_path, real_path):
        a = np.zeros((nv, 3))
        ids, val = read_jodata(path)
        for g, v in zip(ids.tolist(), val):
            k = vidx.get(int(g))
            if k is not None and held[k]:
                a[k] = v
        out.append(a)
    return out[0], out[1]


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
    in ascending global node id; each subdomain keeps its local order, the
    part file's node order, in ``model.sub_order``.  An edge is on the PEC wall when its
    mid-node is in a subdomain's DirichletBCs_Axn0 list; vertex nodes of those
    lists go to ``model.pec_vertex`` (the correction-Jo problem's Dirichlet
    vertices).  A ``volt.dat``
    with gaps becomes the model's delta-gap source; otherwise the antennas
    of ``mtrl.dat`` become its antenna source, with the vertex currents the
    reference builds: from shape definitions (``md``, ``antenna_currents``)
    or from current data files (``rf``, ``antenna_currents_from_files``)."""
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
    sub_nodes = []
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
            sub_nodes.append(gn)
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
    pec_vertex = np.zeros(vert_g.shape[0], bool)
    if pec_gnid:
        g = np.concatenate(pec_gnid)
        pec[eidx[g[eidx[g] >= 0]]] = True
        # vertex nodes of the lists: the correction-Jo problem's Dirichlet vertices
        pec_vertex[vidx[g[vidx[g] >= 0]]] = True
    crd = g_crd[vert_g]
    # each subdomain's local order: its vertices, then its mid-nodes, in the
    # part file's node order (make_MESH_make_ap / make_MESH_change_ap)
    vptr, vord, eptr, eord = [0], [], [0], []
    for gn in sub_nodes:
        v = vidx[gn]
        e = eidx[gn]
        vord.append(v[v >= 0])
        eord.append(e[e >= 0])
        vptr.append(vptr[-1] + int((v >= 0).sum()))
        eptr.append(eptr[-1] + int((e >= 0).sum()))
    sub_order = (np.array(vptr, np.int32), np.concatenate(vord).astype(np.int32), np.array(eptr, np.int32),
                 np.concatenate(eord).astype(np.int32))
    flags = np.union1d(mat.eps_flag, mat.sigma_flag).astype(np.int32)
    # the reference takes the first entry of a flag listed twice (make_elem_em.c:98-109)
    eps_of, sig_of = {}, {}
    for f, v in zip(mat.eps_flag.tolist(), mat.eps.tolist()):
        eps_of.setdefault(f, v)
    for f, v in zip(mat.sigma_flag.tolist(), mat.sigma.tolist()):
        sig_of.setdefault(f, v)
    model = meshgen.Model(
        name=name or os.path.basename(os.path.abspath(model_dir)), n=0,
        size=float(np.max(crd.max(axis=0) - crd.min(axis=0))), vertex_crd=np.ascontiguousarray(crd),
        tets=tets, tet_edges=tet_edges, edges=edges, flag=el_flag,
        mat_flag=flags, mat_eps=np.array([eps_of.get(f, 0.0) for f in flags.tolist()]),
        mat_sigma=np.array([sig_of.get(f, 0.0) for f in flags.tolist()]), omega=mat.omega, pec_edge=pec,
        sub_of_tet=el_sub, nsub=sub, sources=[],
        eps_table=(mat.eps_flag.copy(), mat.eps.copy()), sigma_table=(mat.sigma_flag.copy(), mat.sigma.copy()),
        sub_order=sub_order, pec_vertex=pec_vertex if pec_vertex.any() else None)
    vpath = os.path.join(model_dir, "volt.dat")
    boxes, volts = read_volt(vpath) if os.path.exists(vpath) else (np.zeros((0, 6)), np.zeros(0))
    if volts.shape[0] > 0:
        meshgen.delta_gap_source(model, boxes, volts)
    elif mat.antennas:
        flags_a, jos, jors = [], [], []
        for flag, mode, fname in mat.antennas:
            if mode == "md":
                jo, jor = antenna_currents(model, flag, read_jodefine(os.path.join(model_dir, fname)))
            elif mode == "rf":
                jo, jor = antenna_currents_from_files(model, flag, vert_g, os.path.join(model_dir, fname + "r"),
                                                      os.path.join(model_dir, fname + "i"))
            else:
                raise ValueError(f"antenna mode {mode}")
            flags_a.append(flag)
            jos.append(jo)
            jors.append(jor)
        meshgen.antenna_source(model, flags_a, np.array(jos), np.array(jors))
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
                 B: Optional[np.ndarray] = None, E: Optional[np.ndarray] = None,
                 Je: Optional[np.ndarray] = None) -> None:
    """The result file of one part in the reference's layout
    (``write_outdata_file_HDDM_FW``, ``fileio.c:2930-3160``): the edge
    solution per subdomain as (snid, re, im) records keyed by the
    subdomain's own node ids, and, when given, the element fields
    B = i (nu/omega) rot E, E and Je (from ``HddmSolver.post_em_E``) as real
    and imaginary (nel, 3) documents in each subdomain's element order."""
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
        for label, arr in (("MagneticField", B), ("ElectricField", E), ("CurrentDensity", Je)):
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
