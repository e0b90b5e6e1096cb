"""Synthetic full-wave HDDM models: structured Kuhn tetrahedral meshes with
layered media, conductive "PML" shells, a PEC outer wall, z-dipole sources and
a (jittered) recursive-coordinate-bisection partition into subdomains.

These are the shared inputs of the path: the reference (through its own model
reader, ``lib/std/fileio.c:760-991`` ``read_modeldata_file``) and this package
consume the same mesh, flags, partition and source.  ``write_hddm_model``
writes them in the reference's ADVENTURE HDDM part-file layout so the
reference's unmodified reader and interface-numbering code
(``lib/hddm/make_PartMesh.c``) can run on them.

Conventions that the reference fixes and this generator follows:

* 10-node tetrahedra ("3DQuadraticTetrahedron"): 4 vertices, then the 6
  mid-edge nodes in file order 01, 02, 03, 12, 23, 13.  The reference swaps
  slots 8 and 9 on input to reach its edge table order 01, 02, 03, 12, 13, 23
  (``lib/fem/make_MESH.c:573-584``, ``lib/fem/tetrahedral.h:19-24``).
* every tetrahedron has positive ``tet_Volume6`` (``lib/fem/tetrahedral.c:44-61``).
* permittivity is absolute (F/m) per element flag, conductivity in S/m per
  flag, and ``mu_r = 1`` (``lib/fem/make_elem_em.c:37,98-109``).

Global numbering: vertex ``(i, j, k)`` has id ``i + (n+1)*(j + (n+1)*k)``;
edges are sorted by (lower vertex id, higher vertex id) and their mid-nodes
take ids ``n_vertices + edge_id``.  Subdomain-local node order is ascending
global node id; subdomain element order is ascending global element id.
"""
from __future__ import annotations

import dataclasses
import math
import os
import struct
from typing import List, Optional, Sequence, Tuple

import numpy as np

EPS0 = 8.854e-12
ETA0 = 376.73
FILE_EDGE_PAIRS = ((0, 1), (0, 2), (0, 3), (1, 2), (2, 3), (1, 3))


@dataclasses.dataclass
class ElementSource:
    """The element right-hand side inputs of ``tet_MakeElement_EM_E``
    (``lib/fem/make_elem_em.c:66-330``).  With gaps (``volt.dat`` first line
    dg > 0) every element with a vertex inside a gap box gets the delta-gap
    term and the antennas are ignored; without gaps (dg = 0) every element
    whose flag is an antenna flag gets the antenna current term."""

    gap_box: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 6)))  # x0 x1 y0 y1 z0 z1
    gap_volt: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    antenna_flag: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    antenna_Jo: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 0, 3)))   # (k, nv, 3)
    antenna_Jor: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 0, 3)))  # (k, nv, 3)

    @property
    def n_gaps(self) -> int:
        return int(self.gap_volt.shape[0])

    @property
    def n_antennas(self) -> int:
        return int(self.antenna_flag.shape[0])


@dataclasses.dataclass
class Model:
    """A synthetic full-wave model with one part and ``nsub`` subdomains."""

    name: str
    n: int
    size: float
    vertex_crd: np.ndarray  # (NV, 3) float64
    tets: np.ndarray  # (NT, 4) int32 vertex ids, positively oriented
    tet_edges: np.ndarray  # (NT, 6) int32 global edge ids, file order
    edges: np.ndarray  # (NE, 2) int32 (lo, hi) vertex ids
    flag: np.ndarray  # (NT,) int32 material flag per element
    mat_flag: np.ndarray  # (NF,) int32 flags of the material table (sorted)
    mat_eps: np.ndarray  # (NF,) float64 absolute permittivity [F/m]
    mat_sigma: np.ndarray  # (NF,) float64 conductivity [S/m]
    omega: float
    pec_edge: np.ndarray  # (NE,) bool, edges on the PEC outer wall
    sub_of_tet: np.ndarray  # (NT,) int32 subdomain id
    nsub: int
    # sources: list of right-hand sides; each is (edge ids (k,), values complex (k,))
    sources: List[Tuple[np.ndarray, np.ndarray]]
    # adjoint design problem: tets with their own flag (complex eps_r), probe edges
    design_tets: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    probe_edges: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    # element right-hand side (delta-gap voltages or antenna currents), or None
    element_source: Optional[ElementSource] = None
    # the Permittivity and Conductor lists as a model file gives them, when
    # they differ from the joint table above: (flags, values) each
    eps_table: Optional[Tuple[np.ndarray, np.ndarray]] = None
    sigma_table: Optional[Tuple[np.ndarray, np.ndarray]] = None
    # each subdomain's local vertex and edge order, as a model file gives it
    # (its node order): (vertex ptr, vertex ids, edge ptr, edge ids), or None
    # for ascending global id
    sub_order: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]] = None
    # vertex nodes of the Dirichlet (DirichletBCs_Axn0) lists, one flag per
    # vertex, or None: the full-wave problem ignores them, the correction-Jo
    # problem of an antenna holds its vertices there at zero
    pec_vertex: Optional[np.ndarray] = None

    @property
    def n_vertices(self) -> int:
        return int(self.vertex_crd.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])

    @property
    def n_edges(self) -> int:
        return int(self.edges.shape[0])


# --------------------------------------------------------------------------
# geometry


def _volume6(p: np.ndarray) -> np.ndarray:
    """6 x signed volume with the sign convention of ``tet_Volume6``
    (``lib/fem/tetrahedral.c:44-61``); ``p`` is (..., 4, 3)."""
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    return (
        -x[..., 0] * y[..., 1] * z[..., 2] + x[..., 0] * y[..., 1] * z[..., 3] + x[..., 0] * y[..., 2] * z[..., 1]
        - x[..., 0] * y[..., 2] * z[..., 3] - x[..., 0] * y[..., 3] * z[..., 1] + x[..., 0] * y[..., 3] * z[..., 2]
        + x[..., 1] * y[..., 0] * z[..., 2] - x[..., 1] * y[..., 0] * z[..., 3] - x[..., 1] * y[..., 2] * z[..., 0]
        + x[..., 1] * y[..., 2] * z[..., 3] + x[..., 1] * y[..., 3] * z[..., 0] - x[..., 1] * y[..., 3] * z[..., 2]
        - x[..., 2] * y[..., 0] * z[..., 1] + x[..., 2] * y[..., 0] * z[..., 3] + x[..., 2] * y[..., 1] * z[..., 0]
        - x[..., 2] * y[..., 1] * z[..., 3] - x[..., 2] * y[..., 3] * z[..., 0] + x[..., 2] * y[..., 3] * z[..., 1]
        + x[..., 3] * y[..., 0] * z[..., 1] - x[..., 3] * y[..., 0] * z[..., 2] - x[..., 3] * y[..., 1] * z[..., 0]
        + x[..., 3] * y[..., 1] * z[..., 2] + x[..., 3] * y[..., 2] * z[..., 0] - x[..., 3] * y[..., 2] * z[..., 1]
    )


def kuhn_mesh(n: int, size: float):
    """n^3 hexahedra, each split into 6 Kuhn tetrahedra sharing the cell's
    main diagonal.  Returns (vertex_crd, tets, cell_index_of_tet)."""
    h = size / n
    n1 = n + 1
    # vertex (i, j, k) -> i + (n+1)*(j + (n+1)*k); coordinates are exactly index*h
    K, J, I = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    crd = np.stack([I.ravel() * h, J.ravel() * h, K.ravel() * h], axis=1).astype(np.float64)
    # cell (i, j, k) -> i + n*(j + n*k)
    K, J, I = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ci_, cj_, ck_ = I.ravel(), J.ravel(), K.ravel()
    ncell = n ** 3

    def vid(a, b, c):
        return (a + n1 * (b + n1 * c)).astype(np.int64)

    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = np.empty((ncell, 6, 4), dtype=np.int64)
    for t, pm in enumerate(perms):
        off = np.zeros((4, 3), dtype=np.int64)
        off[1] = off[0]
        off[1][pm[0]] += 1
        off[2] = off[1]
        off[2][pm[1]] += 1
        off[3] = (1, 1, 1)
        for v in range(4):
            tets[:, t, v] = vid(ci_ + off[v][0], cj_ + off[v][1], ck_ + off[v][2])
    tets = tets.reshape(ncell * 6, 4)
    vol = _volume6(crd[tets])
    neg = vol < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    vol = _volume6(crd[tets])
    assert np.all(vol > 0), "Kuhn tetrahedra must be positively oriented"
    cell_of_tet = np.repeat(np.arange(ncell, dtype=np.int64), 6)
    return crd, tets.astype(np.int32), cell_of_tet, (ci_, cj_, ck_)


def edge_table(tets: np.ndarray, nv: int):
    """Unique edges sorted by (lo, hi) and each tetrahedron's 6 edge ids in
    file order 01, 02, 03, 12, 23, 13."""
    pairs = np.stack([np.stack([tets[:, a], tets[:, b]], axis=1) for a, b in FILE_EDGE_PAIRS], axis=1).astype(np.int64)
    lo = pairs.min(axis=2)
    hi = pairs.max(axis=2)
    key = lo * nv + hi
    ukey, inv = np.unique(key.ravel(), return_inverse=True)
    edges = np.stack([ukey // nv, ukey % nv], axis=1).astype(np.int32)
    return edges, inv.reshape(tets.shape[0], 6).astype(np.int32)


def pec_edges(edges: np.ndarray, crd: np.ndarray, size: float) -> np.ndarray:
    """An edge is on the PEC wall when one boundary plane holds both ends."""
    a = crd[edges[:, 0]]
    b = crd[edges[:, 1]]
    tol = 1e-9 * size
    on = np.zeros(edges.shape[0], dtype=bool)
    for ax in range(3):
        for val in (0.0, size):
            on |= (np.abs(a[:, ax] - val) < tol) & (np.abs(b[:, ax] - val) < tol)
    return on


# --------------------------------------------------------------------------
# partition


def rcb_partition(centroids: np.ndarray, leaf_cap: Optional[int] = None, nleaves: Optional[int] = None,
                  jitter: Optional[Tuple[float, float]] = None, seed: int = 0) -> np.ndarray:
    """Recursive coordinate bisection of element centroids.

    Each split takes the longest bounding-box axis of the segment's centroids
    (ties: lowest axis) and sends the elements with the smallest (coordinate,
    element id) to the first child.  The first child gets ``floor(r*N)``
    elements, ``r = 0.5`` (median split) or ``r ~ U[jitter]`` drawn from a
    seeded generator in depth-first order.  Splitting stops at ``nleaves``
    (power of two, balanced) or when a segment holds ``<= leaf_cap`` elements.
    Subdomains are numbered depth first, first child first.
    """
    nt = centroids.shape[0]
    ids = np.arange(nt)
    rank = np.empty((3, nt), dtype=np.int64)
    for ax in range(3):
        order = np.lexsort((ids, centroids[:, ax]))
        rank[ax, order] = np.arange(nt)
    rng = np.random.default_rng(seed)
    sub = np.empty(nt, dtype=np.int32)
    counter = [0]

    def rec(seg: np.ndarray, depth: int):
        n = seg.shape[0]
        stop = (nleaves is not None and (1 << depth) >= nleaves) or (leaf_cap is not None and n <= leaf_cap) or n < 2
        if stop:
            sub[seg] = counter[0]
            counter[0] += 1
            return
        c = centroids[seg]
        ext = c.max(axis=0) - c.min(axis=0)
        ax = int(np.argmax(ext))
        r = 0.5 if jitter is None else float(rng.uniform(jitter[0], jitter[1]))
        m = int(math.floor(r * n))
        m = max(1, min(n - 1, m))
        rk = rank[ax, seg]
        part = np.argpartition(rk, m - 1)
        left = seg[np.sort(part[:m])]
        right = seg[np.sort(part[m:])]
        rec(left, depth + 1)
        rec(right, depth + 1)

    rec(ids, 0)
    return sub


# --------------------------------------------------------------------------
# configurations


def _pml_depth(cidx: Tuple[np.ndarray, np.ndarray, np.ndarray], n: int, npml: int) -> np.ndarray:
    depth = np.zeros(cidx[0].shape[0], dtype=np.int64)
    for c in cidx:
        lo = np.where(c < npml, npml - c, 0)
        hi = np.where(c >= n - npml, c - (n - npml) + 1, 0)
        depth = np.maximum(depth, np.maximum(lo, hi))
    return depth


def pml_sigma(npml: int, h: float, reflection: float = 1e-6) -> np.ndarray:
    """Quadratic conductivity profile per PML depth k = 1..npml:
    sigma_k = sigma_max ((k - 1/2)/npml)^2 with
    sigma_max = -3 ln(R) / (2 eta0 d), d = npml h.  Index 0 (interior) is 0."""
    d = npml * h
    smax = -3.0 * math.log(reflection) / (2.0 * ETA0 * d)
    s = np.zeros(npml + 1)
    for k in range(1, npml + 1):
        s[k] = smax * ((k - 0.5) / npml) ** 2
    return s


def dipole_source(model_edges: np.ndarray, crd: np.ndarray, center: Sequence[float], nedges: int = 4,
                  value: complex = -1j) -> Tuple[np.ndarray, np.ndarray]:
    """Right-hand side ``value`` on the ``nedges`` z-directed edges whose
    midpoints are nearest ``center`` (ties: lower global edge id)."""
    a = crd[model_edges[:, 0]]
    b = crd[model_edges[:, 1]]
    d = b - a
    zdir = (np.abs(d[:, 0]) < 1e-12) & (np.abs(d[:, 1]) < 1e-12) & (np.abs(d[:, 2]) > 0)
    cand = np.nonzero(zdir)[0]
    mid = 0.5 * (a[cand] + b[cand])
    dist = np.sqrt(((mid - np.asarray(center)[None, :]) ** 2).sum(axis=1))
    order = np.lexsort((cand, np.round(dist, 12)))
    pick = np.sort(cand[order[:nedges]])
    return pick.astype(np.int32), np.full(pick.shape[0], value, dtype=np.complex128)


CONFIGS = {
    # name: (n, size, npml, nlayers, freq, partition, extras)
    "c1": dict(n=16, size=1.0, npml=4, layers=None, nleaves=64, leaf_cap=None, jitter=None),
    "c2": dict(n=48, size=1.5, npml=6, layers=8, nleaves=None, leaf_cap=600, jitter=(0.3, 0.7)),
    "c3": dict(n=96, size=1.5, npml=8, layers=8, nleaves=None, leaf_cap=900, jitter=(0.3, 0.7)),
    "c4": dict(n=48, size=1.5, npml=6, layers=8, nleaves=None, leaf_cap=600, jitter=(0.3, 0.7), design=12,
               nprobes=8),
    "c5": dict(n=112, size=1.5, npml=8, layers=8, nleaves=None, leaf_cap=1000, jitter=(0.3, 0.7),
               inclusions=0.05, nsources=16),
}


def design_material(eps_re: np.ndarray, eps_im: np.ndarray, omega: float):
    """Absolute permittivity and conductivity of a complex relative
    permittivity eps_r = eps' - i eps'': A_e = (nu/omega) RR - omega eps0 eps_r SS
    = (nu/omega) RR - (eps omega) SS + i sigma SS with eps = eps0 eps' and
    sigma = omega eps0 eps'' (the reference's convention, make_elem_em.c:230-265)."""
    return EPS0 * np.asarray(eps_re), omega * EPS0 * np.asarray(eps_im)


def make_model(name: str = "c1", n: Optional[int] = None, size: Optional[float] = None, npml: Optional[int] = None,
               layers: Optional[int] = "default", nleaves: Optional[int] = "default", leaf_cap: Optional[int] = "default",
               jitter="default", freq: float = 300e6, seed: int = 0, inclusions: float = 0.0,
               nsources: int = 1, design: int = 0, nprobes: int = 0) -> Model:
    """Build a named configuration (``c1``, ``c2``, ``c3``, ``c5``) or a
    custom one by overriding its fields.  Unknown names start from ``c1``."""
    base = dict(CONFIGS.get(name, CONFIGS["c1"]))
    if n is not None:
        base["n"] = n
    if size is not None:
        base["size"] = size
    if npml is not None:
        base["npml"] = npml
    if layers != "default":
        base["layers"] = layers
    if nleaves != "default":
        base["nleaves"] = nleaves
    if leaf_cap != "default":
        base["leaf_cap"] = leaf_cap
    if jitter != "default":
        base["jitter"] = jitter
    inclusions = base.get("inclusions", inclusions) if inclusions == 0.0 else inclusions
    nsources = base.get("nsources", nsources) if nsources == 1 else nsources
    design = base.get("design", design) if design == 0 else design
    nprobes = base.get("nprobes", nprobes) if nprobes == 0 else nprobes
    n_, L, npml_ = base["n"], base["size"], base["npml"]
    rng = np.random.default_rng(seed)
    crd, tets, cell_of_tet, cidx = kuhn_mesh(n_, L)
    nv = crd.shape[0]
    edges, tet_edges = edge_table(tets, nv)
    h = L / n_
    depth = _pml_depth(cidx, n_, npml_)[cell_of_tet]
    nl = base["layers"] or 1
    if base["layers"]:
        eps_r = rng.uniform(1.0, 10.0, size=nl)
        sig_l = rng.uniform(0.0, 0.01, size=nl)
    else:
        eps_r = np.ones(1)
        sig_l = np.zeros(1)
    kz = cidx[2][cell_of_tet]
    layer = np.minimum(nl - 1, (kz * nl) // n_)
    flag = layer * (npml_ + 1) + depth
    spml = pml_sigma(npml_, h)
    mat_flag = list(range(nl * (npml_ + 1)))
    mat_eps = [EPS0 * eps_r[f // (npml_ + 1)] for f in mat_flag]
    mat_sigma = [sig_l[f // (npml_ + 1)] + spml[f % (npml_ + 1)] for f in mat_flag]
    if inclusions > 0.0:
        nt = tets.shape[0]
        pick = rng.random(nt) < inclusions
        pick &= depth == 0
        inc_ids = np.nonzero(pick)[0]
        epsr_inc = rng.uniform(10.0, 20.0, size=inc_ids.shape[0])
        base_flag = len(mat_flag)
        flag = flag.copy()
        for k, t in enumerate(inc_ids):
            flag[t] = base_flag + k
            mat_flag.append(base_flag + k)
            mat_eps.append(EPS0 * epsr_inc[k])
            mat_sigma.append(sig_l[layer[t]])
    design_tets = np.zeros(0, np.int32)
    omega = 2.0 * math.pi * freq
    if design > 0:
        # central design^3 cells, each tet with its own flag and complex eps_r
        lo_c = (n_ - design) // 2
        cc = np.stack([c[cell_of_tet] for c in cidx], axis=1)
        inside = np.all((cc >= lo_c) & (cc < lo_c + design), axis=1)
        design_tets = np.nonzero(inside)[0].astype(np.int32)
        drng = np.random.default_rng(seed + 101)
        er = drng.uniform(2.0, 4.0, size=design_tets.shape[0])
        ei = drng.uniform(0.0, 0.1, size=design_tets.shape[0])
        de, ds = design_material(er, ei, omega)
        base_flag = len(mat_flag)
        flag = flag.copy()
        for k, t in enumerate(design_tets):
            flag[t] = base_flag + k
            mat_flag.append(base_flag + k)
            mat_eps.append(de[k])
            mat_sigma.append(ds[k])
    centroids = crd[tets].mean(axis=1)
    sub = rcb_partition(centroids, leaf_cap=base["leaf_cap"], nleaves=base["nleaves"], jitter=base["jitter"],
                        seed=seed + 1)
    nsub = int(sub.max()) + 1
    sources = []
    c0 = np.full(3, 0.5 * L)
    sources.append(dipole_source(edges, crd, c0))
    if nsources > 1:
        lo = (npml_ + 2) * h
        hi = L - (npml_ + 2) * h
        for s in range(1, nsources):
            sources.append(dipole_source(edges, crd, rng.uniform(lo, hi, size=3)))
    probe_edges = np.zeros(0, np.int32)
    if nprobes > 0:
        # seeded interior edges outside the PML and outside the design box
        prng = np.random.default_rng(seed + 202)
        mid = 0.5 * (crd[edges[:, 0]] + crd[edges[:, 1]])
        lo_x, hi_x = (npml_ + 0.5) * h, L - (npml_ + 0.5) * h
        ok = np.all((mid > lo_x) & (mid < hi_x), axis=1)
        if design > 0:
            dlo = ((n_ - design) // 2) * h
            dhi = ((n_ - design) // 2 + design) * h
            ok &= ~np.all((mid >= dlo) & (mid <= dhi), axis=1)
        cand = np.nonzero(ok)[0]
        probe_edges = np.sort(prng.choice(cand, size=min(nprobes, cand.shape[0]), replace=False)).astype(np.int32)
    model = Model(
        name=name, n=n_, size=L, vertex_crd=crd, tets=tets, tet_edges=tet_edges, edges=edges,
        flag=flag.astype(np.int32), mat_flag=np.asarray(mat_flag, dtype=np.int32),
        mat_eps=np.asarray(mat_eps, dtype=np.float64), mat_sigma=np.asarray(mat_sigma, dtype=np.float64),
        omega=omega, pec_edge=pec_edges(edges, crd, L), sub_of_tet=sub, nsub=nsub, sources=sources,
        design_tets=design_tets, probe_edges=probe_edges)
    return model


def add_region(model: Model, lo: Sequence[float], hi: Sequence[float], eps: float, sigma: float) -> int:
    """Give the elements whose centroid lies in the box [lo, hi] a new
    material flag (appended to the table, which stays sorted) and return it."""
    cen = model.vertex_crd[model.tets].mean(axis=1)
    inside = np.all((cen >= np.asarray(lo)) & (cen <= np.asarray(hi)), axis=1)
    if not inside.any():
        raise ValueError("no element centroid in the box")
    f = int(model.mat_flag.max()) + 1
    model.flag = np.where(inside, f, model.flag).astype(np.int32)
    model.mat_flag = np.append(model.mat_flag, f).astype(np.int32)
    model.mat_eps = np.append(model.mat_eps, eps)
    model.mat_sigma = np.append(model.mat_sigma, sigma)
    return f


def delta_gap_source(model: Model, boxes, volts) -> ElementSource:
    """Delta-gap voltages (``volt.dat`` with dg > 0): gap k drives the
    vertices inside ``boxes[k]`` = (x0, x1, y0, y1, z0, z1) with ``volts[k]``;
    it acts through the conductivity of the elements that touch them."""
    es = ElementSource(gap_box=np.asarray(boxes, np.float64).reshape(-1, 6),
                       gap_volt=np.asarray(volts, np.float64).ravel())
    model.element_source = es
    return es


def antenna_source(model: Model, flags, jo, jor) -> ElementSource:
    """Antenna currents (``volt.dat`` dg = 0): antenna k acts on the
    elements of flag ``flags[k]`` with the vertex current arrays ``jo[k]``,
    ``jor[k]`` of shape (n_vertices, 3) (the reference's ``antenna.Jo`` and
    ``antenna.Jor`` at each vertex)."""
    nv = model.n_vertices
    es = ElementSource(antenna_flag=np.asarray(flags, np.int32).ravel(),
                       antenna_Jo=np.asarray(jo, np.float64).reshape(-1, nv, 3),
                       antenna_Jor=np.asarray(jor, np.float64).reshape(-1, nv, 3))
    model.element_source = es
    return es


def _g17(v: float) -> str:
    return f"{v:.17e}"


def canonical_material_text(model: Model) -> str:
    """The reference's ``mtrl.dat`` (``lib/std/fileio.c:3474-3572``), with
    values printed to round-trip exactly."""
    lines = [f"Permittivity {len(model.mat_flag)}"]
    lines += [f"{f} {e:.17e}" for f, e in zip(model.mat_flag, model.mat_eps)]
    lines.append("")
    lines.append(f"Conductor {len(model.mat_flag)}")
    lines += [f"{f} {s:.17e}" for f, s in zip(model.mat_flag, model.mat_sigma)]
    lines.append("")
    lines.append("AntennaOmega")
    lines.append(f"{model.omega:.17e}")
    return "\n".join(lines) + "\n"


def round_trip_material(model: Model) -> None:
    """Replace the material values by their printed-and-parsed doubles so the
    values this package uses are bit-identical to what the reference reads."""
    txt = canonical_material_text(model)
    toks = txt.split()
    nf = len(model.mat_flag)
    i = 2
    eps = []
    for _ in range(nf):
        eps.append(float(toks[i + 1]))
        i += 2
    i += 2
    sig = []
    for _ in range(nf):
        sig.append(float(toks[i + 1]))
        i += 2
    model.mat_eps = np.asarray(eps)
    model.mat_sigma = np.asarray(sig)
    model.omega = float(toks[i + 1])


# --------------------------------------------------------------------------
# ADVENTURE HDDM part file (the reference's model input)


def _advdoc(did: str, props: Sequence[Tuple[str, str]], payload: bytes) -> bytes:
    h = bytearray()
    h += struct.pack("<i", len(did)) + did.encode()
    h += struct.pack("<i", len(props))
    for k, v in props:
        h += struct.pack("<i", len(k)) + k.encode()
        h += struct.pack("<i", len(v)) + v.encode()
    return b"AdvDoc\0" + struct.pack("<q", len(payload)) + payload + struct.pack("<q", len(h)) + bytes(h)


def subdomain_views(model: Model):
    """Per subdomain: element ids (ascending), node global ids (ascending,
    vertices then mid-nodes by construction of the numbering), and the
    element node lists in subdomain-local node ids (file order)."""
    nv = model.n_vertices
    order = np.argsort(model.sub_of_tet, kind="stable")
    counts = np.bincount(model.sub_of_tet, minlength=model.nsub)
    starts = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for s in range(model.nsub):
        els = order[starts[s]:starts[s + 1]]
        nodes10 = np.concatenate([model.tets[els], model.tet_edges[els] + nv], axis=1).astype(np.int64)
        gn, inv = np.unique(nodes10.ravel(), return_inverse=True)
        out.append((els, gn, inv.reshape(-1, 10).astype(np.int32)))
    return out


def write_hddm_model(model: Model, directory: str, source_index: Optional[int] = None) -> str:
    """Write ``<directory>/model/advhddm_in_0.adv``, ``<directory>/mtrl.dat``,
    ``<directory>/volt.dat`` (``0``: current input, or the delta-gap
    definitions; ``make_elem_em.c:74-96,332-346``), ``<directory>/source.txt``
    (the edge right-hand sides) and, for antenna currents,
    ``<directory>/antenna.txt`` (both consumed by the oracle harness)."""
    os.makedirs(os.path.join(directory, "model"), exist_ok=True)
    nv = model.n_vertices
    nnd = nv + model.n_edges
    views = subdomain_views(model)
    # part-level interface nodes: nodes shared by >= 2 subdomains
    cnt = np.zeros(nnd, dtype=np.int32)
    for els, gn, _ in views:
        cnt[gn] += 1
    iface = np.nonzero(cnt >= 2)[0]
    ln_of = np.full(nnd, -1, dtype=np.int64)
    ln_of[iface] = np.arange(iface.shape[0])
    pec_node = np.zeros(nnd, dtype=bool)
    pec_node[nv + np.nonzero(model.pec_edge)[0]] = True
    if getattr(model, "pec_vertex", None) is not None:
        pec_node[:nv] = np.asarray(model.pec_vertex, bool)
    tag = "HDDM_Part[0]:0:5EED0000"
    docs = []
    mid_crd = 0.5 * (model.vertex_crd[model.edges[:, 0]] + model.vertex_crd[model.edges[:, 1]])
    crd_all = np.concatenate([model.vertex_crd, mid_crd], axis=0)
    docs.append(_advdoc("00000001:Node@" + tag,
                        [("dimension", "3"), ("num_items_orig", str(nnd)), ("num_items", str(nnd)),
                         ("content_type", "Node")], crd_all.astype("<f8").tobytes()))
    docs.append(_advdoc("00000002:NodeIndex_PartToGlobal@" + tag,
                        [("index_byte", "4"), ("label", "NodeIndex_PartToGlobal"), ("format", "i4"),
                         ("fega_type", "AllNodeVariable"), ("num_items_orig", str(nnd)), ("num_items", str(nnd)),
                         ("content_type", "FEGenericAttribute")], np.arange(nnd, dtype="<i4").tobytes()))
    docs.append(_advdoc("00000003:HDDM_InterfaceDOF@" + tag,
                        [("total_num_midfree", "0"), ("total_num_outfree", "0"),
                         ("total_num_infree", str(iface.shape[0])), ("num_outdom", "0"), ("part_number", "0"),
                         ("num_subdomains", str(model.nsub)), ("dimension", "1"), ("num_parts", "1"),
                         ("content_type", "HDDM_InterfaceDOF")], struct.pack("<i", 0)))
    el_pay, nd_pay, if_pay, bc_pay, fl_pay, ge_pay = (bytearray() for _ in range(6))
    nif_total = 0
    nbc_total = 0
    for els, gn, lnop in views:
        el_pay += struct.pack("<i", els.shape[0]) + lnop.astype("<i4").tobytes()
        nd_pay += struct.pack("<i", gn.shape[0]) + gn.astype("<i4").tobytes()
        loc_if = np.nonzero(cnt[gn] >= 2)[0]
        rec = np.zeros((loc_if.shape[0], 5), dtype="<i4")
        rec[:, 0] = loc_if
        rec[:, 3] = ln_of[gn[loc_if]]
        rec[:, 4] = ln_of[gn[loc_if]]
        if_pay += struct.pack("<i", loc_if.shape[0]) + rec.tobytes()
        nif_total += loc_if.shape[0]
        loc_bc = np.nonzero(pec_node[gn])[0].astype("<i4")
        bc_pay += struct.pack("<i", loc_bc.shape[0]) + loc_bc.tobytes()
        nbc_total += loc_bc.shape[0]
        fl_pay += struct.pack("<i", els.shape[0]) + model.flag[els].astype("<i4").tobytes()
        ge_pay += struct.pack("<i", els.shape[0]) + els.astype("<i4").tobytes()
    nt = model.n_tets
    docs.append(_advdoc("00000004:HDDM_Element@" + tag,
                        [("num_items_orig", str(nt)), ("sum_items", str(nt)), ("dimension", "3"),
                         ("num_nodes_per_element", "10"), ("element_type", "3DQuadraticTetrahedron"),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_Element")], bytes(el_pay)))
    docs.append(_advdoc("00000005:HDDM_NodeIndex@" + tag,
                        [("index_byte", "4"), ("label", "NodeIndex_SubdomainToPart"), ("format", "i4"),
                         ("fega_type", "AllNodeVariable"), ("num_items_orig", str(nnd)),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_FEGenericAttribute")],
                        bytes(nd_pay)))
    docs.append(_advdoc("00000006:InterfaceDOF@" + tag,
                        [("sum_items", str(nif_total)), ("ifd_dimension", "1"), ("index_byte", "4"),
                         ("label", "InterfaceDOF"), ("format", "i4i4i4i4"), ("fega_type", "NodeVariable"),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_FEGenericAttribute")],
                        bytes(if_pay)))
    docs.append(_advdoc("00000007:HDDM_FEGA@" + tag,
                        [("sum_items", str(nbc_total)), ("index_byte", "4"), ("label", "DirichletBCs_Axn0"),
                         ("format", "i4"), ("fega_type", "NodeConstant"), ("num_items_orig", str(nbc_total)),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_FEGenericAttribute")],
                        bytes(bc_pay)))
    docs.append(_advdoc("00000008:HDDM_FEGA@" + tag,
                        [("sum_items", str(nt)), ("index_byte", "4"), ("label", "Flag"), ("format", "i4"),
                         ("fega_type", "AllElementVariable"), ("num_items_orig", str(nt)),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_FEGenericAttribute")],
                        bytes(fl_pay)))
    docs.append(_advdoc("00000009:HDDM_FEGA@" + tag,
                        [("sum_items", "1"), ("DirichletBCs_Axn0", "NEED"), ("N_VERSION", "1"),
                         ("ADVFW_NAME", "ADVENTURE_FullWave"), ("index_byte", "4"), ("label", "Options"),
                         ("format", ""), ("fega_type", "AllElementConstant"), ("num_items_orig", "0"),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_FEGenericAttribute")], b""))
    docs.append(_advdoc("0000000A:HDDM_FEGA@" + tag,
                        [("sum_items", str(nt)), ("index_byte", "4"), ("label", "ElementIndex_SubdomainToGlobal"),
                         ("format", "i4"), ("fega_type", "AllElementVariable"), ("num_items_orig", str(nt)),
                         ("num_subdomains", str(model.nsub)), ("content_type", "HDDM_FEGenericAttribute")],
                        bytes(ge_pay)))
    path = os.path.join(directory, "model", "advhddm_in_0.adv")
    with open(path, "wb") as f:
        for d in docs:
            f.write(d)
    with open(os.path.join(directory, "mtrl.dat"), "w") as f:
        f.write(canonical_material_text(model))
    es = model.element_source
    with open(os.path.join(directory, "volt.dat"), "w") as f:
        # make_elem_em.c:96 reads dg, :332-346 four lines per gap
        if es is not None and es.n_gaps > 0:
            f.write(f"{es.n_gaps}\n")
            for box, dv in zip(es.gap_box, es.gap_volt):
                f.write(f"{_g17(box[0])} {_g17(box[1])}\n{_g17(box[2])} {_g17(box[3])}\n"
                        f"{_g17(box[4])} {_g17(box[5])}\n{_g17(dv)}\n")
        else:
            f.write("0\n")
    # antenna currents per vertex, read by the oracle harness
    if es is not None and es.n_antennas > 0:
        with open(os.path.join(directory, "antenna.txt"), "w") as f:
            f.write(f"{es.n_antennas} {nv}\n")
            for k in range(es.n_antennas):
                f.write(f"{int(es.antenna_flag[k])}\n")
                for v in range(nv):
                    f.write(" ".join(_g17(a) for a in es.antenna_Jo[k, v]) + " " +
                            " ".join(_g17(a) for a in es.antenna_Jor[k, v]) + "\n")
    srcs = model.sources if source_index is None else [model.sources[source_index]]
    with open(os.path.join(directory, "source.txt"), "w") as f:
        f.write(f"{len(srcs)}\n")
        for e, v in srcs:
            f.write(f"{len(e)}\n")
            for ei, vi in zip(e, v):
                f.write(f"{nv + int(ei)} {vi.real:.17e} {vi.imag:.17e}\n")
    return path
