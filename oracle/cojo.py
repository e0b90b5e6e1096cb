"""CPU oracle of the correction-Jo pre-solve of an antenna.

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the CUDA path;
the product never imports it.

main() runs, for every antenna and before the full-wave solve, two
real-symmetric HDDM solves (``main/fullwave/main.c:92-98``:
``hddm_solver_RS`` with ``set_hddm_func_correct_Jor`` and then
``set_hddm_func_correct_Joi``, ``lib/hddm/set_hddm_func.c:90-233``).  This
module restates them in numpy:

* ``partition``: the antenna's integer setup of ``make_PartMesh_FW`` --
  the DOFs of a subdomain are the vertices of its antenna elements in its
  vertex order (``make_PartMesh_make_ANTENNA_make_enf``,
  ``lib/hddm/make_PartMesh.c:973-983``), interface DOFs the antenna vertices
  two or more subdomains hold (``make_PartMesh_FW_change_innerbc_ANTENNA``
  with its ``make_nf``, ``:1288-1340,1546-1575``) that are on no Dirichlet
  list (``:393-421``), the Dirichlet list the
  sorted PEC DOFs then the interface DOFs, or DOF 0 alone when a subdomain
  has neither (``make_PartMesh_make_ANTENNA_change_bc`` / ``_add_inbc``,
  ``:986-1063``);
* ``element_matrices`` / ``element_rhs``: ``tet_MakeElement_correct_Jo``
  (``lib/fem/make_elem.c:10-66``) with ``tet_simple_b/c/d``,
  ``tet_simple_gradgrad`` and ``tet_simple_be_apgrad``
  (``lib/fem/tetrahedral.c:122-220``) in the reference's operation order;
* ``hddm``: the s-mode HDDM loop of the reference's template in real
  arithmetic (``lib/hddm/hddm_solver.h:295-450``, ``hddm_solver_s.h:158-400``,
  the diagonal preconditioner ``hddm_pc.h:52-137``), sums taken in the
  reference's order.  One deviation: each subdomain system is solved
  directly (Cholesky) where the reference runs CG with an incomplete
  Cholesky preconditioner to a relative residual of 1e-12
  (``mymt_RS_AIJ_Solver_CG``, ``lib/mymt_aij_solver/aij_solver_cg.h``), so
  results agree with the reference's to that tolerance, not bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import scipy.linalg

NEARLY_ZERO = 1.0e-60  # lib/std/defs.h:105
TET_M = np.array([[0, 1, 2, 3], [1, 3, 2, 0], [2, 3, 0, 1], [3, 1, 0, 2]])  # lib/fem/tetrahedral.h:14-17


@dataclass
class CojoSub:
    sub: int               # original subdomain id
    els: np.ndarray        # antenna elements, ascending global id
    gid: np.ndarray        # global vertex of each DOF (enf order)
    dof: np.ndarray        # (nel, 4) local DOF of each element vertex
    ibc: np.ndarray        # Dirichlet list
    inbc_nfid: np.ndarray  # interface DOFs, ascending local id
    inbc_ln: np.ndarray    # their interface numbers
    pinned: bool           # DOF 0 held at zero (no PEC and no interface DOF)


@dataclass
class CojoPartition:
    subs: List[CojoSub]
    tfree: int
    iface_gid: np.ndarray


def partition(model, antenna_flag: int, pec_vertex: Optional[np.ndarray] = None) -> CojoPartition:
    nv = model.n_vertices
    if pec_vertex is None:
        pec_vertex = getattr(model, "pec_vertex", None)
    order = np.argsort(model.sub_of_tet, kind="stable")
    counts = np.bincount(model.sub_of_tet, minlength=model.nsub)
    starts = np.concatenate([[0], np.cumsum(counts)])
    so = getattr(model, "sub_order", None)
    per = []
    held = np.zeros(nv, np.int64)
    for s in range(model.nsub):
        els = order[starts[s]:starts[s + 1]]
        els = els[model.flag[els] == antenna_flag]
        if els.shape[0] == 0:
            continue
        v = np.unique(model.tets[els])
        if so is not None:
            # the subdomain's own vertex order (its part file's node order)
            vord = np.asarray(so[1][so[0][s]:so[0][s + 1]])
            v = vord[np.isin(vord, v)]
        held[v] += 1
        per.append((s, els, v))
    # vertices on a Dirichlet list stay out of the interface (the pass that
    # excludes essential BCs, make_PartMesh.c:393-421)
    pec = np.zeros(nv, bool) if pec_vertex is None else np.asarray(pec_vertex, bool)
    iface_gid = np.nonzero((held >= 2) & ~pec)[0]
    ln_of = np.full(nv, -1, np.int64)
    ln_of[iface_gid] = np.arange(iface_gid.shape[0])
    subs = []
    for s, els, v in per:
        loc = np.full(nv, -1, np.int64)
        loc[v] = np.arange(v.shape[0])
        pec_l = np.nonzero(pec_vertex[v])[0] if pec_vertex is not None else np.zeros(0, np.int64)
        if_l = np.nonzero(ln_of[v] >= 0)[0]
        pinned = pec_l.shape[0] == 0 and if_l.shape[0] == 0
        ibc = np.array([0]) if pinned else np.concatenate([pec_l, if_l])
        subs.append(CojoSub(sub=s, els=els, gid=v, dof=loc[model.tets[els]], ibc=ibc.astype(np.int64),
                            inbc_nfid=if_l, inbc_ln=ln_of[v[if_l]], pinned=pinned))
    return CojoPartition(subs=subs, tfree=int(iface_gid.shape[0]), iface_gid=iface_gid)


def _bcd(xyz: np.ndarray):
    """tet_simple_b/c/d for every element: xyz (n, 4, 3) -> b, c, d (n, 4)."""
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    out = []
    for a, p, q in ((y, z, None), (z, x, None), (x, y, None)):
        cols = []
        for i in range(4):
            ii, jj, kk = TET_M[i, 1], TET_M[i, 2], TET_M[i, 3]
            t = a[:, ii] * (p[:, jj] - p[:, kk]) + a[:, jj] * (p[:, kk] - p[:, ii])
            t = t + a[:, kk] * (p[:, ii] - p[:, jj])
            cols.append(-1.0 * t)
        out.append(np.stack(cols, 1))
    return out


def _volume6(xyz: np.ndarray) -> np.ndarray:
    """tet_Volume6 (lib/fem/tetrahedral.c:44-61), term by term."""
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    terms = [(-1, 0, 1, 2), (1, 0, 1, 3), (1, 0, 2, 1), (-1, 0, 2, 3), (-1, 0, 3, 1), (1, 0, 3, 2),
             (1, 1, 0, 2), (-1, 1, 0, 3), (-1, 1, 2, 0), (1, 1, 2, 3), (1, 1, 3, 0), (-1, 1, 3, 2),
             (-1, 2, 0, 1), (1, 2, 0, 3), (1, 2, 1, 0), (-1, 2, 1, 3), (-1, 2, 3, 0), (1, 2, 3, 1),
             (1, 3, 0, 1), (-1, 3, 0, 2), (-1, 3, 1, 0), (1, 3, 1, 2), (1, 3, 2, 0), (-1, 3, 2, 1)]
    sg, i, j, k = terms[0]
    D = -(x[:, i] * y[:, j] * z[:, k])
    for sg, i, j, k in terms[1:]:
        t = x[:, i] * y[:, j] * z[:, k]
        D = D + t if sg > 0 else D - t
    return D


def element_matrices(model, els: np.ndarray) -> np.ndarray:
    """(grad N_i, grad N_j) of each element (tet_simple_gradgrad): (n, 4, 4)."""
    xyz = model.vertex_crd[model.tets[els]]
    b, c, d = _bcd(xyz)
    dd = 1.0 / (6.0 * _volume6(xyz))
    gg = b[:, :, None] * b[:, None, :] + c[:, :, None] * c[:, None, :]
    gg = gg + d[:, :, None] * d[:, None, :]
    return gg * dd[:, None, None]


def element_rhs(model, els: np.ndarray, current: np.ndarray) -> np.ndarray:
    """(J, grad N_i) of each element (tet_simple_be_apgrad): (n, 4)."""
    xyz = model.vertex_crd[model.tets[els]]
    b, c, d = _bcd(xyz)
    u = current[model.tets[els]]  # (n, 4 vertices, 3)
    dd = 1.0 / 24.0
    ag = np.zeros(b.shape)
    for j in range(4):
        t = b * u[:, j, 0][:, None] + c * u[:, j, 1][:, None]
        t = t + d * u[:, j, 2][:, None]
        ag = ag + t * dd
    return ag


def _seq_sum(v: np.ndarray) -> float:
    acc = 0.0
    for t in v.tolist():
        acc += t
    return acc


class _Sub:
    """One subdomain's assembled system (the matrix summed in element order,
    SetAe/SetFe, aij_matrix_func.h:260-338) and its factor."""

    def __init__(self, model, sb: CojoSub, current: np.ndarray):
        n = sb.gid.shape[0]
        A = np.zeros((n, n))
        bvec = np.zeros(n)
        gg = element_matrices(model, sb.els)
        be = element_rhs(model, sb.els, current)
        for k in range(sb.els.shape[0]):
            d = sb.dof[k]
            for i in range(4):
                bvec[d[i]] += be[k, i]
                for j in range(4):
                    if d[i] >= d[j]:
                        A[d[i], d[j]] += gg[k, i, j]
        self.A = np.tril(A) + np.tril(A, -1).T
        self.b = bvec
        isbc = np.zeros(n, bool)
        isbc[sb.ibc] = True
        self.I = np.nonzero(~isbc)[0]
        self.sb = sb
        self.fac = scipy.linalg.cho_factor(self.A[np.ix_(self.I, self.I)]) if self.I.shape[0] else None

    def solve(self, vbc_iface: np.ndarray, with_b: bool) -> np.ndarray:
        """solve_dom*: Dirichlet values (0 at PEC / pinned DOFs, vbc_iface at
        the interface DOFs), the interior solved; returns the whole x."""
        n = self.A.shape[0]
        x = np.zeros(n)
        x[self.sb.inbc_nfid] = vbc_iface
        if self.I.shape[0]:
            rhs = (self.b[self.I] if with_b else 0.0) - self.A[np.ix_(self.I, np.arange(n))] @ x
            x[self.I] = scipy.linalg.cho_solve(self.fac, rhs)
        return x

    def vec(self, x: np.ndarray, with_b: bool) -> np.ndarray:
        """vec = A x (- b) at the interface DOFs (MxV_TMP_AIJ)."""
        r = self.A[self.sb.inbc_nfid] @ x
        return r - self.b[self.sb.inbc_nfid] if with_b else r


def hddm(model, part: CojoPartition, current: np.ndarray, hddm_eps: float = 1e-10, hddm_max_loop: int = 4000):
    """One pass of the pre-solve with vertex currents ``current`` (nv, 3).
    Returns (potential per global vertex, per-subdomain solutions,
    residual history, initial norm)."""
    subs = [_Sub(model, sb, np.asarray(current, np.float64)) for sb in part.subs]
    tf = part.tfree
    Q = np.zeros(tf)
    PC = np.zeros(tf)
    for s in subs:
        x = s.solve(np.zeros(s.sb.inbc_nfid.shape[0]), True)
        v = s.vec(x, True)
        for i, ln in enumerate(s.sb.inbc_ln.tolist()):
            Q[ln] += v[i]
            dg = s.A[s.sb.inbc_nfid[i], s.sb.inbc_nfid[i]]
            PC[ln] += dg if dg != 0.0 else 1.0
    PC = np.where(PC != 0.0, 1.0 / np.where(PC != 0.0, PC, 1.0), 1.0)
    R = Q.copy()
    Z = R * PC
    P = Z.copy()
    U = np.zeros(tf)
    resi = float(np.max(np.abs(R))) if tf else 0.0
    norm0 = resi
    last = resi < NEARLY_ZERO
    r0 = 1.0 / resi if resi != 0.0 else np.inf
    rz = _seq_sum(R * Z)
    hist = []
    loop = 1
    while not last:
        Q = np.zeros(tf)
        for s in subs:
            x = s.solve(P[s.sb.inbc_ln], False)
            v = s.vec(x, False)
            for i, ln in enumerate(s.sb.inbc_ln.tolist()):
                Q[ln] += v[i]
        pq = _seq_sum(P * Q)
        malpha = 0.0 if (abs(rz) < NEARLY_ZERO and abs(pq) < NEARLY_ZERO) else 0.0 - rz / pq
        U = U + malpha * P
        R = R + malpha * Q
        resi = float(np.max(np.abs(R))) * r0
        hist.append(resi)
        Z = R * PC
        rzn = _seq_sum(R * Z)
        beta = 0.0 if (abs(rzn) < NEARLY_ZERO and abs(rz) < NEARLY_ZERO) else rzn / rz
        rz = rzn
        P = Z + beta * P
        if resi < hddm_eps:
            last = True
            P = U.copy()
        if loop == hddm_max_loop:
            last = True
        loop += 1
    phi = np.zeros(model.n_vertices)
    seen = np.zeros(model.n_vertices, bool)
    per_sub = []
    for s in subs:
        x = s.solve(P[s.sb.inbc_ln], True)
        per_sub.append(x)
        new = ~seen[s.sb.gid]
        phi[s.sb.gid[new]] = x[new]
        seen[s.sb.gid] = True
    return phi, per_sub, np.array(hist), norm0
