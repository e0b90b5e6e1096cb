"""CPU backend of one shard of the sharded HDDM solve, for the multi-process
(gloo) tests of ``adventure_fullwave_b200.shard``.  Test infrastructure only.

Each owned subdomain is the oracle's assembled system (``oracle.assemble_sub``,
the reference's TMP_AIJ rows) solved densely after Dirichlet elimination
(SetBC, ``aij_matrix_func.h:60-136``); the COCG is the same recurrence as the
library's kernels (``ITERATION_S_1ST`` / ``ITERATION_S``,
``lib/hddm/hddm_solver_s.h:158-400``), replicated on every rank from the
summed partial vectors, as the library runs it.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import torch

from oracle import oracle

NEARLY_ZERO = 1.0e-60


class _Sub:
    def __init__(self, model, sd):
        rp, col, val, b = oracle.assemble_sub(model, sd)
        n = sd.edge_gid.shape[0]
        a = np.zeros((n, n), dtype=np.complex128)
        for r in range(n):
            for q in range(rp[r], rp[r + 1]):
                a[r, col[q]] = val[q]
                a[col[q], r] = val[q]
        self.a = a
        self.b = b
        bc = np.zeros(n, dtype=bool)
        bc[sd.ibc] = True
        self.interior = np.nonzero(~bc)[0]
        self.iface = np.asarray(sd.inbc_nfid, dtype=np.int64)
        self.ln = np.asarray(sd.inbc_ln, dtype=np.int64)
        self.edge_gid = sd.edge_gid
        ii = self.interior
        self.lu = sla.lu_factor(a[np.ix_(ii, ii)]) if ii.size else None
        self.a_ig = a[np.ix_(ii, self.iface)]
        self.a_gi = a[np.ix_(self.iface, ii)]
        self.a_gg = a[np.ix_(self.iface, self.iface)]
        self.diag_g = np.diag(a)[self.iface]

    def solve_interior(self, rhs):
        return sla.lu_solve(self.lu, rhs) if self.lu is not None else rhs

    def first_q(self):
        x_i = self.solve_interior(self.b[self.interior])
        return self.a_gi @ x_i - self.b[self.iface]

    def iter_q(self, v):
        x_i = self.solve_interior(-(self.a_ig @ v))
        return self.a_gi @ x_i + self.a_gg @ v

    def last_x(self, v):
        x = np.zeros(self.a.shape[0], dtype=np.complex128)
        x[self.interior] = self.solve_interior(self.b[self.interior] - self.a_ig @ v)
        x[self.iface] = v
        return x


class CpuShard:
    """The backend protocol of ``adventure_fullwave_b200.shard.run_sharded``
    on the CPU, for the subdomains [lo, hi) of ``model``."""

    def __init__(self, model, shard, hddm_eps=1e-10, hddm_max_loop=5000):
        self.model = model
        self.lo, self.hi = shard
        self.eps = hddm_eps
        self.max_loop = hddm_max_loop
        self.subs = []
        self.nfree = 0
        self.buffer = None
        self.q_buffer = None

    def sync(self) -> None:
        pass

    def make_tmp_aij(self, source) -> None:
        part = oracle.partition(self.model, source)
        self.nfree = part.tfree
        self.owner = np.full(self.model.n_edges, -1, dtype=np.int64)
        for s in range(len(part.subs) - 1, -1, -1):
            self.owner[part.subs[s].edge_gid] = s
        self.subs = [(s, _Sub(self.model, part.subs[s])) for s in range(self.lo, self.hi)]
        self.buffer = torch.zeros(4 * max(1, self.nfree), dtype=torch.float64)
        self.q_buffer = self.buffer[: 2 * max(1, self.nfree)]

    def _put(self, view, vec):
        v = view.numpy()
        v[0::2] = vec.real
        v[1::2] = vec.imag

    def _get(self, view):
        v = view.numpy()
        return v[0::2] + 1j * v[1::2]

    def first(self) -> None:
        q = np.zeros(self.nfree, dtype=np.complex128)
        pc = np.zeros(self.nfree, dtype=np.complex128)
        for _, sd in self.subs:
            np.add.at(q, sd.ln, sd.first_q())
            np.add.at(pc, sd.ln, sd.diag_g)
        self._put(self.buffer[: 2 * self.nfree], q)
        self._put(self.buffer[2 * self.nfree: 4 * self.nfree], pc)

    def first_finish(self) -> int:
        q = self._get(self.buffer[: 2 * self.nfree])
        pcs = self._get(self.buffer[2 * self.nfree: 4 * self.nfree])
        self.pc = np.where(pcs == 0, 1.0 + 0j, 1.0 / np.where(pcs == 0, 1.0, pcs))
        self.r = q.copy()
        self.z = self.r * self.pc
        self.p = self.z.copy()
        self.u = np.zeros_like(q)
        self.norm0 = float(np.max(np.abs(q))) if q.size else 0.0
        self.rz = np.sum(self.r * self.z)
        self.loop = 1
        self.status = 1 if self.norm0 < NEARLY_ZERO else 0
        if self.status:
            self.p = self.u.copy()
            self.status = 2
        return self.status

    def iterate(self) -> None:
        q = np.zeros(self.nfree, dtype=np.complex128)
        for _, sd in self.subs:
            np.add.at(q, sd.ln, sd.iter_q(self.p[sd.ln]))
        self._put(self.q_buffer[: 2 * self.nfree], q)

    def iterate_finish(self) -> int:
        q = self._get(self.q_buffer[: 2 * self.nfree])
        pq = np.sum(self.p * q)
        malpha = 0j if (abs(self.rz) < NEARLY_ZERO and abs(pq) < NEARLY_ZERO) else -(self.rz / pq)
        self.u = self.u + malpha * self.p
        self.r = self.r + malpha * q
        resi = float(np.max(np.abs(self.r))) / self.norm0
        self.z = self.r * self.pc
        rz = np.sum(self.r * self.z)
        beta = 0j if (abs(rz) < NEARLY_ZERO and abs(self.rz) < NEARLY_ZERO) else rz / self.rz
        self.rz = rz
        if resi < self.eps or self.loop >= self.max_loop:
            self.status = 1
        self.loop += 1
        if self.status == 1:
            self.p = self.u.copy()
            self.status = 2
        else:
            self.p = self.z + beta * self.p
        return self.status

    def last(self) -> None:
        self.x_local = [(s, sd.last_x(self.p[sd.ln])) for s, sd in self.subs]

    def edge_solution_buffer(self):
        x = np.zeros(self.model.n_edges, dtype=np.complex128)
        for s, xl in self.x_local:
            mine = self.owner[self.subs_gid(s)] == s
            x[self.subs_gid(s)[mine]] = xl[mine]
        buf = torch.zeros(2 * self.model.n_edges, dtype=torch.float64)
        self._put(buf, x)
        return buf

    def subs_gid(self, s):
        for t, sd in self.subs:
            if t == s:
                return sd.edge_gid
        raise KeyError(s)

    def edge_solution_from(self, buf):
        return self._get(buf)
