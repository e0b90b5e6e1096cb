"""CPU backend of one shard of the sharded HDDM solve, for the multi-process
(gloo) tests of ``adventure_fullwave_b200.shard``.  Test infrastructure only.

Each owned subdomain is the oracle's assembled system (``oracle.assemble_sub``,
the reference's TMP_AIJ rows) solved densely after Dirichlet elimination
(SetBC, ``aij_matrix_func.h:60-136``); the COCG is the same recurrence as the
library's kernels (``ITERATION_S_1ST`` / ``ITERATION_S``,
``lib/hddm/hddm_solver_s.h:158-400``), on the DOFs each shard holds, with
the packed exchange of the shared ones, as the library runs it.
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
    on the CPU, for the subdomains [lo, hi) of ``model``; ``bounds`` are all
    shards' ranges.  The COCG runs on the interface DOFs the shard's
    subdomains hold, the sums over the DOFs it owns, as the library's."""

    def __init__(self, model, shard, bounds, hddm_eps=1e-10, hddm_max_loop=5000):
        self.model = model
        self.lo, self.hi = shard
        self.bounds = list(bounds)
        self.eps = hddm_eps
        self.max_loop = hddm_max_loop
        self.subs = []
        self.nfree = 0

    def sync(self) -> None:
        pass

    def make_tmp_aij(self, source) -> None:
        part = oracle.partition(self.model, source)
        self.nfree = part.tfree
        self.owner = np.full(self.model.n_edges, -1, dtype=np.int64)
        for s in range(len(part.subs) - 1, -1, -1):
            self.owner[part.subs[s].edge_gid] = s
        self.subs = [(s, _Sub(self.model, part.subs[s])) for s in range(self.lo, self.hi)]
        # the layout: held DOFs, owned ones (shard of the first holder), packed positions
        shard_of = np.searchsorted(np.asarray(self.bounds), np.arange(len(part.subs)), side="right") - 1
        me = int(shard_of[self.lo])
        holders = [[] for _ in range(self.nfree)]
        for s, sd in enumerate(part.subs):
            for g in sd.inbc_ln.tolist():
                holders[g].append(int(shard_of[s]))
        self.held, self.owned, self.pos = [], [], []
        shared = 0
        for g in range(self.nfree):
            ks = holders[g]
            ps = -1
            if len(set(ks)) >= 2:
                ps = shared
                shared += 1
            if me in ks:
                self.held.append(g)
                self.owned.append(ks[0] == me)
                self.pos.append(ps)
        self.held = np.array(self.held, np.int64)
        self.owned = np.array(self.owned, bool)
        self.pos = np.array(self.pos, np.int64)
        self.n_shared = shared
        n = max(1, shared)
        self.pack = torch.zeros(4 * n, dtype=torch.float64)
        self.pack_q = self.pack[: 2 * n]
        self.scal = torch.zeros(8, dtype=torch.float64)
        self.scal_sums = self.scal[0:3]
        self.scal_pq = self.scal[0:2]
        self.scal_max = self.scal[4:5]
        for v in ("p", "u", "r", "z", "q", "pc"):
            setattr(self, v, np.zeros(self.nfree, dtype=np.complex128))

    def _put(self, view, vec):
        v = view.numpy()
        v[0::2] = vec.real
        v[1::2] = vec.imag

    def _get(self, view):
        v = view.numpy()
        return v[0::2] + 1j * v[1::2]

    def _pack(self, partial, at):
        packed = np.zeros(max(1, self.n_shared), dtype=np.complex128)
        sh = self.pos >= 0
        packed[self.pos[sh]] = partial[self.held[sh]]
        self._put(self.pack[2 * at * max(1, self.n_shared): 2 * (at + 1) * max(1, self.n_shared)], packed)

    def _unpack(self, partial, at):
        packed = self._get(self.pack[2 * at * max(1, self.n_shared): 2 * (at + 1) * max(1, self.n_shared)])
        out = partial[self.held].copy()
        sh = self.pos >= 0
        out[sh] = packed[self.pos[sh]]
        return out

    def _partial(self, per_sub):
        v = np.zeros(self.nfree, dtype=np.complex128)
        for _, sd in self.subs:
            np.add.at(v, sd.ln, per_sub(sd))
        return v

    def first(self) -> None:
        self.q_part = self._partial(lambda sd: sd.first_q())
        self.pc_part = self._partial(lambda sd: sd.diag_g)
        self._pack(self.q_part, 0)
        self._pack(self.pc_part, 1)

    def first_sums(self) -> None:
        h = self.held
        q = self._unpack(self.q_part, 0)
        pcs = self._unpack(self.pc_part, 1)
        self.pc[h] = np.where(pcs == 0, 1.0 + 0j, 1.0 / np.where(pcs == 0, 1.0, pcs))
        self.q[h] = q
        self.r[h] = q
        self.z[h] = self.r[h] * self.pc[h]
        self.p[h] = self.z[h]
        self.u[h] = 0
        self._local_sums()

    def _local_sums(self):
        o = self.held[self.owned]
        rz = np.sum(self.r[o] * self.z[o])
        sc = self.scal.numpy()
        sc[0], sc[1], sc[2] = rz.real, rz.imag, float(np.sum(np.abs(self.r[o]) ** 2))
        sc[4] = float(np.max(np.abs(self.r[o]))) if o.size else 0.0

    def first_finish(self) -> int:
        sc = self.scal.numpy()
        self.norm0 = float(sc[4])
        self.rz = complex(sc[0], sc[1])
        self.loop = 1
        self.status = 1 if self.norm0 < NEARLY_ZERO else 0
        if self.status:
            self.p[self.held] = self.u[self.held]
            self.status = 2
        return self.status

    def iterate(self) -> None:
        self.q_part = self._partial(lambda sd: sd.iter_q(self.p[sd.ln]))
        self._pack(self.q_part, 0)

    def iterate_pq(self) -> None:
        h = self.held
        self.q[h] = self._unpack(self.q_part, 0)
        o = self.held[self.owned]
        pq = np.sum(self.p[o] * self.q[o])
        sc = self.scal.numpy()
        sc[0], sc[1] = pq.real, pq.imag

    def iterate_update(self) -> None:
        sc = self.scal.numpy()
        pq = complex(sc[0], sc[1])
        malpha = 0j if (abs(self.rz) < NEARLY_ZERO and abs(pq) < NEARLY_ZERO) else -(self.rz / pq)
        h = self.held
        self.u[h] = self.u[h] + malpha * self.p[h]
        self.r[h] = self.r[h] + malpha * self.q[h]
        self.z[h] = self.r[h] * self.pc[h]
        self._local_sums()

    def iterate_finish(self) -> int:
        sc = self.scal.numpy()
        resi = float(sc[4]) / self.norm0
        rz = complex(sc[0], sc[1])
        beta = 0j if (abs(rz) < NEARLY_ZERO and abs(self.rz) < NEARLY_ZERO) else rz / self.rz
        self.rz = rz
        if resi < self.eps or self.loop >= self.max_loop:
            self.status = 1
        self.loop += 1
        h = self.held
        if self.status == 1:
            self.p[h] = self.u[h]
            self.status = 2
        else:
            self.p[h] = self.z[h] + beta * self.p[h]
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
