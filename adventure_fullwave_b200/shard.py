"""Sharded HDDM solve over several GPUs: one process and one context per rank.

The reference's p-mode splits the subdomains into parts, one per MPI rank;
every interface iteration the parts exchange their contributions on the DOFs
they share with their neighbours and all-reduce the COCG scalars
(``lib/hddm/hddm_solver_ph.h:112-329``).  Here a shard is a contiguous range
of subdomain ids: the partitioner numbers the RCB leaves in tree order, so a
contiguous range is a union of RCB subtrees.  Each shard runs the COCG on the
interface DOFs its subdomains hold; every DOF has one owner, the shard of the
first subdomain holding it, and the dot products and the max-norm run over
the owned DOFs and are summed (or maxed) over the ranks.  Per iteration the
ranks all-reduce a packed vector of the DOFs two or more shards hold (the
partial Q), then (p, q), then (r, z), |r|^2 and max|r|; the shards holding a
DOF compute the same bits for it, so their scalars and iteration counts
agree.

``run_sharded`` is the orchestration; a backend does the work of one shard.
``GpuShard`` runs a shard on this rank's GPU through the C ABI (the exchange
buffers are torch tensors, reduced with ``torch.distributed.all_reduce`` over
NCCL).  A backend only needs the attributes and methods ``GpuShard`` has.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np

from . import hddm

# exchange(buf, op) reduces buf over the ranks in place; op is "sum" or "max"
ExchangeFn = Callable[[object, str], None]


def shard_ranges(model, world: int) -> List[Tuple[int, int]]:
    """Contiguous subdomain ranges, one per rank, with about equal element
    counts (the work of a subdomain grows with its elements)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    nsub = int(model.nsub)
    if world > nsub:
        raise ValueError("more ranks than subdomains")
    cost = np.bincount(np.asarray(model.sub_of_tet), minlength=nsub).astype(np.float64)
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        # first subdomain boundary at or after r/world of the work, keeping
        # at least one subdomain per remaining rank
        b = int(np.searchsorted(cum, total * r / world, side="left"))
        b = max(b, bounds[-1] + 1)
        b = min(b, nsub - (world - r))
        bounds.append(b)
    bounds.append(nsub)
    return [(bounds[i], bounds[i + 1]) for i in range(world)]


def shard_bounds(model, world: int) -> List[int]:
    """The ranges of ``shard_ranges`` as world+1 boundaries."""
    r = shard_ranges(model, world)
    return [a for a, _ in r] + [r[-1][1]]


def run_sharded(backend, exchange: ExchangeFn, source=0):
    """One sharded HDDM solve.  Every rank calls ``exchange`` on the same
    buffers in the same order.  Returns the backend's edge solution summed
    over ranks (the whole solution on every rank) and the number of COCG
    iterations."""
    backend.make_tmp_aij(source)
    backend.first()
    exchange(backend.pack, "sum")
    backend.sync()
    backend.first_sums()
    exchange(backend.scal_sums, "sum")
    exchange(backend.scal_max, "max")
    backend.sync()
    status = backend.first_finish()
    iterations = 0
    while status == 0:
        backend.iterate()
        exchange(backend.pack_q, "sum")
        backend.sync()
        backend.iterate_pq()
        exchange(backend.scal_pq, "sum")
        backend.sync()
        backend.iterate_update()
        exchange(backend.scal_sums, "sum")
        exchange(backend.scal_max, "max")
        backend.sync()
        status = backend.iterate_finish()
        iterations += 1
    backend.last()
    x = backend.edge_solution_buffer()
    exchange(x, "sum")
    return backend.edge_solution_from(x), iterations


class GpuShard:
    """One shard on this rank's GPU through the C ABI.  ``bounds`` are all
    shards' subdomain ranges (``shard_bounds``)."""

    def __init__(self, model, shard: Tuple[int, int], bounds: Sequence[int], device: int = 0, **opts):
        import torch

        self._torch = torch
        self.solver = hddm.HddmSolver(model, device=device, shard=shard, **opts)
        self.n_shared = self.solver.shard_set_layout(bounds)
        self.n_edges = int(model.n_edges)
        self.device = torch.device("cuda", device)
        n = max(1, self.n_shared)
        # the packed partial Q, then (first step) the packed diagonal
        self.pack = torch.zeros(4 * n, dtype=torch.float64, device=self.device)
        self.pack_q = self.pack[: 2 * n]
        # [0..2] summed ((p, q) in [0..1] during the pq step), [4] maxed
        self.scal = torch.zeros(8, dtype=torch.float64, device=self.device)
        self.scal_sums = self.scal[0:3]
        self.scal_pq = self.scal[0:2]
        self.scal_max = self.scal[4:5]
        self.solver.shard_set_exchange(self.pack.data_ptr(), self.scal.data_ptr())

    def sync(self) -> None:
        """The library reads the buffers on its own stream: finish the reduction first."""
        self._torch.cuda.current_stream(self.device).synchronize()

    def make_tmp_aij(self, source) -> None:
        self.solver.make_tmp_aij(source)

    def first(self) -> None:
        self.solver.shard_first()

    def first_sums(self) -> None:
        self.solver.shard_first_sums()

    def first_finish(self) -> int:
        return self.solver.shard_first_finish()

    def iterate(self) -> None:
        self.solver.shard_iterate()

    def iterate_pq(self) -> None:
        self.solver.shard_iterate_pq()

    def iterate_update(self) -> None:
        self.solver.shard_iterate_update()

    def iterate_finish(self) -> int:
        return self.solver.shard_iterate_finish()

    def last(self) -> None:
        self.solver.solve_dom_last()

    def edge_solution_buffer(self):
        x = self.solver.edge_solution()
        return self._torch.from_numpy(np.ascontiguousarray(np.stack([x.real, x.imag], 1).ravel())).to(self.device)

    def edge_solution_from(self, buf) -> np.ndarray:
        v = buf.cpu().numpy()
        return v[0::2] + 1j * v[1::2]

    def close(self) -> None:
        self.solver.close()


def torch_exchange(group=None) -> ExchangeFn:
    """Sum or max over the ranks of ``group`` (torch.distributed, NCCL for
    CUDA tensors, gloo for CPU tensors), in place."""
    import torch.distributed as dist

    ops = {"sum": dist.ReduceOp.SUM, "max": dist.ReduceOp.MAX}

    def _reduce(buf, op):
        dist.all_reduce(buf, op=ops[op], group=group)

    return _reduce


def sharded_solve(model, source=0, rank: int = 0, world: int = 1, device: int = 0, group=None, **opts):
    """A sharded solve with ``GpuShard`` and NCCL: the call every rank makes
    (under torchrun, after ``init_process_group("nccl")``)."""
    lo, hi = shard_ranges(model, world)[rank]
    backend = GpuShard(model, (lo, hi), shard_bounds(model, world), device=device, **opts)
    try:
        return run_sharded(backend, torch_exchange(group), source)
    finally:
        backend.close()


def run_lockstep(backends: Sequence, source=0):
    """Several shards driven in turn by one process, their buffers reduced on
    the device of the first: the protocol of ``run_sharded`` without a
    process group (used to check a sharded solve on one GPU)."""
    import torch

    def exchange(bufs, op):
        total = bufs[0].clone()
        for b in bufs[1:]:
            o = b.to(total.device)
            total = total + o if op == "sum" else torch.maximum(total, o)
        for b in bufs:
            b.copy_(total.to(b.device))

    def each(method):
        return [getattr(b, method)() for b in backends]

    def sync():
        for b in backends:
            b.sync()

    for b in backends:
        b.make_tmp_aij(source)
    each("first")
    exchange([b.pack for b in backends], "sum")
    sync()
    each("first_sums")
    exchange([b.scal_sums for b in backends], "sum")
    exchange([b.scal_max for b in backends], "max")
    sync()
    status = each("first_finish")
    iterations = 0
    while status[0] == 0:
        each("iterate")
        exchange([b.pack_q for b in backends], "sum")
        sync()
        each("iterate_pq")
        exchange([b.scal_pq for b in backends], "sum")
        sync()
        each("iterate_update")
        exchange([b.scal_sums for b in backends], "sum")
        exchange([b.scal_max for b in backends], "max")
        sync()
        status = each("iterate_finish")
        if len(set(status)) != 1:
            raise RuntimeError("shards disagree on the COCG status")
        iterations += 1
    each("last")
    xs = [b.edge_solution_buffer() for b in backends]
    exchange(xs, "sum")
    return backends[0].edge_solution_from(xs[0]), iterations
