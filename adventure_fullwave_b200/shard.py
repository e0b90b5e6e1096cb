"""Sharded HDDM solve over several GPUs: one process and one context per rank.

The reference's p-mode splits the subdomains into parts, one per MPI rank,
and every interface iteration sums the parts' contributions to the interface
vector and the COCG scalars (``lib/hddm/hddm_solver_ph.h:112-329``).  Here a
shard is a contiguous range of subdomain ids: the partitioner numbers the RCB
leaves in tree order, so a contiguous range is a union of RCB subtrees.  Every
rank keeps the whole interface vector; per iteration the ranks sum one
vector, the shard's partial Q (and on the first step the preconditioner
diagonal), with one all-reduce, and then all run the same COCG update on the
same sums, so their scalars and iteration counts agree.

``run_sharded`` is the orchestration; a backend does the work of one shard.
``GpuShard`` runs a shard on this rank's GPU through the C ABI (the exchange
buffer is a torch tensor, summed with ``torch.distributed.all_reduce`` over
NCCL).  A backend only needs the methods ``GpuShard`` has.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np

from . import hddm

ExchangeFn = Callable[[object], None]


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


def run_sharded(backend, exchange: ExchangeFn, source=0):
    """One sharded HDDM solve.  ``exchange(buf)`` sums ``buf`` over the ranks
    in place; every rank calls it the same number of times.  Returns the
    backend's edge solution summed over ranks (the whole solution on every
    rank) and the number of COCG iterations."""
    backend.make_tmp_aij(source)
    backend.first()
    exchange(backend.buffer)
    backend.sync()
    status = backend.first_finish()
    iterations = 0
    while status == 0:
        backend.iterate()
        exchange(backend.q_buffer)
        backend.sync()
        status = backend.iterate_finish()
        iterations += 1
    backend.last()
    x = backend.edge_solution_buffer()
    exchange(x)
    return backend.edge_solution_from(x), iterations


class GpuShard:
    """One shard on this rank's GPU through the C ABI."""

    def __init__(self, model, shard: Tuple[int, int], device: int = 0, **opts):
        import torch

        self._torch = torch
        self.solver = hddm.HddmSolver(model, device=device, shard=shard, **opts)
        self.nfree = int(self.solver.sizes()["total_free"])
        self.n_edges = int(model.n_edges)
        self.device = torch.device("cuda", device)
        # partial Q (complex, total_free), then the partial PC diagonal
        self.buffer = torch.zeros(4 * max(1, self.nfree), dtype=torch.float64, device=self.device)
        self.q_buffer = self.buffer[: 2 * max(1, self.nfree)]
        self.solver.shard_set_exchange(self.buffer.data_ptr())

    def sync(self) -> None:
        """The library reads the buffer on its own stream: finish the sum first."""
        self._torch.cuda.current_stream(self.device).synchronize()

    def make_tmp_aij(self, source) -> None:
        self.solver.make_tmp_aij(source)

    def first(self) -> None:
        self.solver.shard_first()

    def first_finish(self) -> int:
        return self.solver.shard_first_finish()

    def iterate(self) -> None:
        self.solver.shard_iterate()

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
    """Sum over the ranks of ``group`` (torch.distributed, NCCL for CUDA
    tensors, gloo for CPU tensors), in place."""
    import torch.distributed as dist

    def _sum(buf):
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)

    return _sum


def sharded_solve(model, source=0, rank: int = 0, world: int = 1, device: int = 0, group=None, **opts):
    """A sharded solve with ``GpuShard`` and NCCL: the call every rank makes
    (under torchrun, after ``init_process_group("nccl")``)."""
    lo, hi = shard_ranges(model, world)[rank]
    backend = GpuShard(model, (lo, hi), device=device, **opts)
    try:
        return run_sharded(backend, torch_exchange(group), source)
    finally:
        backend.close()


def run_lockstep(backends: Sequence, source=0):
    """Several shards driven in turn by one process, their buffers summed on
    the device of the first: the same protocol as ``run_sharded`` without a
    process group (used to check a sharded solve on one GPU)."""

    def exchange(bufs):
        total = bufs[0].clone()
        for b in bufs[1:]:
            total += b.to(total.device)
        for b in bufs:
            b.copy_(total.to(b.device))

    for b in backends:
        b.make_tmp_aij(source)
    for b in backends:
        b.first()
    exchange([b.buffer for b in backends])
    for b in backends:
        b.sync()
    status = [b.first_finish() for b in backends]
    iterations = 0
    while status[0] == 0:
        for b in backends:
            b.iterate()
        exchange([b.q_buffer for b in backends])
        for b in backends:
            b.sync()
        status = [b.iterate_finish() for b in backends]
        if len(set(status)) != 1:
            raise RuntimeError("shards disagree on the COCG status")
        iterations += 1
    for b in backends:
        b.last()
    xs = [b.edge_solution_buffer() for b in backends]
    exchange(xs)
    return backends[0].edge_solution_from(xs[0]), iterations
