"""The sharded HDDM solve (one rank per GPU, the reference's p-mode parts):
subdomain ranges, and the rank protocol of ``shard.run_sharded`` with two
gloo ranks on the CPU, against the oracle's single-process solve."""
import multiprocessing as mp
import os
import socket
import tempfile

import numpy as np
import pytest

from adventure_fullwave_b200 import meshgen, shard
from helpers import rel_l2
from oracle import oracle


def _model():
    m = meshgen.make_model("x", n=8, size=1.0, npml=2, nleaves=8, seed=3)
    meshgen.round_trip_material(m)
    return m


def test_shard_ranges_cover_contiguously():
    m = meshgen.make_model("c1")
    for world in (1, 2, 3, 4, 7):
        r = shard.shard_ranges(m, world)
        assert r[0][0] == 0 and r[-1][1] == m.nsub
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert all(hi > lo for lo, hi in r)
        cost = np.bincount(m.sub_of_tet, minlength=m.nsub)
        share = np.array([cost[lo:hi].sum() for lo, hi in r]) / cost.sum()
        assert share.max() <= 1.0 / world + cost.max() / cost.sum() + 1e-12
    with pytest.raises(ValueError):
        shard.shard_ranges(m, m.nsub + 1)


def test_cpu_backend_alone_matches_oracle():
    """One rank owning every subdomain: the backend itself against the oracle."""
    from shard_cpu import CpuShard

    m = _model()
    part = oracle.partition(m)
    xo, _, hist, _ = oracle.hddm(m, part, 1e-10, 5000)
    x, it = shard.run_sharded(CpuShard(m, (0, m.nsub), [0, m.nsub], hddm_eps=1e-10), lambda buf, op: None, 0)
    assert rel_l2(x, xo) <= 1e-8
    assert abs(it - len(hist)) <= max(2, len(hist) // 20)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist

    from shard_cpu import CpuShard

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        m = _model()
        lo, hi = shard.shard_ranges(m, world)[rank]
        b = CpuShard(m, (lo, hi), shard.shard_bounds(m, world), hddm_eps=1e-10)
        x, it = shard.run_sharded(b, shard.torch_exchange(), 0)
        np.savez(f"{out}_{rank}.npz", x=x, it=it, lo=lo, hi=hi, n_shared=b.n_shared, nfree=b.nfree,
                 held=b.held.shape[0], owned=int(b.owned.sum()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_single_process():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "x")
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        for p in procs:
            if p.is_alive():
                p.kill()
        assert all(p.exitcode == 0 for p in procs)
        res = [np.load(f"{out}_{r}.npz") for r in range(world)]
    m = _model()
    part = oracle.partition(m)
    xo, _, hist, _ = oracle.hddm(m, part, 1e-10, 5000)
    # every rank ends with the whole solution and the same iteration count
    assert int(res[0]["it"]) == int(res[1]["it"])
    assert np.array_equal(res[0]["x"], res[1]["x"])
    assert int(res[0]["hi"]) == int(res[1]["lo"]) and 0 < int(res[0]["hi"]) < m.nsub
    # the packed exchange: the same shared DOFs on both ranks, fewer than the
    # interface; every DOF owned by exactly one rank
    assert int(res[0]["n_shared"]) == int(res[1]["n_shared"])
    assert 0 < int(res[0]["n_shared"]) < int(res[0]["nfree"])
    assert int(res[0]["owned"]) + int(res[1]["owned"]) == int(res[0]["nfree"])
    assert rel_l2(res[0]["x"], xo) <= 1e-8
    assert abs(int(res[0]["it"]) - len(hist)) <= max(2, len(hist) // 20)
