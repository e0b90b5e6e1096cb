"""The library's sharded solve on one GPU: two shard contexts driven in turn
by one process (``shard.run_lockstep``, the partial sums added on the
device), against the unsharded solve of the same model."""
import numpy as np
import pytest

from adventure_fullwave_b200 import _lib, hddm, meshgen, shard
from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_two_shards_match_unsharded(precision):
    m = meshgen.make_model("x", n=12, size=1.0, npml=2, nleaves=6, seed=5)
    meshgen.round_trip_material(m)
    opts = dict(hddm_eps=1e-10, hddm_max_loop=20000, precision=precision, ir_max_steps=2)
    with hddm.HddmSolver(m, **opts) as s:
        r = s.solve(0)
        x_ref = s.edge_solution()
    backends = [shard.GpuShard(m, rng, shard.shard_bounds(m, 2), device=0, **opts) for rng in shard.shard_ranges(m, 2)]
    try:
        x, it = shard.run_lockstep(backends, 0)
    finally:
        for b in backends:
            b.close()
    assert rel_l2(x, x_ref) <= (1e-8 if precision == "fp64" else 1e-6)
    assert abs(it - r.iterations) <= max(2, r.iterations // 20)


def test_sharded_context_refuses_whole_solve():
    m = meshgen.make_model("x", n=6, size=1.0, npml=1, nleaves=4, seed=1)
    meshgen.round_trip_material(m)
    with hddm.HddmSolver(m, shard=(0, 2)) as s:
        with pytest.raises(_lib.FwgpuError):
            s.solve(0)
    with pytest.raises(_lib.FwgpuError):
        hddm.HddmSolver(m, shard=(2, 9))
