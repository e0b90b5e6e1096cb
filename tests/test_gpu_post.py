"""The post step on the GPU (fwgpu_post_em_E: HDDM_post_em_E,
main/fullwave/fullwave.c:639-763) against the reference's own element
results (golden fixtures) and the oracle: bit for bit."""
import dataclasses

import numpy as np
import pytest

from adventure_fullwave_b200 import _lib, hddm, meshgen
from helpers import golden
from oracle import oracle

pytestmark = pytest.mark.gpu


def dropped_material(model):
    """The model with the first Permittivity and Conductor entries left out
    (the reference's post with the same shortened lists is the fixture's
    ``post_drop``)."""
    return dataclasses.replace(model, mat_flag=model.mat_flag[1:], mat_eps=model.mat_eps[1:],
                               mat_sigma=model.mat_sigma[1:])


@pytest.mark.parametrize("name", ["tiny", "layered"])
@pytest.mark.parametrize("tag", ["post", "post_drop"])
def test_post_vs_reference(name, tag):
    z, params, model = golden(name)
    m = dropped_material(model) if tag == "post_drop" else model
    with hddm.HddmSolver(m) as s:
        B, E, Je = s.post_em_E(z["x"])
    assert np.array_equal(B, z[f"{tag}_B"])
    assert np.array_equal(E, z[f"{tag}_E"])
    assert np.array_equal(Je, z[f"{tag}_Je"])


def test_post_after_solve_uses_the_solution():
    z, params, model = golden("layered")
    with hddm.HddmSolver(model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
        with pytest.raises(_lib.FwgpuError):
            s.post_em_E()  # no solution yet
        s.solve(0)
        x = s.edge_solution()
        got = s.post_em_E()
    want = oracle.post_em_E(model, x)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_post_device_buffers_and_skipped_results():
    import torch

    model = meshgen.make_model("c1")
    meshgen.round_trip_material(model)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(model.n_edges) + 1j * rng.standard_normal(model.n_edges)
    want = oracle.post_em_E(model, x)
    with hddm.HddmSolver(model) as s:
        host = s.post_em_E(x)
        dev = torch.device("cuda", 0)
        xd = torch.from_numpy(np.stack([x.real, x.imag], 1).ravel().copy()).to(dev)
        outs = [torch.full((6 * model.n_tets,), np.nan, dtype=torch.float64, device=dev) for _ in range(3)]
        s.post_em_E_into(xd.data_ptr(), outs[0].data_ptr(), 0, outs[2].data_ptr())
        torch.cuda.synchronize()
    for g, w in zip(host, want):
        assert np.array_equal(g, w)
    b = outs[0].cpu().numpy()
    je = outs[2].cpu().numpy()
    assert np.array_equal(b[0::2] + 1j * b[1::2], want[0].ravel())
    assert np.array_equal(je[0::2] + 1j * je[1::2], want[2].ravel())
    assert np.isnan(outs[1].cpu().numpy()).all()  # skipped result untouched


def test_post_after_a_batched_solve_uses_the_source_last_read():
    m = meshgen.make_model("c5", n=8, size=1.0, npml=2, leaf_cap=200, seed=7, nsources=3)
    meshgen.round_trip_material(m)
    with hddm.HddmSolver(m, hddm_eps=1e-10, hddm_max_loop=20000) as s:
        s.solve_multi([0, 1, 2])
        x1 = s.edge_solution_multi(1)
        got = s.post_em_E()
    want = oracle.post_em_E(m, x1)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
