"""fwgpu_skyline_solve_noalloc: the batched skyline substitution for callers
that cannot allocate device memory when they solve (a host framework that
owns the device memory through its own pool, or a loop that must stay out of
the allocator).  Its work vectors live in a fixed device array; this test
checks its output against the regular solver's (fwgpu_hddm_solve on a model
with one subdomain, where the HDDM solve is a direct solve of the skyline
system), on two calls in a row with different right-hand sides, and checks
that sizes beyond the fixed array are refused."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_regular_solver():
    import torch

    from adventure_fullwave_b200 import _lib, hddm, meshgen

    model = meshgen.make_model("x", n=5, size=1.0, npml=1, nleaves=1)
    meshgen.round_trip_material(model)
    with hddm.HddmSolver(model, hddm_eps=1e-6, hddm_max_loop=100) as s:
        r = s.solve(0)
        x_ref = s.edge_solution()
        idx1, idx2, nlen = s.skyline_profile(0)
        fac = s.factor(0)
        maps = s.subdomain_maps(0)
        _, _, _, b = s.tmp_aij(0)
    assert r.iterations == 0
    n = idx1.shape[0]
    # right-hand side after Dirichlet elimination: the PEC rows carry their value, zero
    b = b.copy()
    b[maps["ibc"]] = 0.0

    lib = _lib.load()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    # a batch of two copies of the system
    row_off = torch.tensor([0, n, 2 * n], dtype=torch.int32, device=dev)
    mat_off = torch.tensor([0, nlen], dtype=torch.int64, device=dev)
    i1 = torch.tensor(np.concatenate([idx1, idx1]), dtype=torch.int32, device=dev)
    i2 = torch.tensor(np.concatenate([idx2, idx2]), dtype=torch.int32, device=dev)
    mat = torch.tensor(np.stack([np.concatenate([fac, fac]).real, np.concatenate([fac, fac]).imag], 1).ravel(),
                       dtype=torch.float64, device=dev)
    x = torch.zeros(4 * n, dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def solve(b1, b2):
        bb = np.concatenate([b1, b2])
        bt = torch.tensor(np.stack([bb.real, bb.imag], 1).ravel(), dtype=torch.float64, device=dev)
        rc = lib.fwgpu_skyline_solve_noalloc(2, 2 * n, _dev(row_off), _dev(mat_off), _dev(i1), _dev(i2), _dev(mat),
                                             _dev(bt), _dev(x), stream)
        assert rc == _lib.OK, lib.fwgpu_last_error().decode()
        torch.cuda.synchronize(dev)
        xh = x.cpu().numpy()
        xc = xh[0::2] + 1j * xh[1::2]
        return xc[:n], xc[n:]

    def check(x_local, scale):
        got = np.zeros_like(x_ref)
        got[maps["edge_gid"]] = x_local
        want = scale * x_ref
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)

    xa, xb = solve(b, 2.0 * b)
    check(xa, 1.0)
    check(xb, 2.0)
    # second call in a row, other right-hand sides: nothing stale from the first
    xa, xb = solve(3.0 * b, b)
    check(xa, 3.0)
    check(xb, 1.0)


def test_noalloc_refuses_sizes_beyond_the_work_array():
    from adventure_fullwave_b200 import _lib

    lib = _lib.load()
    rc = lib.fwgpu_skyline_solve_noalloc(1, _lib.NOALLOC_MAX_ROWS + 1, None, None, None, None, None, None, None,
                                         None)
    assert rc == _lib.ERR_ARG
    assert "exceeds" in lib.fwgpu_last_error().decode()
