"""Parity of the CUDA path (through the C ABI) with the oracle, the
reference's golden outputs and an FP64 sparse direct solve.

Tolerances: integer work (numbering, skyline profile) and the assembled
matrix are bit-exact; the FP64 factor agrees to 1e-12 relative (parallel
dot products sum in a different order); FP64 solutions at a tight COCG
tolerance agree to 1e-8 relative L2; the FP32-factor path with FP64
refinement agrees with the FP64 path to 1e-6 relative L2.  Against the
exact discrete solution (oracle/direct.py) an HDDM solve stopped at
hddm_eps has an error of a few hddm_eps (the reference's own C1 solve:
3.9e-6 at 1e-6, 3.5e-10 at 1e-10)."""
import numpy as np
import pytest

from adventure_fullwave_b200 import _lib, hddm, meshgen
from helpers import golden, rel_l2
from oracle import direct, oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["tiny", "layered"])
def test_assembly_profile_factor(name):
    z, params, model = golden(name)
    part = oracle.partition(model)
    with hddm.HddmSolver(model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
        s.make_tmp_aij(0)
        s.solve_dom_1st()
        for k in range(model.nsub):
            rp, col, val, b = s.tmp_aij(k)
            assert np.array_equal(rp, z[f"s{k}_aij_row_ptr"])
            assert np.array_equal(col, z[f"s{k}_aij_col"])
            assert np.array_equal(val, z[f"s{k}_aij_val"]), "assembled values must be bit-identical"
            _, _, _, bo = oracle.assemble_sub(model, part.subs[k])
            assert np.array_equal(b, bo)
            idx1, idx2, nlen = s.skyline_profile(k)
            assert np.array_equal(idx1, z[f"s{k}_idx1"]) and np.array_equal(idx2, z[f"s{k}_idx2"])
            ref = z[f"s{k}_fac"]
            assert nlen == ref.shape[0]
            fac = s.factor(k)
            assert np.max(np.abs(fac - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["tiny", "layered"])
def test_fp64_solution_vs_reference(name):
    z, params, model = golden(name)
    x, r = hddm.hddm_solver_CS(model, 0, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"])
    assert r.converged
    assert abs(r.iterations - int(z["iterations"][0])) <= max(2, int(0.05 * int(z["iterations"][0])))
    assert r.initial_norm == pytest.approx(float(z["norm0"][0]), rel=1e-6)
    assert rel_l2(x, z["x"]) <= 1e-8


def test_c1_fp64_vs_reference():
    """C1 (16^3 cells, 64 subdomains) to hddm_eps 1e-10 against the
    reference's own run: every edge value within 1e-8 relative L2 (the north
    star's bar for the FP64 path is 1e-6), the initial norm and the first 20
    residuals within 1e-9 relative (the reference's full-precision history),
    the iteration count within 5 % (693 in the reference)."""
    z, params, model = golden("c1")
    assert params["eps"] == 1e-10
    with hddm.HddmSolver(model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
        r = s.solve(0)
        x = s.edge_solution()
        hist = s.history()
    assert r.converged and r.final_resi < params["eps"]
    n_ref = int(z["iterations"][0])
    print(f"C1 eps 1e-10: {r.iterations} iterations (reference {n_ref}), "
          f"rel L2 vs reference {rel_l2(x, z['x']):.2e}")
    assert abs(r.iterations - n_ref) <= 0.05 * n_ref
    assert r.initial_norm == pytest.approx(float(z["norm0_full"][0]), rel=1e-12)
    assert np.allclose(hist[:20], z["hist_full"][:20], rtol=1e-9, atol=0)
    assert rel_l2(x, z["x"]) <= 1e-8


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_c1_vs_direct_solve(precision):
    """The error of the C1 solve against the FP64 sparse direct solve of
    the global system, at hddm_eps 1e-6 and 1e-10: within 10 hddm_eps."""
    model = meshgen.make_model("c1")
    meshgen.round_trip_material(model)
    xd = direct.solve(model, 0)
    for eps in (1e-6, 1e-10):
        x, r = hddm.hddm_solver_CS(model, 0, hddm_eps=eps, hddm_max_loop=40000, precision=precision,
                                   ir_max_steps=2)
        err = rel_l2(x, xd)
        print(f"C1 {precision} eps {eps:g}: {r.iterations} iterations, rel L2 vs direct {err:.2e}")
        assert r.converged
        assert err <= 10 * eps


@pytest.mark.parametrize("name,n", [("c2_head", 10), ("c3_head", 3)])
def test_first_iterations_vs_reference(name, n):
    """C2 (48^3 cells, 1,654 subdomains, 323,905 interface DOFs) and C3
    (96^3 cells, 8,822 subdomains, 2,436,383 interface DOFs): the initial
    max-norm and the residuals of the first interface iterations against
    the reference's run of the same model (full precision)."""
    z, params, model = golden(name)
    with hddm.HddmSolver(model, hddm_eps=1e-12, hddm_max_loop=n) as s:
        r = s.solve(0)
        hist = s.history()
        assert s.sizes()["total_free"] == int(z["total_free"][0])
    assert r.iterations == n and not r.converged
    rel = np.abs(hist[:n] / z["hist_full"] - 1.0)
    print(f"{name} norm0 {r.initial_norm!r} vs {float(z['norm0_full'][0])!r}; "
          f"first {n} residuals max rel dev {rel.max():.1e}")
    assert r.initial_norm == pytest.approx(float(z["norm0_full"][0]), rel=1e-12)
    assert rel.max() <= 1e-9


def test_c2_profiles_vs_oracle():
    """The skyline profile (idx1, idx2, nlen) of every C2 subdomain, computed
    on the device, equals the oracle's (the oracle's equals the reference's
    on the golden models)."""
    model = meshgen.make_model("c2")
    meshgen.round_trip_material(model)
    part = oracle.partition(model)
    with hddm.HddmSolver(model, hddm_eps=1e-6, hddm_max_loop=1) as s:
        s.make_tmp_aij(0)
        s.solve_dom_1st()
        for k in range(0, model.nsub, 7):
            idx1, idx2, nlen = s.skyline_profile(k)
            o1, o2, on, _ = oracle.factor_sub(model, part.subs[k])
            assert np.array_equal(idx1, o1) and np.array_equal(idx2, o2) and nlen == on, k


def test_c1_tight_tolerance_vs_oracle():
    model = meshgen.make_model("c1")
    meshgen.round_trip_material(model)
    part = oracle.partition(model)
    xo, _, ho, _ = oracle.hddm(model, part, 1e-10, 20000)
    x, r = hddm.hddm_solver_CS(model, 0, hddm_eps=1e-10, hddm_max_loop=20000)
    assert r.converged
    assert rel_l2(x, xo) <= 1e-7


def test_fp32_ir_vs_fp64():
    model = meshgen.make_model("c1")
    meshgen.round_trip_material(model)
    x64, r64 = hddm.hddm_solver_CS(model, 0, hddm_eps=1e-8, hddm_max_loop=20000)
    x32, r32 = hddm.hddm_solver_CS(model, 0, hddm_eps=1e-8, hddm_max_loop=20000, precision="fp32_ir",
                                   ir_max_steps=2)
    assert r32.converged
    assert rel_l2(x32, x64) <= 1e-6


@pytest.mark.parametrize("kernel", ["warp", "blockinv", "cta", "global"])
@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_solve_kernels_vs_oracle(kernel, precision):
    """Every batched subdomain-solve kernel against the oracle's FP64 HDDM at
    a tight tolerance, on subdomains large enough for multi-block sweeps and
    rows longer than 64 stored entries."""
    model = meshgen.make_model("x", n=12, size=1.0, npml=2, nleaves=6, seed=5)
    meshgen.round_trip_material(model)
    part = oracle.partition(model)
    xo, _, _, _ = oracle.hddm(model, part, 1e-10, 20000)
    x, r = hddm.hddm_solver_CS(model, 0, hddm_eps=1e-10, hddm_max_loop=20000, precision=precision,
                               ir_max_steps=2, solve_kernel=kernel)
    assert r.converged
    assert r.solve_kernel == kernel
    assert rel_l2(x, xo) <= (1e-7 if precision == "fp64" else 1e-6)


def test_single_subdomain_is_a_direct_solve():
    model = meshgen.make_model("x", n=4, size=1.0, npml=1, nleaves=1)
    meshgen.round_trip_material(model)
    part = oracle.partition(model)
    assert part.tfree == 0
    xo, _, _, _ = oracle.hddm(model, part, 1e-6, 100)
    x, r = hddm.hddm_solver_CS(model, 0, hddm_eps=1e-6, hddm_max_loop=100)
    assert r.iterations == 0
    assert rel_l2(x, xo) <= 1e-12


def test_resolve_matches_fresh_solve():
    model = meshgen.make_model("x", n=8, size=1.0, npml=2, nleaves=8, nsources=2, seed=4)
    meshgen.round_trip_material(model)
    with hddm.HddmSolver(model, hddm_eps=1e-9, hddm_max_loop=5000) as s:
        s.solve(0)
        r1 = s.resolve(1)
        x1 = s.edge_solution()
    x1f, r1f = hddm.hddm_solver_CS(model, 1, hddm_eps=1e-9, hddm_max_loop=5000)
    assert r1.iterations == r1f.iterations
    assert rel_l2(x1, x1f) <= 1e-12


def test_not_converged_status():
    model = meshgen.make_model("c1")
    with hddm.HddmSolver(model, hddm_eps=1e-12, hddm_max_loop=5, graph_iterations=4) as s:
        r = s.solve(0)
        assert not r.converged and r.iterations == 5
        assert len(s.history()) == 5
        with pytest.raises(_lib.FwgpuError) as e:
            s.resolve(0, raise_not_converged=True)
        assert e.value.code == _lib.ERR_NOT_CONVERGED


def test_call_order_is_checked():
    model = meshgen.make_model("tiny", n=4, npml=1, nleaves=4)
    with hddm.HddmSolver(model) as s:
        with pytest.raises(_lib.FwgpuError) as e:
            s.solve_dom_1st()
        assert e.value.code == _lib.ERR_STATE
        with pytest.raises(_lib.FwgpuError):
            s.iteration_s()


def test_slot_by_slot_equals_driver():
    z, params, model = golden("tiny")
    with hddm.HddmSolver(model, hddm_eps=params["eps"], hddm_max_loop=params["max_loop"]) as s:
        s.make_tmp_aij(0)
        s.solve_dom_1st()
        st = s.iteration_s_1st()
        n = 0
        while st == 0:
            st = s.iteration_s()
            n += 1
        s.solve_dom_last()
        x = s.edge_solution()
    assert rel_l2(x, z["x"]) <= 1e-8
    assert abs(n - int(z["iterations"][0])) <= 2


def test_contexts_with_different_subdomain_sizes_coexist():
    """Kernel shared-memory limits are process-wide: a context created later
    with smaller subdomains must not break the launches of an earlier one."""
    big = meshgen.make_model("x", n=12, size=1.0, npml=2, nleaves=6, seed=5)
    small = meshgen.make_model("x", n=8, size=1.0, npml=2, nleaves=16, seed=2)
    for m in (big, small):
        meshgen.round_trip_material(m)
    with hddm.HddmSolver(big, hddm_eps=1e-8, hddm_max_loop=20000) as sa:
        ra = sa.solve(0)
        xa = sa.edge_solution()
        for prec in ("fp64", "fp32_ir"):
            with hddm.HddmSolver(small, hddm_eps=1e-8, hddm_max_loop=20000, precision=prec) as sb:
                assert sb.solve(0).converged
        rb = sa.resolve(0)
        assert ra.converged and rb.converged
        assert rel_l2(sa.edge_solution(), xa) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_solves_are_reproducible(precision):
    """Two contexts, each with its own setup-time timing, give the same
    iteration count and the same bits: the timed choice never changes the
    order of the sums."""
    model = meshgen.make_model("x", n=12, size=1.5, npml=2, layers=3, nleaves=None, leaf_cap=150,
                               jitter=(0.3, 0.7), seed=7)
    meshgen.round_trip_material(model)
    runs = []
    for _ in range(3):
        x, r = hddm.hddm_solver_CS(model, 0, hddm_eps=1e-8, hddm_max_loop=20000, precision=precision)
        runs.append((x, r))
    for x, r in runs[1:]:
        assert r.iterations == runs[0][1].iterations
        assert np.array_equal(x, runs[0][0])
