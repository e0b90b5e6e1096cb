"""Benchmark of the B200 HDDM hot path: time to reach a 1e-6 max-norm
relative interface residual (the reference's COCG criterion,
lib/hddm/hddm_solver_s.h:311-318,370) on a synthetic layered-PML model,
by default C3 (96^3 cells x 6 tets, the configuration the FP32+IR target
is quoted on).

One step = one full HDDM solve with the model resident in HBM: element
assembly into the subdomain envelopes, LDL^T factors, first solve, COCG to
``--eps``, final solves.  ``value`` is seconds per solve on the device
(CUDA events on the solver's stream, max over ranks); ``e2e`` is the same
solve through the public API from host arrays (subdomain setup, uploads,
solve, download of the edge solution) timed per step.

    python bench.py [--gpus N --steps K --warmup W] [--config c3] [--precision fp64|fp32_ir]
    python bench.py --impl reference ...   # the reference's own CPU solver

``value`` is the FP64 solve (the reference's arithmetic); the line adds
``mixed_precision`` (the same model solved with FP32 factors and FP64
refinement to the same tolerance: time, iterations and relative L2 distance
to the FP64 solution, ``--mixed-steps`` timed solves), ``adjoint`` (the C4
design-region model: one forward solve and the backward call on its
factors), ``c2`` (the C2 model, FP64), ``correct_jo`` (the correction-Jo
pre-solve of the sample's antenna), ``sample`` (the reference's shipped
model) and ``accuracy`` (C1 solved in FP64 and FP32+IR, each solution's
relative L2 error against the FP64 sparse direct solve of the global system
kept in tests/golden/direct_c1.npz).

Under torchrun (N > 1) the model is sharded: every rank solves a contiguous
range of the subdomains and the ranks sum the partial interface vector with
one NCCL all-reduce per iteration (``adventure_fullwave_b200.shard``); rank 0
prints the line (``--replicas``: independent copies instead).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

from adventure_fullwave_b200 import meshgen  # noqa: E402

METRIC = "time-to-1e-6 HDDM residual, batched FP32+IR vs plain FP64, 1 B200; grad time"
WORKLOADS = {
    "c1": "C1: [0,1]^3 16^3 hexes x 6 Kuhn tets (24,576 tets), vacuum, 4-cell PML, PEC wall, 300 MHz, "
          "centre z-dipole, RCB 1 part x 64 subdomains",
    "c2": "C2: [0,1.5]^3 48^3 hexes x 6 tets (663,552 tets), 8 random layers, 6-cell PML, PEC wall, 300 MHz, "
          "centre z-dipole, jittered RCB (leaf cap 600) 1 part x 1654 subdomains",
    "c3": "C3: [0,1.5]^3 96^3 hexes x 6 tets (5,308,416 tets), 8 random layers, 8-cell PML, PEC wall, 300 MHz, "
          "centre z-dipole, jittered RCB (leaf cap 900) 1 part x 8822 subdomains",
    "c4": "C4: the C2 mesh and medium with a central 12^3-cell design region (10,368 tets, per-tet complex eps_r, "
          "eps' ~ U[2,4], eps'' ~ U[0,0.1]); J = sum |E|^2 on 8 probe edges; forward solve + adjoint gradient",
    "c5": "C5: [0,1.5]^3 112^3 hexes x 6 tets (8,429,568 tets), 8 random layers + 5% inclusions eps_r ~ U[10,20], "
          "8-cell PML, PEC wall, 300 MHz, jittered RCB (leaf cap 1000); 16 seeded z-dipoles solved together on "
          "one set of FP32 factors with FP64 refinement, then the adjoint gradient of J = sum |E|^2 on 8 probe edges "
          "over a central 12^3-cell design region for every source (one batched adjoint solve)",
}
# COCG iterations to 1e-6 of the FP64 GPU solve on each model (B200, this
# code); the reference's CPU time is extrapolated with them where running the
# reference to convergence would take hours (C2: ~7,800 iterations at about
# 1.1 s each, C3: ~9,000 at about 10 s each).
ITERS_FP64 = {"c1": 450, "c2": 7807, "c3": 8991}
DIRECT_FIXTURE = os.path.join(REPO, "tests", "golden", "direct_c1.npz")
TRAFFIC = os.path.join(REPO, "profiles", "dram_traffic.json")


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            t = [x.strip() for x in line.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                mx = max(mx, float(t[2]))
            except ValueError:
                continue
            for n, v in zip(names, t[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(sz: dict, precision: str, ir_steps: int) -> int:
    """Bytes one batched subdomain-solve phase of an interface iteration must
    move at least: (k+1) passes over the interior envelope (k = refinement
    steps; FP64 has k = 0, and a second sweep over the same rows counts once),
    the interface-row and coupling operators once (value + column), the
    interior operator once per refinement step, c_v = 4 passes over the
    subdomains' local FP64 vectors and the interface values in and out."""
    elem = 16 if precision == "fp64" else 8
    k = 0 if precision == "fp64" else ir_steps
    b = (k + 1) * sz["nlen_interior"] * elem
    b += (sz["nnz_interface_rows"] + sz["nnz_coupling"]) * 20
    b += k * sz["nnz_interior"] * 20
    b += sz["total_dofs"] * 16 * 4
    b += sz["total_iface_slots"] * (4 + 16 + 16)
    return int(b)


SAMPLE_FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "ref_sample.npz")
COJO_FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "ref_cojo.npz")


def sample_model():
    """The reference's shipped sample model with its antenna currents, from
    the fixture tests/golden/make_sample.py made by running the reference."""
    from adventure_fullwave_b200 import advio, meshgen

    z = np.load(SAMPLE_FIXTURE)
    tets, tet_edges = z["tets"], z["tet_edges"]
    ne = int(tet_edges.max()) + 1
    edges = np.zeros((ne, 2), np.int32)
    for q, (a, b) in enumerate(advio._MID_PAIRS):
        edges[tet_edges[:, q], 0] = np.minimum(tets[:, a], tets[:, b])
        edges[tet_edges[:, q], 1] = np.maximum(tets[:, a], tets[:, b])
    m = meshgen.Model(name="sample", n=0, size=0.0, vertex_crd=z["vertex_crd"], tets=tets, tet_edges=tet_edges,
                      edges=edges, flag=z["flag"].astype(np.int32), mat_flag=z["mat_flag"], mat_eps=z["mat_eps"],
                      mat_sigma=z["mat_sigma"], omega=float(z["omega"][0]), pec_edge=np.zeros(ne, bool),
                      sub_of_tet=z["sub_of_tet"].astype(np.int32), nsub=int(z["nsub"][0]), sources=[],
                      sub_order=(z["sub_vertex_ptr"], z["sub_vertex_order"], z["sub_edge_ptr"], z["sub_edge_order"]))
    jo = np.zeros((1, m.n_vertices, 3))
    jor = np.zeros((1, m.n_vertices, 3))
    jo[0, z["antenna_vertices"]] = z["antenna_Jo"]
    jor[0, z["antenna_vertices"]] = z["antenna_Jor"]
    meshgen.antenna_source(m, z["antenna_flag"], jo, jor)
    return m, z


def post_algorithmic_bytes(model) -> int:
    """Bytes the post step must move at least: per element its 4 vertex ids,
    6 edge ids, Permittivity mark and conductivity (16 + 24 + 1 + 8 B) and
    its three results (3 x 3 complex, 144 B); each vertex coordinate triple
    (24 B) and each edge value (16 B) once."""
    return int(model.n_tets * (16 + 24 + 1 + 8 + 144) + model.n_vertices * 24 + model.n_edges * 16)


def ncu_traffic(config: str, precision: str):
    """DRAM bytes (read + write) of one subdomain-solve phase of an interface
    iteration, from the ncu capture summarised in profiles/dram_traffic.json
    (with the command that made it), when one covers this workload."""
    try:
        with open(TRAFFIC) as f:
            t = json.load(f).get(f"{config}_{precision}")
        return None if t is None else int(t["bytes_per_phase"])
    except (OSError, ValueError, KeyError):
        return None


def make_model(config: str):
    model = meshgen.make_model(config)
    meshgen.round_trip_material(model)
    return model


def run_reference_sample(model, n_loop: int):
    """One run of the reference itself (oracle/_ref/fw_ref_harness, built from
    its sources, single thread) on ``model``: setup, ``n_loop`` COCG
    iterations, the last solves.  Returns the harness's timings and the
    seconds of every interface iteration after the first, or None when the
    harness is not built."""
    sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
    import refdump

    if not os.path.exists(refdump.HARNESS):
        return None
    wd = tempfile.mkdtemp(prefix="fwbench_")
    try:
        t0 = time.time()
        out = refdump.run_harness(model, 1e-6, n_loop, dump=0, workdir=wd, timeout=1700)
        j = dict(out["json"])
        j["wall_s"] = time.time() - t0
        j["iteration_s"] = [float(v) for v in out["iteration_s"]]
        return j
    finally:
        shutil.rmtree(wd, ignore_errors=True)


def extrapolate(j, per_iter: float, n_iters: int) -> float:
    """The reference's time to 1e-6: its setup (reading, integer setup,
    assembly, factors, first solve) + n_iters interface iterations + the
    last solves."""
    return j["t_init_s"] + j["t_first_s"] + n_iters * per_iter + j["t_last_s"]


def cpu_baseline_reference(model, config: str, sample_iters: int, n_iters: int):
    """The reference on a bounded sample of the workload (setup plus
    ``sample_iters`` + 1 COCG iterations), extrapolated to ``n_iters``."""
    j = run_reference_sample(model, sample_iters + 1)
    if j is None:
        return None
    per_iter = float(np.mean(j["iteration_s"])) if j["iteration_s"] else 0.0
    setup = j["t_init_s"] + j["t_first_s"]
    return {"value": extrapolate(j, per_iter, n_iters), "unit": "s", "cores": 1, "kind": "reference",
            "sample": f"reference s-mode solver on the {config} model: setup + {sample_iters + 1} COCG iterations "
                      f"({j['wall_s']:.1f} s wall), {per_iter:.3f} s/iteration (mean of {len(j['iteration_s'])}) "
                      f"extrapolated to {n_iters} iterations",
            "setup_s": setup, "per_iteration_s": per_iter, "iterations_assumed": n_iters}


def run_reference(args):
    """The reference arm: one step = one interface iteration of the
    reference's own solver on the same model (single thread), W warm-up
    iterations then K timed; the line's value is the reference's setup +
    the GPU FP64 iteration count x the mean timed iteration + its last
    solves (a converged reference run of C2 or C3 would take hours)."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    model = make_model(args.config)
    n_iters = ITERS_FP64.get(args.config, 5000)
    j = run_reference_sample(model, args.warmup + args.steps + 1)
    if j is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/fw_ref_harness is not built"}))
        return 0
    timed = j["iteration_s"][args.warmup:args.warmup + args.steps]
    per_iter = float(np.mean(timed))
    value = extrapolate(j, per_iter, n_iters)
    sample = (f"reference s-mode solver on the {args.config} model, single thread: setup "
              f"{j['t_init_s'] + j['t_first_s']:.1f} s, {args.warmup} warm-up + {len(timed)} timed COCG iterations "
              f"({per_iter:.3f} s each), extrapolated to {n_iters} iterations (the GPU FP64 count)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_iter * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded generator; no dataset)",
            "config": {"workload": WORKLOADS.get(args.config, args.config), "precision": "fp64",
                       "hddm_eps": args.eps},
            "step": "one interface iteration of the reference (subdomain solves + COCG step)",
            "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    rank, world, local = env_rank()
    dist = None
    if world > 1 or args.sharded:
        import torch
        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        if not dist_mod.is_initialized():
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29531")
            dist_mod.init_process_group("nccl", rank=rank, world_size=world,
                                        timeout=__import__("datetime").timedelta(seconds=600))
        dist = dist_mod
        if args.sharded or not args.replicas:
            return run_sharded_bench(args, rank, world, local, dist)
    from adventure_fullwave_b200 import hddm

    def opts(**kw):
        o = dict(hddm_eps=args.eps, hddm_max_loop=args.max_loop, precision=args.precision,
                 ir_max_steps=args.ir_steps, ir_tol=args.ir_tol, ir_relax=args.ir_relax,
                 graph_iterations=args.graph_iters, device=local, solve_kernel=args.solve_kernel,
                 stage_cap=args.stage_cap, stage_warps=args.stage_warps)
        o.update(kw)
        return o

    def solve_s(r):
        return (r.t_setup_ms + r.t_iterate_ms + r.t_last_ms) / 1e3

    model = make_model(args.config)
    solver = hddm.HddmSolver(model, **opts())
    for _ in range(args.warmup):
        solver.solve(0)
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    clocks.start()
    times, iters, launches, results = [], [], [], []
    for _ in range(args.steps):
        r = solver.solve(0)
        results.append(r)
        times.append(solve_s(r))
        iters.append(r.iterations)
        launches.append(r.kernel_launches)
    clk = clocks.stop()
    total = float(np.sum(times))
    if dist:
        import torch

        t = torch.tensor([total], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
        dist.barrier()
    value = total / args.steps
    sz = solver.sizes()
    x_check = solver.edge_solution()

    # kernel timing of the dominant phase for the roofline
    prof = solver.profile_iteration(reps=args.prof_reps)
    peak, peak_kind = load_peaks()
    alg = algorithmic_bytes(sz, args.precision, args.ir_steps)
    achieved = alg / (prof["subsolve_ms"] * 1e-3) / 1e9
    traffic = ncu_traffic(args.config, args.precision)
    kname = {"warp": "rhs_kernel + subsolve_staged_kernel + iface_product_kernel",
             "blockinv": "rhs_kernel + subsolve_staged_kernel (block-inverse layout) + iface_product_kernel",
             "cta": "subsolve_cta_kernel", "global": "subsolve_kernel"}.get(results[-1].solve_kernel,
                                                                           results[-1].solve_kernel)
    roofline = {"bound": "hbm", "kernel": f"{kname} (one batched subdomain solve of an interface iteration)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} hbm_gbs", "traffic": traffic, "algorithmic_bytes": alg,
                "kernel_ms": prof["subsolve_ms"], "interface_kernels_ms": prof["interface_ms"],
                "iteration_ms_graph": prof["iteration_ms"],
                "timing": "CUDA events on the solver's stream over repeated iteration-mode launches"}

    # the post step (element B, E, Je from the converged edge values)
    post = None
    if not args.no_post:
        solver.resolve(0)
        post_ms = solver.profile_post(reps=args.prof_reps)
        pb = post_algorithmic_bytes(model)
        B, E, Je = solver.post_em_E()
        post_gbs = pb / (post_ms * 1e-3) / 1e9
        post = {"kernel": "post_em_E_kernel (HDDM_post_em_E over every element)", "kernel_ms": post_ms,
                "algorithmic_bytes": pb, "achieved": post_gbs, "peak": peak, "unit": "GB/s", "frac": post_gbs / peak,
                "peak_source": f"{peak_kind} hbm_gbs", "n_tets": model.n_tets,
                "finite": bool(np.isfinite(B).all() and np.isfinite(E).all() and np.isfinite(Je).all()),
                "timing": "device events per launch, L2 evicted before each"}
    solver.close()

    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        # the same model with FP32 factors and FP64 refinement, to the same tolerance
        with hddm.HddmSolver(model, **opts(precision="fp32_ir")) as s32:
            s32.solve(0)
            t32, it32 = [], []
            for _ in range(args.mixed_steps):
                r32 = s32.solve(0)
                t32.append(solve_s(r32))
                it32.append(r32.iterations)
            x32 = s32.edge_solution()
        v32 = float(np.mean(t32))
        mixed = {"fp32_ir_s": v32, "fp64_s": value, "fp64_over_fp32_ir": value / v32,
                 "fp32_ir_iterations": int(np.mean(it32)), "fp64_iterations": int(np.mean(iters)),
                 "rel_l2_vs_fp64": float(np.linalg.norm(x32 - x_check) / np.linalg.norm(x_check)),
                 "ir_steps": args.ir_steps, "ir_relax": args.ir_relax, "converged": bool(r32.converged),
                 "solve_kernel": r32.solve_kernel, "stage_cap": r32.stage_cap, "stage_warps": r32.stage_warps,
                 "timed_solves": args.mixed_steps}

    # the C2 model, FP64 (the configuration of the earlier lines)
    c2 = None
    if args.config != "c2" and not args.no_c2:
        m2 = make_model("c2")
        with hddm.HddmSolver(m2, **opts()) as s2:
            s2.solve(0)
            r2 = s2.solve(0)
            p2 = s2.profile_iteration(reps=args.prof_reps)
            a2 = algorithmic_bytes(s2.sizes(), args.precision, args.ir_steps)
        c2 = {"workload": WORKLOADS["c2"], "time_s": solve_s(r2), "iterations": r2.iterations,
              "phase_ms": p2["subsolve_ms"], "phase_frac": a2 / (p2["subsolve_ms"] * 1e-3) / 1e9 / peak,
              "timing": "device events of one solve (second of two)"}

    adjoint = None
    if not args.no_adjoint:
        # the adjoint is quoted on the C2 mesh with the design region (C4)
        adj_model = model if len(model.design_tets) > 0 else make_model("c4")
        with hddm.HddmSolver(adj_model, **opts()) as adj_solver:
            adj_solver.solve(0)
            # the backward: one adjoint HDDM solve on the forward factors plus the gradient kernel
            r = adj_solver.solve(0)
            t0 = time.perf_counter()
            J, ge, gs, ra = adj_solver.adjoint_gradient()
            t_adj = time.perf_counter() - t0
        adjoint = {"config": "c4", "forward_s": solve_s(r), "adjoint_s": t_adj,
                   "adjoint_over_forward": t_adj / solve_s(r), "J": J,
                   "forward_iterations": r.iterations, "adjoint_iterations": ra.iterations,
                   "n_design": int(len(adj_model.design_tets)),
                   "grad_finite": bool(np.all(np.isfinite(ge)) and np.all(np.isfinite(gs))),
                   "timing": "forward: device events of one solve; adjoint: host wall time of the backward call "
                             "(adjoint HDDM solve on the forward factors + gradient kernel)"}

    # the reference's shipped sample model, to the same tolerance as the
    # reference's own run kept in tests/golden/ref_sample.npz
    sample = None
    if not args.no_sample and os.path.exists(SAMPLE_FIXTURE):
        sm, z = sample_model()
        with hddm.HddmSolver(sm, hddm_eps=float(z["eps"][0]), hddm_max_loop=40000, device=local) as ss:
            ss.solve(None)
            rs = ss.solve(None)
            xs = ss.edge_solution()
        ref = z["x_sample"]
        got = xs[::int(z["x_sample_stride"][0])]
        sample = {"model": "the reference's shipped sample (main/fullwave/MODEL): 6 parts x 73 subdomains, "
                           "one antenna", "n_tets": sm.n_tets, "hddm_eps": float(z["eps"][0]),
                  "time_s": solve_s(rs), "iterations": rs.iterations,
                  "reference_iterations": int(z["iterations"][0]),
                  "initial_norm": rs.initial_norm, "reference_initial_norm": float(z["norm0"][0]),
                  "rel_l2_vs_reference": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                  "timing": "device events of one solve (second of two)"}

    # the correction-Jo pre-solve of the sample's antenna (main.c:92-98), both
    # passes, against the reference's own pre-solve kept in tests/golden/ref_cojo.npz
    correct_jo = None
    if not args.no_sample and os.path.exists(SAMPLE_FIXTURE) and os.path.exists(COJO_FIXTURE):
        try:
            cz = np.load(COJO_FIXTURE)
            es = sm.element_source
            t0 = time.perf_counter()
            with hddm.CorrectJoSolver(sm, int(cz["sample_flag"][0]), device=local) as cs:
                t1 = time.perf_counter()
                ihr, rr = cs.solve(es.antenna_Jor[0])
                ihi, ri = cs.solve(es.antenna_Jo[0])
                t2 = time.perf_counter()
            want = cz["sample_ihr"]
            got = ihr[cz["sample_vertex"]]
            correct_jo = {"model": "the sample's antenna: 7 subdomains, 26 interface DOFs (vertices)",
                          "iterations": [rr.iterations, ri.iterations],
                          "reference_iterations": [int(cz["sample_hist_r"].shape[0]), int(cz["sample_hist_i"].shape[0])],
                          "device_ms": [rr.t_setup_ms + rr.t_iterate_ms + rr.t_last_ms,
                                        ri.t_setup_ms + ri.t_iterate_ms + ri.t_last_ms],
                          "host_s": {"context": t1 - t0, "two_passes": t2 - t1},
                          "rel_l2_vs_reference_Ihr": float(np.linalg.norm(got - want) / np.linalg.norm(want)),
                          "Ihi_max_abs": float(np.abs(ihi).max())}
        except Exception as exc:  # reported, never fatal to the headline line
            correct_jo = {"error": repr(exc)}

    # C1 against the exact discrete solution (FP64 sparse direct solve)
    accuracy = None
    if not args.no_accuracy and os.path.exists(DIRECT_FIXTURE):
        xd = np.load(DIRECT_FIXTURE)["x"]
        m1 = make_model("c1")
        accuracy = {"model": "C1", "reference_solution": "FP64 sparse direct solve of the global system "
                                                         "(SuperLU, oracle/direct.py)", "hddm_eps": args.eps}
        for prec in ("fp64", "fp32_ir"):
            x1, r1 = hddm.hddm_solver_CS(m1, 0, **opts(precision=prec))
            accuracy[prec] = {"rel_l2_error": float(np.linalg.norm(x1 - xd) / np.linalg.norm(xd)),
                              "iterations": r1.iterations}

    # end to end through the public API from host arrays
    e2e_times = []
    h2d = sum(a.nbytes for a in (model.vertex_crd, model.tets, model.tet_edges, model.flag, model.pec_edge,
                                 model.sub_of_tet, model.mat_flag, model.mat_eps, model.mat_sigma))
    d2h = model.n_edges * 16
    e2e_parts = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        with hddm.HddmSolver(model, **opts()) as s2:
            t1 = time.perf_counter()
            r2 = s2.solve(0)
            t2 = time.perf_counter()
            xe = s2.edge_solution()
        t3 = time.perf_counter()
        e2e_times.append(t3 - t0)
        # where the host time goes: context (host integer setup, uploads),
        # the solve call (its device time in r2), the download and release
        e2e_parts.append({"context_s": t1 - t0, "solve_call_s": t2 - t1,
                          "solve_device_s": (r2.t_setup_ms + r2.t_iterate_ms + r2.t_last_ms) / 1e3,
                          "download_release_s": t3 - t2})
    e2e = float(np.mean(e2e_times))
    if dist:
        import torch

        t = torch.tensor([e2e], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_reference(model, args.config, args.ref_iters,
                                     int(np.mean(iters)) if args.precision == "fp64" else
                                     ITERS_FP64.get(args.config, int(np.mean(iters))))
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if args.precision == "fp64" else "c64 factor, c128 refinement and COCG",
        "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": WORKLOADS.get(args.config, args.config), "precision": args.precision,
                   "hddm_eps": args.eps, "n_tets": model.n_tets, "n_subdomains": model.nsub,
                   "interface_dofs": sz["total_free"], "ir_steps": args.ir_steps if args.precision != "fp64" else 0,
                   "l2": "inputs larger than L2 (envelope %.0f MB)" % (
                       sz["nlen_interior"] * (16 if args.precision == "fp64" else 8) / 1e6),
                   "parallelism": f"{world} replica(s)"},
        "iterations": int(np.mean(iters)), "setup_ms": float(np.mean([r.t_setup_ms for r in results])),
        "iterate_ms": float(np.mean([r.t_iterate_ms for r in results])),
        "solve_kernel": {"kernel": results[-1].solve_kernel, "stage_cap": results[-1].stage_cap,
                         "stage_warps": results[-1].stage_warps},
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "parts": e2e_parts[-1] if e2e_parts else None},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(np.sum(launches)),
        "solution_check": {"finite": bool(np.all(np.isfinite(x_check))), "final_resi": results[-1].final_resi},
    }
    for k, v in (("mixed_precision", mixed), ("adjoint", adjoint), ("c2", c2), ("post", post), ("sample", sample),
                 ("correct_jo", correct_jo), ("accuracy", accuracy)):
        if v is not None:
            line[k] = v
    print(json.dumps(line))
    return 0


def run_c5(args):
    """C5: one step = the 16 sources solved together to ``--eps`` on one set
    of factors (``fwgpu_hddm_solve_multi``, FP32 factors with FP64
    refinement unless --precision fp64), then the batched adjoint of every
    source (``fwgpu_adjoint_gradient_multi``).  The value is the device time
    of the batched forward solve; a 16-source solve to 1e-6 takes minutes at
    this size, so run it with small --steps / --warmup by hand."""
    from adventure_fullwave_b200 import hddm

    precision = "fp32_ir" if args.precision == "fp64" and not args.c5_fp64 else args.precision
    model = meshgen.make_model("c5", design=12, nprobes=8)
    meshgen.round_trip_material(model)
    clocks = ClockSampler(0)
    with hddm.HddmSolver(model, hddm_eps=args.eps, hddm_max_loop=args.max_loop, precision=precision,
                         ir_max_steps=args.ir_steps, ir_relax=args.ir_relax, graph_iterations=args.graph_iters) as s:
        srcs = list(range(len(model.sources)))
        for _ in range(args.warmup):
            s.solve_multi(srcs)
        clocks.start()
        times, iters, adj = [], [], []
        for _ in range(args.steps):
            res = s.solve_multi(srcs)
            times.append((res[0].t_setup_ms + res[0].t_iterate_ms + res[0].t_last_ms) / 1e3)
            iters.append([r.iterations for r in res])
            # the forward result goes to stderr at once: the batched adjoint
            # that follows takes about as long again
            print(json.dumps({"c5_forward_s": times[-1], "iterations_per_source": iters[-1],
                              "converged": [bool(r.converged) for r in res]}), file=sys.stderr, flush=True)
            if not args.no_adjoint:
                t0 = time.perf_counter()
                J, ge, gs, ares = s.adjoint_gradient_multi()
                adj.append(time.perf_counter() - t0)
        clk = clocks.stop()
        conv = [bool(r.converged) for r in res]
        sz = s.sizes()
    value = float(np.mean(times))
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 factor, c128 refinement and COCG" if precision == "fp32_ir" else "c128",
            "data": "synthetic (seeded generator; no dataset)",
            "config": {"workload": WORKLOADS["c5"], "precision": precision, "hddm_eps": args.eps,
                       "n_tets": model.n_tets, "n_subdomains": model.nsub, "interface_dofs": sz["total_free"],
                       "sources": len(model.sources), "parallelism": "1 GPU"},
            "iterations_per_source": iters[-1], "converged": conv,
            "per_source_iteration_ms": value * 1e3 / max(1, max(iters[-1])),
            "clocks": clk}
    if adj:
        line["adjoint"] = {"batched_adjoint_s": float(np.mean(adj)), "adjoint_over_forward": float(np.mean(adj)) / value,
                           "adjoint_iterations_per_source": [r.iterations for r in ares],
                           "adjoint_converged": [bool(r.converged) for r in ares],
                           "n_design": int(model.design_tets.shape[0]), "J": [float(v) for v in J],
                           "grad_finite": bool(np.isfinite(ge).all() and np.isfinite(gs).all()),
                           "timing": "host wall time of the batched backward call"}
    print(json.dumps(line))
    return 0


def run_sharded_bench(args, rank, world, local, dist):
    """N > 1: one model sharded over the ranks (contiguous subdomain ranges),
    the partial interface vector summed over NCCL every iteration.  Total
    work is fixed as N grows (strong scaling).  Time per solve: CUDA events on
    each rank around the driver, max over ranks."""
    import torch

    from adventure_fullwave_b200 import shard

    model = make_model(args.config)
    lo, hi = shard.shard_ranges(model, world)[rank]
    opts = dict(hddm_eps=args.eps, hddm_max_loop=args.max_loop, precision=args.precision,
                ir_max_steps=args.ir_steps, ir_tol=args.ir_tol, ir_relax=args.ir_relax,
                solve_kernel=args.solve_kernel, stage_cap=args.stage_cap, stage_warps=args.stage_warps)
    exch = shard.torch_exchange()
    backend = shard.GpuShard(model, (lo, hi), shard.shard_bounds(model, world), device=local, **opts)
    for _ in range(args.warmup):
        shard.run_sharded(backend, exch, 0)
    clocks = ClockSampler(local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    its = []
    for _ in range(args.steps):
        x, it = shard.run_sharded(backend, exch, 0)
        its.append(it)
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = torch.tensor([ev0.elapsed_time(ev1) / 1e3 / args.steps], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = float(t.item())
    backend.close()
    # end to end: shard setup from host arrays, solve, the summed solution on the host
    dist.barrier()
    t0 = time.perf_counter()
    x, _ = shard.sharded_solve(model, 0, rank=rank, world=world, device=local, **opts)
    e2e = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(e2e, op=dist.ReduceOp.MAX)
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return 0
    h2d = sum(a.nbytes for a in (model.vertex_crd, model.tets, model.tet_edges, model.flag, model.pec_edge,
                                 model.sub_of_tet, model.mat_flag, model.mat_eps, model.mat_sigma))
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
        "dtype": "c128" if args.precision == "fp64" else "c64 factor, c128 refinement and COCG",
        "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": WORKLOADS.get(args.config, args.config), "precision": args.precision,
                   "hddm_eps": args.eps, "n_subdomains": model.nsub,
                   "l2": "inputs larger than L2",
                   "parallelism": f"{world} shards (contiguous subdomain ranges), NCCL all-reduce of the "
                                  f"interface vector per iteration"},
        "iterations": int(np.mean(its)),
        "e2e": {"value": float(e2e.item()), "unit": "s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(model.n_edges * 16)},
        "roofline": None, "cpu_baseline": None, "clocks": clk,
        "gpu_launches": None,
        "solution_check": {"finite": bool(np.all(np.isfinite(x)))},
    }
    print(json.dumps(line))
    return 0


def run_ncu_case(args):
    """A short run for ncu captures: setup, the first solve,
    ``--ncu-iters`` interface iterations launched one by one, the last solve
    and the post step."""
    from adventure_fullwave_b200 import hddm

    model = make_model(args.config)
    with hddm.HddmSolver(model, hddm_eps=args.eps, hddm_max_loop=args.max_loop, precision=args.precision,
                         ir_max_steps=args.ir_steps, ir_tol=args.ir_tol, solve_kernel=args.solve_kernel,
                         stage_cap=args.stage_cap, stage_warps=args.stage_warps) as s:
        s.make_tmp_aij(0)
        s.solve_dom_1st()
        s.iteration_s_1st()
        for _ in range(args.ncu_iters):
            s.iteration_s()
        s.solve_dom_last()
        s.post_em_E()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--c5-fp64", action="store_true", help="C5 in FP64 (default: FP32 factors + FP64 refinement)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_ir"])
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--max-loop", type=int, default=50000)
    ap.add_argument("--ir-steps", type=int, default=1)
    ap.add_argument("--ir-tol", type=float, default=0.0)
    ap.add_argument("--ir-relax", type=float, default=0.0, help="refine only while the COCG residual is above this")
    ap.add_argument("--no-mixed", action="store_true", help="skip the FP32+IR comparison solve")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the C4 adjoint sample of a C2 run")
    ap.add_argument("--no-post", action="store_true", help="skip the post-step measurement")
    ap.add_argument("--no-sample", action="store_true", help="skip the reference's shipped sample model")
    ap.add_argument("--no-c2", action="store_true", help="skip the C2 solve of a run on another model")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the C1 solves against the direct solution")
    ap.add_argument("--mixed-steps", type=int, default=1, help="timed FP32+IR solves (after one untimed)")
    ap.add_argument("--replicas", action="store_true", help="N > 1: independent replicas instead of shards")
    ap.add_argument("--sharded", action="store_true", help="the sharded driver even at N = 1 (one shard)")
    ap.add_argument("--graph-iters", type=int, default=32)
    ap.add_argument("--solve-kernel", default="auto", choices=["auto", "warp", "cta", "global"])
    ap.add_argument("--stage-cap", type=int, default=0, help="staging buffer elements (0: timed choice)")
    ap.add_argument("--stage-warps", type=int, default=0, help="warps per subdomain, 1, 2 or 4 (0: timed choice)")
    ap.add_argument("--prof-reps", type=int, default=50)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--ref-iters", type=int, default=1, help="timed reference iterations of the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="bench", choices=["bench", "ncu"])
    ap.add_argument("--ncu-iters", type=int, default=20)
    args = ap.parse_args()
    if args.mode == "ncu":
        return run_ncu_case(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "c5":
        return run_c5(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
