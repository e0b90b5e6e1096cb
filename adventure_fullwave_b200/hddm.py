"""Host API of the B200 HDDM hot path, shaped after the reference's solver
interface.

The reference drives one full-wave solve through ``hddm_solver_CS(pm,
options, set_hddm_func_fullwave)`` (``lib/hddm/hddm_solver.h:25-183``), which
walks the plug-in table ``HDDM_FUNC`` (``lib/std/types.h:629-730``) slot by
slot for every (part, subdomain).  ``HddmSolver`` exposes the same slots,
each batched over all subdomains on the GPU (``make_tmp_aij``,
``solve_dom_1st``, ``iteration_s_1st``, ``iteration_s``, ``solve_dom_last``),
and ``hddm_solver_CS`` runs the whole loop like the reference's driver.

Options keep the reference's names and meaning: ``hddm_eps`` is the
max-norm relative interface residual at which COCG stops (``-hddm-eps``,
default 1e-3), ``hddm_max_loop`` caps the iterations (``-hddm-max-loop``,
default 4000).  Errors are raised as ``FwgpuError`` instead of the
reference's print-and-exit.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import FwgpuError  # noqa: F401  (re-exported)

# batched subdomain-solve kernels (FWGPU_SOLVE_*); "auto" times the candidates once
SOLVE_KERNELS = {"auto": 0, "warp": 1, "cta": 2, "global": 3, "blockinv": 4}
_KERNEL_NAMES = {v: k for k, v in SOLVE_KERNELS.items()}

P = ctypes.POINTER


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(P(ctype))


@dataclass
class HddmResult:
    iterations: int
    converged: bool
    initial_norm: float
    final_resi: float
    final_resi_l2: float
    t_setup_ms: float
    t_iterate_ms: float
    t_last_ms: float
    kernel_launches: int = 0
    solve_kernel: str = ""
    stage_cap: int = 0
    stage_warps: int = 0


def _mesh_struct(model):
    a = {}
    a["crd"] = np.ascontiguousarray(model.vertex_crd, dtype=np.float64)
    a["tv"] = np.ascontiguousarray(model.tets, dtype=np.int32)
    a["te"] = np.ascontiguousarray(model.tet_edges, dtype=np.int32)
    a["flag"] = np.ascontiguousarray(model.flag, dtype=np.int32)
    a["pec"] = np.ascontiguousarray(model.pec_edge, dtype=np.uint8)
    a["sub"] = np.ascontiguousarray(model.sub_of_tet, dtype=np.int32)
    order = [None] * 4
    so = getattr(model, "sub_order", None)
    if so is not None:
        for k, v in enumerate(so):
            a[f"ord{k}"] = np.ascontiguousarray(v, dtype=np.int32)
            order[k] = _ptr(a[f"ord{k}"], ctypes.c_int32)
    mesh = _lib.FwMesh(
        int(a["crd"].shape[0]), _ptr(a["crd"], ctypes.c_double), int(a["tv"].shape[0]),
        _ptr(a["tv"], ctypes.c_int32), _ptr(a["te"], ctypes.c_int32), _ptr(a["flag"], ctypes.c_int32),
        int(a["pec"].shape[0]), _ptr(a["pec"], ctypes.c_uint8), int(model.nsub), _ptr(a["sub"], ctypes.c_int32),
        *order)
    return mesh, a


def _maps(fn, handle, s: int) -> dict:
    nel, nmp, nbc, ninbc = (ctypes.c_int32() for _ in range(4))
    _lib.check(fn(handle, s, ctypes.byref(nel), ctypes.byref(nmp), ctypes.byref(nbc), ctypes.byref(ninbc), None,
                  None, None, None, None))
    nop = np.zeros(10 * nel.value, np.int32)
    ibc = np.zeros(max(1, nbc.value), np.int32)
    nf = np.zeros(max(1, ninbc.value), np.int32)
    ln = np.zeros(max(1, ninbc.value), np.int32)
    gid = np.zeros(max(1, nmp.value), np.int32)
    i32 = ctypes.c_int32
    _lib.check(fn(handle, s, None, None, None, None, _ptr(nop, i32), _ptr(ibc, i32), _ptr(nf, i32), _ptr(ln, i32),
                  _ptr(gid, i32)))
    return dict(nel=nel.value, nmp=nmp.value, nop=nop.reshape(-1, 10), ibc=ibc[: nbc.value],
                inbc_nfid=nf[: ninbc.value], inbc_ln_part=ln[: ninbc.value], edge_gid=gid[: nmp.value])


class Partition:
    """Host-only integer setup (the reference's make_PartMesh_FW for one
    part): subdomain-local numbering, Dirichlet lists and interface maps.
    Needs no GPU."""

    def __init__(self, model):
        self._lib = _lib.load()
        mesh, keep = _mesh_struct(model)
        h = ctypes.c_void_p()
        _lib.check(self._lib.fwgpu_partition_build(ctypes.byref(mesh), ctypes.byref(h)))
        self._h = h
        ns, tf = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.fwgpu_partition_info(h, ctypes.byref(ns), ctypes.byref(tf)))
        self.n_subdomains = ns.value
        self.total_free = tf.value

    def maps(self, s: int) -> dict:
        return _maps(self._lib.fwgpu_partition_maps, self._h, s)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.fwgpu_partition_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HddmSolver:
    """All subdomains of one full-wave model resident on one GPU.

    ``model`` is an ``adventure_fullwave_b200.meshgen.Model`` (or any object
    with the same fields).  ``precision`` is ``"fp64"`` (the reference's
    complex FP64 skyline factors) or ``"fp32_ir"`` (factors stored and
    applied in complex FP32, FP64 iterative refinement of every subdomain
    solve).
    """

    def __init__(self, model, hddm_eps: float = 1e-3, hddm_max_loop: int = 4000, precision: str = "fp64",
                 ir_max_steps: int = 1, ir_tol: float = 0.0, graph_iterations: int = 16, device: int = 0,
                 solve_kernel: str = "auto", stage_cap: int = 0, ir_relax: float = 0.0,
                 shard: Optional[Tuple[int, int]] = None, stage_warps: int = 0, stall_copy_test: int = 0):
        lib = _lib.load()
        self._lib = lib
        self.model = model
        self.hddm_eps = float(hddm_eps)
        self.hddm_max_loop = int(hddm_max_loop)
        mesh, a = _mesh_struct(model)
        a["mf"] = np.ascontiguousarray(model.mat_flag, dtype=np.int32)
        a["me"] = np.ascontiguousarray(model.mat_eps, dtype=np.float64)
        a["ms"] = np.ascontiguousarray(model.mat_sigma, dtype=np.float64)
        a["ef"], a["sf"] = a["mf"], a["mf"]
        if getattr(model, "eps_table", None) is not None:
            a["ef"] = np.ascontiguousarray(model.eps_table[0], dtype=np.int32)
            a["me"] = np.ascontiguousarray(model.eps_table[1], dtype=np.float64)
        if getattr(model, "sigma_table", None) is not None:
            a["sf"] = np.ascontiguousarray(model.sigma_table[0], dtype=np.int32)
            a["ms"] = np.ascontiguousarray(model.sigma_table[1], dtype=np.float64)
        mt = _lib.FwMaterial(int(a["ef"].shape[0]), _ptr(a["ef"], ctypes.c_int32), _ptr(a["me"], ctypes.c_double),
                             int(a["sf"].shape[0]), _ptr(a["sf"], ctypes.c_int32), _ptr(a["ms"], ctypes.c_double),
                             float(model.omega))
        prec = {"fp64": _lib.PREC_FP64, "fp32_ir": _lib.PREC_FP32_IR}[precision]
        self.precision = precision
        kern = SOLVE_KERNELS[solve_kernel]
        opts = _lib.FwOptions(self.hddm_eps, self.hddm_max_loop, prec, int(ir_max_steps), float(ir_tol),
                              int(graph_iterations), int(device), kern, int(stage_cap), float(ir_relax),
                              int(shard[0]) if shard else 0, int(shard[1]) if shard else 0, int(stage_warps),
                              int(stall_copy_test))
        handle = ctypes.c_void_p()
        rc = lib.fwgpu_create(ctypes.byref(mesh), ctypes.byref(mt), ctypes.byref(opts), ctypes.byref(handle))
        if rc != 0 and handle.value:
            lib.fwgpu_destroy(handle)
        _lib.check(rc)
        self._h = handle
        self._multi_n = 0
        self.n_edges = int(model.n_edges)
        self.n_tets = int(model.n_tets)
        if getattr(model, "element_source", None) is not None:
            self.set_element_source(model.element_source)

    # -- lifecycle --------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.fwgpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- sources -----------------------------------------------------------
    def _source(self, source) -> Tuple[_lib.FwSource, tuple]:
        if source is None:
            return _lib.FwSource(0, None, None), ()
        if isinstance(source, int):
            edges, vals = self.model.sources[source]
        else:
            edges, vals = source
        e = np.ascontiguousarray(edges, dtype=np.int32)
        v = np.ascontiguousarray(np.stack([np.real(vals), np.imag(vals)], axis=1).ravel(), dtype=np.float64)
        return _lib.FwSource(int(e.shape[0]), _ptr(e, ctypes.c_int32), _ptr(v, ctypes.c_double)), (e, v)

    def set_element_source(self, es) -> None:
        """Delta-gap voltages or antenna currents (``meshgen.ElementSource``)
        added to every later right-hand side; None clears them."""
        if es is None:
            _lib.check(self._lib.fwgpu_set_element_source(self._h, None))
            return
        box = np.ascontiguousarray(es.gap_box, np.float64).reshape(-1)
        volt = np.ascontiguousarray(es.gap_volt, np.float64)
        flags = np.ascontiguousarray(es.antenna_flag, np.int32)
        jo = np.ascontiguousarray(es.antenna_Jo, np.float64).reshape(-1)
        jor = np.ascontiguousarray(es.antenna_Jor, np.float64).reshape(-1)
        if es.n_antennas and jo.shape[0] != 3 * self.model.n_vertices * es.n_antennas:
            raise ValueError("antenna currents need 3 values per vertex per antenna")
        c = _lib.FwElementSource(int(es.n_gaps), _ptr(box, ctypes.c_double), _ptr(volt, ctypes.c_double),
                                 int(es.n_antennas), _ptr(flags, ctypes.c_int32), _ptr(jo, ctypes.c_double),
                                 _ptr(jor, ctypes.c_double))
        _lib.check(self._lib.fwgpu_set_element_source(self._h, ctypes.byref(c)))

    # -- the reference's plug-in slots, batched ----------------------------
    def make_tmp_aij(self, source=0) -> None:
        src, keep = self._source(source)
        _lib.check(self._lib.fwgpu_make_tmp_aij(self._h, ctypes.byref(src)))

    def solve_dom_1st(self) -> None:
        _lib.check(self._lib.fwgpu_solve_dom_1st(self._h))

    def iteration_s_1st(self) -> int:
        st = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_iteration_s_1st(self._h, ctypes.byref(st)))
        return st.value

    def iteration_s(self) -> int:
        st = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_iteration_s(self._h, ctypes.byref(st)))
        return st.value

    def solve_dom_last(self) -> None:
        _lib.check(self._lib.fwgpu_solve_dom_last(self._h))

    # -- batched driver ----------------------------------------------------
    def solve(self, source=0, raise_not_converged: bool = False) -> HddmResult:
        src, keep = self._source(source)
        res = _lib.FwResult()
        allow = () if raise_not_converged else (_lib.ERR_NOT_CONVERGED,)
        _lib.check(self._lib.fwgpu_hddm_solve(self._h, ctypes.byref(src), ctypes.byref(res)), allow=allow)
        return self._result(res)

    def solve_multi(self, sources: Sequence, raise_not_converged: bool = False) -> list:
        """Up to 16 sources solved together on one set of factors (one
        assembly, one factorisation, the sources' COCGs in lockstep).
        Returns one result per source; ``edge_solution_multi(k)`` gives
        source k's solution."""
        srcs = [self._source(s) for s in sources]
        if not 1 <= len(srcs) <= _lib.MAX_RHS:
            raise ValueError(f"1 to {_lib.MAX_RHS} sources")
        arr = (_lib.FwSource * len(srcs))(*[s for s, _ in srcs])
        res = (_lib.FwResult * len(srcs))()
        allow = () if raise_not_converged else (_lib.ERR_NOT_CONVERGED,)
        self._multi_n = 0
        _lib.check(self._lib.fwgpu_hddm_solve_multi(self._h, len(srcs), arr, res), allow=allow)
        self._multi_n = len(srcs)
        return [self._result(r) for r in res]

    def edge_solution_multi(self, k: int) -> np.ndarray:
        x = np.zeros(2 * self.n_edges, dtype=np.float64)
        _lib.check(self._lib.fwgpu_get_edge_solution_multi(self._h, int(k), _ptr(x, ctypes.c_double)))
        return x[0::2] + 1j * x[1::2]

    def resolve(self, source, raise_not_converged: bool = False) -> HddmResult:
        src, keep = self._source(source)
        res = _lib.FwResult()
        allow = () if raise_not_converged else (_lib.ERR_NOT_CONVERGED,)
        _lib.check(self._lib.fwgpu_hddm_resolve(self._h, ctypes.byref(src), ctypes.byref(res)), allow=allow)
        return self._result(res)

    @staticmethod
    def _result(r: _lib.FwResult) -> HddmResult:
        return HddmResult(int(r.iterations), bool(r.converged), float(r.initial_norm), float(r.final_resi),
                          float(r.final_resi_l2), float(r.t_setup_ms), float(r.t_iterate_ms), float(r.t_last_ms),
                          int(r.kernel_launches), _KERNEL_NAMES.get(int(r.solve_kernel), ""),
                          int(r.stage_cap), int(r.stage_warps))

    def adjoint_gradient(self, probe_edges=None, design_tets=None):
        """Backward of the last ``solve``: J = sum |x_p|^2 over ``probe_edges``
        and its gradient with respect to the permittivity eps [F/m] and
        conductivity sigma [S/m] of every element of ``design_tets``, by one
        adjoint HDDM solve on the same factors.  Returns
        (J, dJ/deps, dJ/dsigma, adjoint HddmResult)."""
        pe = np.ascontiguousarray(self.model.probe_edges if probe_edges is None else probe_edges, dtype=np.int32)
        dt = np.ascontiguousarray(self.model.design_tets if design_tets is None else design_tets, dtype=np.int32)
        ge = np.zeros(max(1, dt.shape[0]), np.float64)
        gs = np.zeros(max(1, dt.shape[0]), np.float64)
        J = ctypes.c_double()
        res = _lib.FwResult()
        _lib.check(self._lib.fwgpu_adjoint_gradient(self._h, int(pe.shape[0]), _ptr(pe, ctypes.c_int32),
                                                    int(dt.shape[0]), _ptr(dt, ctypes.c_int32), ctypes.byref(J),
                                                    _ptr(ge, ctypes.c_double), _ptr(gs, ctypes.c_double),
                                                    ctypes.byref(res)), allow=(_lib.ERR_NOT_CONVERGED,))
        n = dt.shape[0]
        return J.value, ge[:n], gs[:n], self._result(res)

    def adjoint_gradient_multi(self, probe_edges=None, design_tets=None):
        """Backward of the last ``solve_multi`` for every source at once: the
        adjoint right-hand sides of all sources in one batched solve on the
        same factors.  Returns (J (n_src,), dJ/deps (n_src, n_design),
        dJ/dsigma (n_src, n_design), adjoint HddmResults)."""
        pe = np.ascontiguousarray(self.model.probe_edges if probe_edges is None else probe_edges, dtype=np.int32)
        dt = np.ascontiguousarray(self.model.design_tets if design_tets is None else design_tets, dtype=np.int32)
        ns = _lib.MAX_RHS
        J = np.zeros(ns, np.float64)
        ge = np.zeros(ns * max(1, dt.shape[0]), np.float64)
        gs = np.zeros(ns * max(1, dt.shape[0]), np.float64)
        res = (_lib.FwResult * ns)()
        _lib.check(self._lib.fwgpu_adjoint_gradient_multi(self._h, int(pe.shape[0]), _ptr(pe, ctypes.c_int32),
                                                          int(dt.shape[0]), _ptr(dt, ctypes.c_int32),
                                                          _ptr(J, ctypes.c_double), _ptr(ge, ctypes.c_double),
                                                          _ptr(gs, ctypes.c_double), res),
                   allow=(_lib.ERR_NOT_CONVERGED,))
        n = self._multi_n
        nd = dt.shape[0]
        return (J[:n], ge[:n * nd].reshape(n, nd), gs[:n * nd].reshape(n, nd), [self._result(r) for r in res[:n]])

    def profile_iteration(self, reps: int = 50) -> dict:
        """Average device time of the kernels of one interface iteration
        (CUDA events on the solver's stream).  Overwrites the iteration
        state: call ``resolve`` afterwards for a solution."""
        prof = _lib.FwKernelProfile()
        _lib.check(self._lib.fwgpu_profile_iteration(self._h, int(reps), ctypes.byref(prof)))
        return dict(subsolve_ms=prof.subsolve_ms, interface_ms=prof.interface_ms, iteration_ms=prof.iteration_ms,
                    reps=prof.reps)

    # -- post step -----------------------------------------------------------
    def post_em_E(self, x=None):
        """Element results of the post step (``HDDM_post_em_E``,
        ``main/fullwave/fullwave.c:639-763``) from the edge solution ``x``
        (complex, n_edges; None: the last solution): (B, E, Je), each
        (n_tets, 3) complex in global element order, where B is
        i (nu/omega) rot E, E the field at the centroid and Je = sigma E, all
        three from the edge values scaled by nu/omega as the reference does."""
        xin = None
        if x is not None:
            x = np.asarray(x)
            if x.shape != (self.n_edges,):
                raise ValueError("x needs one value per edge")
            xin = np.ascontiguousarray(np.stack([x.real, x.imag], 1).ravel(), np.float64)
        outs = [np.zeros(6 * self.n_tets, np.float64) for _ in range(3)]
        _lib.check(self._lib.fwgpu_post_em_E(self._h, None if xin is None else _ptr(xin, ctypes.c_double),
                                             *[_ptr(o, ctypes.c_double) for o in outs]))
        return tuple((o[0::2] + 1j * o[1::2]).reshape(self.n_tets, 3) for o in outs)

    def post_em_E_into(self, x_ptr: int, b_ptr: int, e_ptr: int, je_ptr: int) -> None:
        """``post_em_E`` on raw pointers (host memory or 16-byte aligned
        device memory of the solver's device; 0 for the last solution or to
        skip a result), e.g. ``tensor.data_ptr()`` of CUDA tensors, so that
        the results stay on the device."""
        ptrs = [ctypes.c_void_p(int(p)) if p else None for p in (x_ptr, b_ptr, e_ptr, je_ptr)]
        _lib.check(self._lib.fwgpu_post_em_E(self._h, *ptrs))

    def profile_post(self, reps: int = 20) -> float:
        """Average device time [ms] of one post-step kernel launch, L2
        evicted before each launch."""
        ms = ctypes.c_double()
        _lib.check(self._lib.fwgpu_profile_post(self._h, int(reps), ctypes.byref(ms)))
        return ms.value

    # -- sharded solve (one context per rank) --------------------------------
    def shard_set_layout(self, shard_first) -> int:
        """The subdomain ranges of all shards (``shard_first``: n_shards+1
        boundaries); returns the number of interface DOFs held by two or
        more shards, the length of the packed exchange."""
        f = np.ascontiguousarray(shard_first, dtype=np.int32)
        n = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_shard_set_layout(self._h, int(f.shape[0] - 1), _ptr(f, ctypes.c_int32),
                                                     ctypes.byref(n)))
        return n.value

    def shard_set_exchange(self, pack_ptr: int, scal_ptr: int) -> None:
        """Device buffers: 4*n_shared doubles (packed Q and diagonal) and 8
        doubles (scalars)."""
        _lib.check(self._lib.fwgpu_shard_set_exchange(self._h, ctypes.c_void_p(int(pack_ptr)),
                                                      ctypes.c_void_p(int(scal_ptr))))

    def shard_first(self) -> None:
        _lib.check(self._lib.fwgpu_shard_first(self._h))

    def shard_first_sums(self) -> None:
        _lib.check(self._lib.fwgpu_shard_first_sums(self._h))

    def shard_iterate_pq(self) -> None:
        _lib.check(self._lib.fwgpu_shard_iterate_pq(self._h))

    def shard_iterate_update(self) -> None:
        _lib.check(self._lib.fwgpu_shard_iterate_update(self._h))

    def shard_first_finish(self) -> int:
        st = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_shard_first_finish(self._h, ctypes.byref(st)))
        return st.value

    def shard_iterate(self) -> None:
        _lib.check(self._lib.fwgpu_shard_iterate(self._h))

    def shard_iterate_finish(self) -> int:
        st = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_shard_iterate_finish(self._h, ctypes.byref(st)))
        return st.value

    # -- results -----------------------------------------------------------
    def edge_solution(self) -> np.ndarray:
        x = np.zeros(2 * self.n_edges, dtype=np.float64)
        _lib.check(self._lib.fwgpu_get_edge_solution(self._h, _ptr(x, ctypes.c_double)))
        return x[0::2] + 1j * x[1::2]

    def history(self) -> np.ndarray:
        n = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_get_history(self._h, None, 0, ctypes.byref(n)))
        h = np.zeros(max(1, n.value), dtype=np.float64)
        _lib.check(self._lib.fwgpu_get_history(self._h, _ptr(h, ctypes.c_double), n.value, ctypes.byref(n)))
        return h[: n.value]

    def write_calc_log(self, path: str, result: "HddmResult", mode: str = "a") -> None:
        """Append (or write, mode "w") the last solve's residual history to
        ``path`` as the reference's calc_log section (``calc_log_section``)."""
        with open(path, mode) as f:
            f.write(calc_log_section(self.sizes()["total_free"], result.initial_norm, self.history()))

    def sizes(self) -> dict:
        s = _lib.FwSizes()
        _lib.check(self._lib.fwgpu_get_sizes(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in _lib.FwSizes._fields_}

    # -- introspection -----------------------------------------------------
    def subdomain_maps(self, s: int) -> dict:
        return _maps(self._lib.fwgpu_get_subdomain_maps, self._h, s)

    def skyline_profile(self, s: int) -> Tuple[np.ndarray, np.ndarray, int]:
        nmp = self.subdomain_maps(s)["nmp"]
        idx1 = np.zeros(nmp, np.int32)
        idx2 = np.zeros(nmp, np.int32)
        nlen = ctypes.c_int32()
        i32 = ctypes.c_int32
        _lib.check(self._lib.fwgpu_get_skyline_profile(self._h, s, _ptr(idx1, i32), _ptr(idx2, i32),
                                                       ctypes.byref(nlen)))
        return idx1, idx2, nlen.value

    def tmp_aij(self, s: int):
        nmp = self.subdomain_maps(s)["nmp"]
        nnz = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_get_tmp_aij(self._h, s, ctypes.byref(nnz), None, None, None, None))
        rp = np.zeros(nmp + 1, np.int32)
        col = np.zeros(max(1, nnz.value), np.int32)
        val = np.zeros(2 * max(1, nnz.value), np.float64)
        b = np.zeros(2 * nmp, np.float64)
        i32 = ctypes.c_int32
        _lib.check(self._lib.fwgpu_get_tmp_aij(self._h, s, ctypes.byref(nnz), _ptr(rp, i32), _ptr(col, i32),
                                               _ptr(val, ctypes.c_double), _ptr(b, ctypes.c_double)))
        n = nnz.value
        return rp, col[:n], val[0:2 * n:2] + 1j * val[1:2 * n:2], b[0::2] + 1j * b[1::2]

    def factor(self, s: int) -> np.ndarray:
        idx1, idx2, nlen = self.skyline_profile(s)
        m = np.zeros(2 * nlen, np.float64)
        _lib.check(self._lib.fwgpu_get_factor(self._h, s, _ptr(m, ctypes.c_double)))
        return m[0::2] + 1j * m[1::2]


def calc_log_section(total_free: int, initial_norm: float, history) -> str:
    """The full-wave section of the reference's convergence log
    (calc_log/log_g_HDDM_Full_Wave): two blank lines and the title
    (HDDM_set_HDDM_Opt_log, lib/hddm/set_hddm_func.c:37-51), the interface
    DOF count (lib/hddm/hddm_solver.h:88-92), the initial line with the
    max-norm of r0 (lib/hddm/hddm_solver_s.h:203-207) and one line
    "iteration resi" per interface iteration (:319-323), in the reference's
    printf formats."""
    lines = ["", "", "# Full Wave Analysis", f"# DOF on interface {int(total_free)}",
             f"0 {1.0:e}  # Norm {float(initial_norm):e}"]
    lines += [f"{k} {float(r):e}" for k, r in enumerate(history, 1)]
    return "\n".join(lines) + "\n"


def relative_permittivity_gradient(g_eps: np.ndarray, g_sigma: np.ndarray, omega: float, eps0: float = 8.854e-12):
    """Gradient with respect to eps_r = eps' - i eps'' of each design element
    (eps = eps0 eps', sigma = omega eps0 eps''): (dJ/deps', dJ/deps'')."""
    return eps0 * np.asarray(g_eps), omega * eps0 * np.asarray(g_sigma)


def hddm_solver_CS(model, source=0, **opts) -> Tuple[np.ndarray, HddmResult]:
    """One full-wave HDDM solve (the reference's ``hddm_solver_CS`` with
    ``set_hddm_func_fullwave``); returns the edge solution and the result."""
    with HddmSolver(model, **opts) as s:
        r = s.solve(source)
        return s.edge_solution(), r


# -- correction-Jo pre-solve ---------------------------------------------------

def _pec_vertex(model, pec_vertex):
    if pec_vertex is None:
        # the model's own Dirichlet vertices (advio.load_model reads them)
        pec_vertex = getattr(model, "pec_vertex", None)
    if pec_vertex is None:
        return None, None
    a = np.ascontiguousarray(pec_vertex, dtype=np.uint8)
    if a.shape != (int(model.n_vertices),):
        raise ValueError("pec_vertex must hold one flag per vertex")
    return a, a.ctypes.data_as(ctypes.c_void_p)


class CorrectJoPartition:
    """Host-only integer setup of one antenna's correction-Jo problem (the
    ANTENNA part of the reference's make_PartMesh_FW,
    lib/hddm/make_PartMesh.c:973-1063,1288-1340,1546-1575): per subdomain
    holding antenna elements, its vertex DOFs, Dirichlet list and interface
    entries.  Needs no GPU."""

    def __init__(self, model, antenna_flag: int, pec_vertex=None):
        self._lib = _lib.load()
        mesh, keep = _mesh_struct(model)
        pv, pv_ptr = _pec_vertex(model, pec_vertex)
        h = ctypes.c_void_p()
        _lib.check(self._lib.fwgpu_cojo_partition_build(ctypes.byref(mesh), int(antenna_flag), pv_ptr,
                                                        ctypes.byref(h)))
        self._h = h
        ns, tf = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.fwgpu_partition_info(h, ctypes.byref(ns), ctypes.byref(tf)))
        self.n_subdomains = ns.value
        self.total_free = tf.value
        ids = np.zeros(max(1, ns.value), np.int32)
        _lib.check(self._lib.fwgpu_cojo_partition_subdomains(h, _ptr(ids, ctypes.c_int32)))
        self.subdomain_ids = ids[: ns.value]

    def maps(self, s: int) -> dict:
        """Maps of the problem's subdomain s: ``edge_gid`` holds the global
        vertex of each local DOF (the reference's enf order)."""
        return _maps(self._lib.fwgpu_partition_maps, self._h, s)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.fwgpu_partition_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CorrectJoSolver:
    """The correction-Jo pre-solve of one antenna on one GPU: the reference's
    ``hddm_solver_RS`` with ``set_hddm_func_correct_Jor`` and then
    ``set_hddm_func_correct_Joi`` (main/fullwave/main.c:92-98,
    lib/hddm/set_hddm_func.c:90-233).  A real-symmetric HDDM for a potential
    at the vertices of the antenna's elements, stiffness (grad, grad) and
    right-hand side (J, grad N_i) of the vertex currents J
    (lib/fem/make_elem.c:10-66), interface PCG with the diagonal
    preconditioner.  ``hddm_eps`` and ``hddm_max_loop`` are the reference's
    coJo-hddm-eps (1e-10) and coJo-hddm-max-loop (4000).  One ``solve`` per
    pass; the second reuses the factors."""

    def __init__(self, model, antenna_flag: int, hddm_eps: float = 1e-10, hddm_max_loop: int = 4000,
                 pec_vertex=None, graph_iterations: int = 16, device: int = 0, solve_kernel: str = "auto"):
        lib = _lib.load()
        self._lib = lib
        self.model = model
        self.antenna_flag = int(antenna_flag)
        self.n_vertices = int(model.n_vertices)
        mesh, keep = _mesh_struct(model)
        pv, pv_ptr = _pec_vertex(model, pec_vertex)
        opts = _lib.FwOptions(float(hddm_eps), int(hddm_max_loop), _lib.PREC_FP64, 1, 0.0, int(graph_iterations),
                              int(device), SOLVE_KERNELS[solve_kernel], 0, 0.0, 0, 0, 0, 0)
        handle = ctypes.c_void_p()
        rc = lib.fwgpu_cojo_create(ctypes.byref(mesh), self.antenna_flag, pv_ptr, ctypes.byref(opts),
                                   ctypes.byref(handle))
        if rc != 0 and handle.value:
            lib.fwgpu_destroy(handle)
        _lib.check(rc)
        self._h = handle

    def solve(self, current, raise_not_converged: bool = False) -> Tuple[np.ndarray, HddmResult]:
        """One pass with the vertex currents ``current`` (n_vertices x 3):
        the potential at every vertex (0 off the antenna) and the result."""
        j = np.ascontiguousarray(current, dtype=np.float64)
        if j.shape != (self.n_vertices, 3):
            raise ValueError("current must be n_vertices x 3")
        phi = np.zeros(self.n_vertices, np.float64)
        r = _lib.FwResult()
        rc = self._lib.fwgpu_cojo_solve(self._h, _ptr(j, ctypes.c_double), ctypes.byref(r), _ptr(phi, ctypes.c_double))
        _lib.check(rc, () if raise_not_converged else (_lib.ERR_NOT_CONVERGED,))
        return phi, HddmSolver._result(r)

    def history(self) -> np.ndarray:
        return HddmSolver.history(self)

    def sizes(self) -> dict:
        return HddmSolver.sizes(self)

    def write_calc_log(self, path: str, result: HddmResult, part: str, antenna: int = 0, mode: str = "a") -> None:
        """Append (or write, mode "w") the last pass's residual history as
        the reference's correction-Jo log section; part is "Real" or
        "Imaginary" (correct_jo_log_section)."""
        with open(path, mode) as f:
            f.write(correct_jo_log_section(part, antenna, self.sizes()["total_free"], result.initial_norm,
                                           self.history()))

    def subdomain_ids(self) -> np.ndarray:
        n = ctypes.c_int32()
        _lib.check(self._lib.fwgpu_cojo_subdomains(self._h, ctypes.byref(n), None))
        ids = np.zeros(max(1, n.value), np.int32)
        _lib.check(self._lib.fwgpu_cojo_subdomains(self._h, ctypes.byref(n), _ptr(ids, ctypes.c_int32)))
        return ids[: n.value]

    def subdomain_maps(self, s: int) -> dict:
        return _maps(self._lib.fwgpu_get_subdomain_maps, self._h, s)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.fwgpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def correct_jo_log_section(part: str, antenna: int, total_free: int, initial_norm: float, history) -> str:
    """One correction-Jo section of the reference's convergence log: title
    "Correction Jo : Real part" or "Imaginary part"
    (HDDM_set_HDDM_Opt_correct_Jor/Joi, lib/hddm/set_hddm_func.c:266-298),
    the antenna number, then the lines calc_log_section writes."""
    body = calc_log_section(total_free, initial_norm, history).split("\n")[3:]
    lines = ["", "", f"# Correction Jo : {part} part", "", f"#   Antenna number = {int(antenna)}"] + body
    return "\n".join(lines)


def hddm_solver_RS_correct_jo(model, k: int = 0, **opts):
    """main()'s pre-solve for antenna k of ``model.element_source``: the pass
    on the real part of the currents (Jor), then on the imaginary part (Jo).
    Returns (Ihr, Ihi) per vertex and the two results."""
    es = model.element_source
    with CorrectJoSolver(model, int(es.antenna_flag[k]), **opts) as s:
        ihr, rr = s.solve(es.antenna_Jor[k])
        ihi, ri = s.solve(es.antenna_Jo[k])
    return ihr, ihi, (rr, ri)
