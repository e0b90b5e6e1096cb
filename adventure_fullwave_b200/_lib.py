"""ctypes binding of the C ABI in ``include/fwgpu.h`` (``libfwgpu.so``).

The library is loaded from this package directory.  There is no fallback:
if the shared library is missing the import of the solver fails loudly, and
without a CUDA device every call that needs the GPU returns
``FWGPU_ERR_CUDA``, which is raised as ``FwgpuError``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfwgpu.so")

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_STATE = -3
ERR_NOT_CONVERGED = -4
ERR_BREAKDOWN = -5
ERR_NOMEM = -6
ERR_MESH = -7
ERR_NONFINITE = -8
ERR_TIMEOUT = -9
NOALLOC_MAX_ROWS = 262144

PREC_FP64 = 0
PREC_FP32_IR = 1
MAX_RHS = 16

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
P = ctypes.POINTER


class FwMesh(ctypes.Structure):
    _fields_ = [
        ("n_vertices", c_i32), ("vertex_crd", P(c_dbl)),
        ("n_tets", c_i32), ("tet_vertices", P(c_i32)), ("tet_edges", P(c_i32)), ("tet_flag", P(c_i32)),
        ("n_edges", c_i32), ("pec_edge", P(ctypes.c_uint8)),
        ("n_subdomains", c_i32), ("sub_of_tet", P(c_i32)),
        ("sub_vertex_ptr", P(c_i32)), ("sub_vertex_order", P(c_i32)),
        ("sub_edge_ptr", P(c_i32)), ("sub_edge_order", P(c_i32)),
    ]


class FwMaterial(ctypes.Structure):
    _fields_ = [
        ("n_eps", c_i32), ("eps_flag", P(c_i32)), ("eps", P(c_dbl)),
        ("n_sigma", c_i32), ("sigma_flag", P(c_i32)), ("sigma", P(c_dbl)),
        ("omega", c_dbl),
    ]


class FwSource(ctypes.Structure):
    _fields_ = [("n_entries", c_i32), ("edge", P(c_i32)), ("value", P(c_dbl))]


class FwElementSource(ctypes.Structure):
    _fields_ = [("n_gaps", c_i32), ("gap_box", P(c_dbl)), ("gap_volt", P(c_dbl)), ("n_antennas", c_i32),
                ("antenna_flag", P(c_i32)), ("antenna_Jo", P(c_dbl)), ("antenna_Jor", P(c_dbl))]


class FwOptions(ctypes.Structure):
    _fields_ = [
        ("hddm_eps", c_dbl), ("hddm_max_loop", c_i32), ("precision", c_i32), ("ir_max_steps", c_i32),
        ("ir_tol", c_dbl), ("graph_iterations", c_i32), ("device", c_i32), ("solve_kernel", c_i32),
        ("stage_cap", c_i32), ("ir_relax", c_dbl), ("shard_begin", c_i32), ("shard_end", c_i32),
        ("stage_warps", c_i32), ("stall_copy_test", c_i32),
    ]


class FwSizes(ctypes.Structure):
    _fields_ = [
        ("n_subdomains", c_i32), ("total_free", c_i32), ("total_dofs", c_i64), ("total_interior", c_i64),
        ("nlen_reference", c_i64), ("nlen_interior", c_i64), ("nnz_lower", c_i64),
        ("nnz_interface_rows", c_i64), ("nnz_coupling", c_i64), ("nnz_interior", c_i64),
        ("total_iface_slots", c_i64), ("max_local_dofs", c_i32), ("max_interior", c_i32),
    ]


class FwResult(ctypes.Structure):
    _fields_ = [
        ("iterations", c_i32), ("converged", c_i32), ("initial_norm", c_dbl), ("final_resi", c_dbl),
        ("final_resi_l2", c_dbl), ("t_setup_ms", c_dbl), ("t_iterate_ms", c_dbl), ("t_last_ms", c_dbl),
        ("kernel_launches", c_i64), ("solve_kernel", c_i32), ("stage_cap", c_i32),
        ("stage_warps", c_i32), ("reserved", c_i32),
    ]


class FwKernelProfile(ctypes.Structure):
    _fields_ = [("subsolve_ms", c_dbl), ("interface_ms", c_dbl), ("iteration_ms", c_dbl), ("reps", c_i32)]


# every symbol the header declares, with its argument types
SIGNATURES = {
    "fwgpu_create": [P(FwMesh), P(FwMaterial), P(FwOptions), P(ctypes.c_void_p)],
    "fwgpu_destroy": [ctypes.c_void_p],
    "fwgpu_get_sizes": [ctypes.c_void_p, P(FwSizes)],
    "fwgpu_last_error": [],
    "fwgpu_abi_version": [],
    "fwgpu_partition_build": [P(FwMesh), P(ctypes.c_void_p)],
    "fwgpu_partition_destroy": [ctypes.c_void_p],
    "fwgpu_partition_info": [ctypes.c_void_p, P(c_i32), P(c_i32)],
    "fwgpu_partition_maps": [ctypes.c_void_p, c_i32, P(c_i32), P(c_i32), P(c_i32), P(c_i32), P(c_i32),
                             P(c_i32), P(c_i32), P(c_i32), P(c_i32)],
    "fwgpu_make_tmp_aij": [ctypes.c_void_p, P(FwSource)],
    "fwgpu_set_element_source": [ctypes.c_void_p, P(FwElementSource)],
    "fwgpu_solve_dom_1st": [ctypes.c_void_p],
    "fwgpu_iteration_s_1st": [ctypes.c_void_p, P(c_i32)],
    "fwgpu_iteration_s": [ctypes.c_void_p, P(c_i32)],
    "fwgpu_solve_dom_last": [ctypes.c_void_p],
    "fwgpu_hddm_solve": [ctypes.c_void_p, P(FwSource), P(FwResult)],
    "fwgpu_hddm_resolve": [ctypes.c_void_p, P(FwSource), P(FwResult)],
    "fwgpu_profile_iteration": [ctypes.c_void_p, c_i32, P(FwKernelProfile)],
    "fwgpu_adjoint_gradient": [ctypes.c_void_p, c_i32, P(c_i32), c_i32, P(c_i32), P(c_dbl), P(c_dbl), P(c_dbl),
                               P(FwResult)],
    "fwgpu_post_em_E": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fwgpu_profile_post": [ctypes.c_void_p, c_i32, P(c_dbl)],
    "fwgpu_hddm_solve_multi": [ctypes.c_void_p, c_i32, P(FwSource), P(FwResult)],
    "fwgpu_get_edge_solution_multi": [ctypes.c_void_p, c_i32, P(c_dbl)],
    "fwgpu_adjoint_gradient_multi": [ctypes.c_void_p, c_i32, P(c_i32), c_i32, P(c_i32), P(c_dbl), P(c_dbl), P(c_dbl),
                                     P(FwResult)],
    "fwgpu_shard_set_layout": [ctypes.c_void_p, c_i32, P(c_i32), P(c_i32)],
    "fwgpu_shard_set_exchange": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fwgpu_shard_first": [ctypes.c_void_p],
    "fwgpu_shard_first_sums": [ctypes.c_void_p],
    "fwgpu_shard_first_finish": [ctypes.c_void_p, P(c_i32)],
    "fwgpu_shard_iterate": [ctypes.c_void_p],
    "fwgpu_shard_iterate_pq": [ctypes.c_void_p],
    "fwgpu_shard_iterate_update": [ctypes.c_void_p],
    "fwgpu_shard_iterate_finish": [ctypes.c_void_p, P(c_i32)],
    "fwgpu_skyline_solve_noalloc": [c_i32, c_i32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p],
    "fwgpu_cojo_create": [P(FwMesh), c_i32, ctypes.c_void_p, P(FwOptions), P(ctypes.c_void_p)],
    "fwgpu_cojo_solve": [ctypes.c_void_p, P(c_dbl), P(FwResult), P(c_dbl)],
    "fwgpu_cojo_set_current": [ctypes.c_void_p, P(c_dbl)],
    "fwgpu_cojo_subdomains": [ctypes.c_void_p, P(c_i32), P(c_i32)],
    "fwgpu_cojo_partition_build": [P(FwMesh), c_i32, ctypes.c_void_p, P(ctypes.c_void_p)],
    "fwgpu_cojo_partition_subdomains": [ctypes.c_void_p, P(c_i32)],
    "fwgpu_get_edge_solution": [ctypes.c_void_p, P(c_dbl)],
    "fwgpu_get_history": [ctypes.c_void_p, P(c_dbl), c_i32, P(c_i32)],
    "fwgpu_get_subdomain_maps": [ctypes.c_void_p, c_i32, P(c_i32), P(c_i32), P(c_i32), P(c_i32), P(c_i32),
                                 P(c_i32), P(c_i32), P(c_i32), P(c_i32)],
    "fwgpu_get_skyline_profile": [ctypes.c_void_p, c_i32, P(c_i32), P(c_i32), P(c_i32)],
    "fwgpu_get_tmp_aij": [ctypes.c_void_p, c_i32, P(c_i32), P(c_i32), P(c_i32), P(c_dbl), P(c_dbl)],
    "fwgpu_get_factor": [ctypes.c_void_p, c_i32, P(c_dbl)],
}


class FwgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fwgpu error {code}: {msg}")
        self.code = code


_lib = None


def load() -> ctypes.CDLL:
    """Load ``libfwgpu.so`` (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with adventure_fullwave_b200.build.build()")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_char_p if name == "fwgpu_last_error" else ctypes.c_int
    _lib = lib
    return lib


def check(rc: int, allow=()) -> int:
    if rc != OK and rc not in allow:
        raise FwgpuError(rc, load().fwgpu_last_error().decode())
    return rc
