"""FP64 sparse direct solve of the global full-wave system.

TEST INFRASTRUCTURE ONLY (the checker, never the product): it gives the
exact solution of the discrete problem the HDDM solves iteratively, so the
error of an HDDM result can be stated against it rather than against
another iterative run.

The global system is the one every subdomain system is a piece of:
element matrices (nu/omega) RR - eps omega SS + i sigma SS of the restated
element routine (``orc_element_matrix``, bit-identical to the reference's
``tet_MakeElement_EM_E``, ``lib/fem/make_elem_em.c:14-330``) summed over
all elements into one matrix over the global edges (``mymt_CS_AIJ_SetAe``,
``lib/mymt_aij_solver/aij_matrix_func.h:260-326``, without the split into
subdomains), the edge source and element right-hand sides summed the same
way, and the PEC edges eliminated with value 0 (``mymt_CS_AIJ_SetBC``,
``aij_matrix_func.h:60-136``).  The HDDM's interface problem, solved
exactly, gives this same solution, so ``||x_hddm - x_direct|| /
||x_direct||`` is the HDDM result's error.  The sparse LU is SuperLU
through ``scipy.sparse.linalg.splu`` (complex128; minimum-degree ordering
on A^T + A, which the symmetric system suits: on C1 it fills 22 M entries
against 38 M with the default ordering).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import oracle


def element_matrices(model) -> np.ndarray:
    """(n_tets, 6, 6) complex element matrices, rows and columns in the
    order of ``model.tet_edges[t][oracle.FILE_SLOT]``."""
    lib = oracle.load()
    lib.orc_element_matrix.restype = ctypes.c_int
    eps, sig = oracle.material_per_element(model)
    nt = model.n_tets
    out = np.zeros((nt, 6, 6), np.complex128)
    ae = np.zeros(72, np.float64)
    crd = model.vertex_crd
    for t in range(nt):
        v = model.tets[t]
        xyz = np.ascontiguousarray(np.concatenate([crd[v, 0], crd[v, 1], crd[v, 2]]), np.float64)
        bad = lib.orc_element_matrix(oracle._p(xyz, ctypes.c_double), ctypes.c_double(eps[t]),
                                     ctypes.c_double(sig[t]), ctypes.c_double(model.omega),
                                     oracle._p(ae, ctypes.c_double))
        if bad:
            raise ValueError(f"element {t}: non-positive volume")
        out[t] = (ae[0::2] + 1j * ae[1::2]).reshape(6, 6)
    return out


def assemble(model, source=0):
    """Global matrix (CSR, free edges only), right-hand side and the free
    edge ids.  ``source`` is an index into ``model.sources``, an
    (edges, values) pair or None."""
    import scipy.sparse as sp

    ne = model.n_edges
    gid = model.tet_edges[:, oracle.FILE_SLOT].astype(np.int64)
    am = element_matrices(model)
    rows = np.repeat(gid, 6, axis=1).ravel()
    cols = np.tile(gid, (1, 6)).ravel()
    A = sp.coo_matrix((am.ravel(), (rows, cols)), shape=(ne, ne)).tocsr()
    b = np.zeros(ne, np.complex128)
    if getattr(model, "element_source", None) is not None:
        be = oracle.element_rhs(model)
        # element vectors are in the same slot order as the element matrices
        np.add.at(b, gid, be)
    if source is not None:
        e, v = model.sources[source] if isinstance(source, int) else source
        np.add.at(b, np.asarray(e, np.int64), np.asarray(v, np.complex128))
    free = np.nonzero(~model.pec_edge.astype(bool))[0]
    return A[free][:, free].tocsc(), b[free], free


def solve(model, source=0) -> np.ndarray:
    """The exact discrete solution on every global edge (0 on the PEC wall)."""
    from scipy.sparse.linalg import splu

    A, b, free = assemble(model, source)
    x = np.zeros(model.n_edges, np.complex128)
    x[free] = splu(A, permc_spec="MMD_AT_PLUS_A").solve(b)
    return x
