// Internal host-side data structures of the HDDM hot path.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/fwgpu.h"

namespace fw {

// The plan's concatenated host arrays (gigabytes on the largest models) are
// written once, slice by slice, on all host threads.  This allocator leaves
// new elements uninitialised, so that resize() does not first zero-fill them
// on one thread; every element is then written by exactly one worker.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <typename U>
  NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
  template <typename U>
  void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new (static_cast<void *>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U *p, Args &&...args) {
    ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
  }
};
template <typename T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

// Element edge table of the reference (lib/fem/tetrahedral.h:19-24):
// slot i joins vertices kTetN[i][0] and kTetN[i][1]; kTetN[i][2..3] is the
// opposite edge.
constexpr int kTetN[6][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}};
// File order of the 6 mid-nodes is 01,02,03,12,23,13; the reference swaps
// node slots 8 and 9 (lib/fem/make_MESH.c:573-584), so element slot i reads
// file mid-node kFileSlot[i].
constexpr int kFileSlot[6] = {0, 1, 2, 3, 5, 4};

// Per-subdomain integer data, the state make_PartMesh_FW leaves in DomMesh.
struct SubHost {
  std::vector<int32_t> els;       // global element ids, ascending
  int32_t nap = 0;                // local vertices
  int32_t nmp = 0;                // local edge DOFs
  std::vector<int32_t> nop;       // 10*nel: 4 local vertex ids, 6 local edge ids (tet_n order)
  std::vector<int32_t> edge_gid;  // nmp: global edge id of each local edge DOF
  std::vector<int32_t> ibc;       // Dirichlet list: sorted PEC edge ids then interface nfids
  int32_t npec = 0;
  std::vector<int32_t> inbc_nfid; // sorted
  std::vector<int32_t> inbc_ln;   // global interface id of each inbc entry
  std::vector<uint8_t> isbc;      // nmp
  std::vector<int32_t> cidx;      // nmp: interior (compressed) index, -1 for Dirichlet DOFs
  std::vector<int32_t> slot;      // nmp: interface slot (position in inbc), -1 otherwise
  int32_t nI = 0;                 // interior DOFs
  int32_t nG = 0;                 // interface DOFs
  // structural lower-triangle rows (sorted columns), local DOF ids
  std::vector<int32_t> row_ptr;   // nmp+1
  std::vector<int32_t> col;       // nnz
};

struct Model {
  int32_t nv = 0, nt = 0, ne = 0, nsub = 0;
  std::vector<double> crd;
  std::vector<int32_t> tv, te, flag, sub_of_tet;
  std::vector<uint8_t> pec;
  // each subdomain's local vertex and edge order (empty: ascending global id)
  std::vector<int32_t> sub_vptr, sub_vord, sub_eptr, sub_eord;
  // material resolved per element (the reference's first-match linear search
  // over the flag tables, lib/fem/make_elem_em.c:98-109)
  std::vector<double> el_eps, el_sigma;
  // 1 when the element's flag is in the Permittivity list: the post step
  // uses nu = 7.957747e+05 there and 0 elsewhere (main/fullwave/fullwave.c:672-677)
  std::vector<uint8_t> el_has_nu;
  double omega = 0.0;
};

// Host plan: integer maps and index lists for the device gathers.
struct Plan {
  std::vector<SubHost> subs;
  int32_t total_free = 0;            // interface DOFs
  std::vector<int32_t> iface_gid;    // global edge id of each interface DOF
  std::vector<int32_t> iface_owner_sub;
  // concatenated over subdomains (sub-major, elements in sub order)
  std::vector<int32_t> el_order;     // global element id of each element slot
  std::vector<int64_t> sub_el_off;   // nsub+1
  std::vector<int64_t> sub_dof_off;  // nsub+1, offsets of local DOF arrays
  std::vector<int64_t> sub_nnz_off;  // nsub+1, offsets of lower CSR entries
  std::vector<int64_t> sub_int_off;  // nsub+1, offsets of interior arrays
  std::vector<int64_t> sub_if_off;   // nsub+1, offsets of interface slot arrays
  // lower CSR (local rows, concatenated), row_ptr relative to sub_nnz_off
  HostVec<int32_t> csr_row_ptr;  // sum(nmp+1)
  HostVec<int32_t> csr_col;      // local col
  HostVec<int64_t> contrib_ptr;  // nnz_total+1
  HostVec<int64_t> contrib;      // element-slot*36 + (i*6+j)
  HostVec<uint8_t> isbc;         // sum(nmp)
  // per-iteration operators (positions into the global lower-CSR value array)
  // coupling: interior row c -> interface slots   (b_I = -A_IG v)
  HostVec<int32_t> cpl_ptr;      // sum(nI+1), relative
  HostVec<int32_t> cpl_col;      // interface slot
  HostVec<int64_t> cpl_src;      // lower-CSR position
  // interface rows: slot k -> (interior c) or (interface slot)
  HostVec<int32_t> ifr_ptr;      // sum(nG+1), relative
  HostVec<int32_t> ifr_col;      // >=0 interior index, <0: -(slot+1)
  HostVec<int64_t> ifr_src;
  // interior operator (both triangles), for FP64 refinement residuals
  HostVec<int32_t> aii_ptr;      // sum(nI+1), relative
  HostVec<int32_t> aii_col;
  HostVec<int64_t> aii_src;
  // interface slot data
  HostVec<int32_t> if_ln;        // sum(nG): global interface id
  HostVec<int64_t> if_diag_src;  // sum(nG): lower-CSR position of the diagonal, -1 if absent
  HostVec<int32_t> if_local;     // sum(nG): local DOF id
  // interior data
  HostVec<int32_t> int_local;    // sum(nI): local DOF id
  HostVec<int64_t> int_diag_src; // sum(nI): lower-CSR position of the diagonal
  // gather of q into Q: for each interface DOF g, the (sub-major) slots in sub order
  std::vector<int32_t> gq_ptr;       // total_free+1
  HostVec<int64_t> gq_slot;      // global slot index (sub_if_off + k)
  int64_t nnz_total = 0;
  int64_t nlen_reference = 0;
  int32_t el_dofs = 6;               // DOFs per element: 6 edges, or 4 vertices (correction-Jo problem)
  int32_t max_local = 0, max_interior = 0, max_iface = 0;
};

// Builds the plan; returns an empty string on success or an error message.
std::string build_plan(const Model &m, Plan &p);

// Row pointers and column maps of the grid-wide products over all
// subdomains' rows at once (the concatenated interior rows and interface
// slots): cpl (interior row -> interface DOF), ifr (interface slot -> global
// interior row, or -(interface DOF)-1), aii (interior row -> global interior
// row); *_off are the per-subdomain offsets of the lists (nsub+1).
struct GlobalRows {
  std::vector<int64_t> cpl_off, ifr_off, aii_off;
  HostVec<int64_t> cpl_rowptr, ifr_rowptr, aii_rowptr;
  HostVec<int32_t> cpl_gcol, ifr_gcol, aii_gcol;
};
void global_rows(const Plan &p, GlobalRows &g);

// The interior envelope of every subdomain from the reference's skyline
// profile idx1 (one entry per local DOF, concatenated): the first interior
// column env_lo and the position env_ptr of every interior row (each
// subdomain from an even position), the envelope position of every lower
// entry (dst, -1 outside the interior envelope), the total length nlen and
// the reference's skyline length nlen_ref (advlas_skyline.c:20-24).
struct EnvelopeLayout {
  std::vector<int32_t> env_lo;
  std::vector<int64_t> env_ptr;
  HostVec<int64_t> dst;
  int64_t nlen = 0, nlen_ref = 0;
};
void envelope_layout(const Plan &p, const int32_t *idx1, EnvelopeLayout &e);
// The plan of one antenna's correction-Jo problem (vertex DOFs of the
// elements carrying antenna_flag); sub_map receives the original subdomain id
// of each of its subdomains.  pec_vertex: one flag per vertex, or empty.
std::string build_plan_cojo(const Model &m, int32_t antenna_flag, const std::vector<uint8_t> &pec_vertex, Plan &p,
                            std::vector<int32_t> &sub_map);

}  // namespace fw
