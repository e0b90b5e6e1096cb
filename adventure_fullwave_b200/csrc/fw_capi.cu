// C ABI of the HDDM hot path (include/fwgpu.h): context, uploads and the
// host orchestration of the device kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "fw_internal.h"
#include "fw_kernels.cuh"

namespace {
// An NVTX range over one library call, so that a profiler's timeline (nsys,
// or ncu --nvtx) shows the reference's slots; without a tool attached a
// range costs a call into a no-op.
struct Trace {
  explicit Trace(const char *name) { nvtxRangePushA(name); }
  ~Trace() { nvtxRangePop(); }
  Trace(const Trace &) = delete;
  Trace &operator=(const Trace &) = delete;
};
}  // namespace

namespace {

thread_local std::string g_last_error = "";

int set_error(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

#define FW_CUDA(call)                                                                                \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) {                                                                         \
      return set_error(e_ == cudaErrorMemoryAllocation ? FWGPU_ERR_NOMEM : FWGPU_ERR_CUDA,           \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    }                                                                                                \
  } while (0)

}  // namespace

namespace fw {
// error text for fwgpu_last_error from entry points outside this file
void record_error(const std::string &msg) { g_last_error = msg; }
}  // namespace fw

struct fwgpu_context {
  fw::Model m;
  fw::Plan p;
  fwgpu_options opts{};
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  int stage = 0;  // 0 created, 1 assembled, 2 first solve, 3 interface iteration, 4 last step

  // static device data
  int32_t *d_tv = nullptr, *d_el_order = nullptr, *d_mesh_status = nullptr;
  double *d_crd = nullptr, *d_el_eps = nullptr, *d_el_sigma = nullptr;
  int64_t *d_cptr = nullptr, *d_contrib = nullptr;
  double2 *d_aval = nullptr;
  int32_t *d_row_ptr = nullptr, *d_col = nullptr, *d_idx1 = nullptr;
  uint8_t *d_isbc = nullptr;
  int64_t *d_dof_off = nullptr, *d_nnz_off = nullptr;
  // envelope
  std::vector<int32_t> h_idx1;
  std::vector<int32_t> h_env_lo;
  std::vector<int64_t> h_env_ptr;
  int64_t nlen_int = 0;
  int64_t nlen_ref = 0;
  double2 *d_L64 = nullptr;
  float2 *d_L32 = nullptr;
  int32_t *d_env_lo = nullptr;
  int64_t *d_env_ptr = nullptr;
  // operators and right-hand sides
  std::vector<double2> h_b_local;  // TMP_B per local DOF (concatenated)
  double2 *d_cpl_val = nullptr, *d_ifr_val = nullptr, *d_aii_val = nullptr, *d_pcloc = nullptr;
  double2 *d_fI = nullptr, *d_fG = nullptr;
  int64_t *d_edge_src = nullptr;
  double2 *d_xedge = nullptr;
  double2 *d_xfwd = nullptr;        // forward solution kept during an adjoint solve
  int32_t *d_te = nullptr;          // tet edges (adjoint gradient)
  fw::DevProblem dp{};
  fw::CocgScalars *d_sc = nullptr;
  fw::CocgScalars *h_sc = nullptr;  // pinned
  double *d_hist = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool factor_bad = false;
  bool factor_fresh = false;       // factor matches the assembled values
  bool solve_tuned = false;        // the subdomain-solve kernel has been chosen
  // assembly work buffers kept for the context's lifetime (repeated solves)
  double *d_elmat = nullptr;       // element matrices, 72 doubles per element
  int64_t *d_cpl_src = nullptr, *d_ifr_src = nullptr, *d_aii_src = nullptr, *d_diag_src = nullptr;
  std::vector<int32_t> h_src_owner, h_src_local;  // first subdomain holding each edge, and its local DOF
  bool warp_ok = false;            // the staged warp-per-subdomain kernel fits in shared memory
  bool sharded = false;            // solves a range of the subdomains (fwgpu_shard_* calls)
  // sharded solve: the caller's packed exchange and scalar buffers, and the
  // shard layout (held interface DOFs, owned, packed positions)
  double2 *d_pack = nullptr;
  double *d_scal = nullptr;
  int32_t shard_lo = 0, shard_hi = 0;
  int32_t n_shared = -1;           // -1: no layout yet
  // batched sources (fwgpu_hddm_solve_multi)
  fw::MultiProblem mp{};
  fw::MultiScalars *h_ms = nullptr;
  cudaGraphExec_t multi_graph = nullptr;
  int multi_n = 0;                 // sources of the last batched solve (0: none)
  int32_t *d_blk_off = nullptr;    // staged solve block table (current staging capacity)
  int2 *d_blk_tab = nullptr;
  // block-inverse layout of the factor (FWGPU_SOLVE_BLOCKINV)
  bool inv_ok = false;             // its block table is built and its kernel fits in shared memory
  int64_t inv_len = 0;             // elements of Linv
  int64_t *d_inv_ptr = nullptr;
  int32_t *d_inv_blk_off = nullptr;
  int2 *d_inv_blk_tab = nullptr;
  double2 *d_Linv64 = nullptr;
  float2 *d_Linv32 = nullptr;
  std::vector<int> stage_caps;     // staging capacities that fit in shared memory
  std::vector<int32_t> h_order;    // subdomains by interior size, largest first (the device sub_order)
  std::vector<int32_t> h_nblk;     // staged blocks of each subdomain at the current capacity
  int64_t launches = 0;            // kernels launched since the last reset
  int64_t *d_env_dst = nullptr;    // lower entry -> envelope position (-1: outside)
  // element right-hand side (fwgpu_set_element_source)
  bool el_src = false;             // an element source is set
  bool el_src_off = false;         // the adjoint solve assembles its own source only
  int32_t n_gaps = 0;
  double *d_gap = nullptr;         // 7 per gap: box x0 x1 y0 y1 z0 z1, dV
  int32_t *d_el_ant = nullptr;     // antenna of each element, -1 for none
  double *d_Jo = nullptr, *d_Jor = nullptr;
  double2 *d_elrhs = nullptr;      // 6 per element slot
  int64_t *d_rhs_ptr = nullptr;    // per local DOF (concatenated): its element contributions
  int32_t *d_rhs_src = nullptr;    // element slot * 6 + edge
  int64_t *d_int_pos = nullptr, *d_if_pos = nullptr;  // local DOF of each interior / interface entry
  double2 *d_b_edge = nullptr;     // edge-source TMP_B (host-built)
  double2 *d_b_local = nullptr;    // TMP_B of every subdomain
  // post step (fwgpu_post_em_E)
  bool xedge_ok = false;           // d_xedge holds a whole edge solution
  uint8_t *d_el_has_nu = nullptr;
  double2 *d_post = nullptr;       // 3 x 3 complex per element (B, E, Je), when the caller's buffers are on the host
  double2 *d_post_x = nullptr;     // the caller's edge solution, when it is on the host
  // per-entity solution: edges, or vertices of the correction-Jo problem
  int64_t n_out = 0;
  // correction-Jo problem of one antenna (fwgpu_cojo_*): its element flag
  // (-1: the full-wave problem), the original subdomain id of each of its
  // subdomains and the current of the pass (3 per vertex)
  int32_t cojo_flag = -1;
  std::vector<int32_t> cojo_sub;
  double *d_cojo_J = nullptr;

  template <typename T>
  int alloc(T **ptr, size_t count) {
    *ptr = nullptr;
    if (count == 0) count = 1;
    void *raw = nullptr;
    cudaError_t e = cudaMalloc(&raw, count * sizeof(T));
    if (e != cudaSuccess)
      return set_error(FWGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(raw);
    *ptr = (T *)raw;
    return FWGPU_OK;
  }
  template <typename T, typename A>
  int upload(T **ptr, const std::vector<T, A> &v) {
    int rc = alloc(ptr, v.size());
    if (rc) return rc;
    if (!v.empty()) FW_CUDA(cudaMemcpyAsync(*ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return FWGPU_OK;
  }
  void release(void *ptr) {
    if (!ptr) return;
    auto it = std::find(allocs.begin(), allocs.end(), ptr);
    if (it != allocs.end()) {
      cudaFree(*it);
      allocs.erase(it);
    }
  }
};

namespace {

#define FW_TRY(expr)           \
  do {                         \
    int rc_ = (expr);          \
    if (rc_ != FWGPU_OK) return rc_; \
  } while (0)


int resolve_material(fw::Model &m, const fwgpu_mesh *mesh, const fwgpu_material *mt) {
  m.el_eps.assign(m.nt, 0.0);
  m.el_sigma.assign(m.nt, 0.0);
  m.el_has_nu.assign(m.nt, 0);
  // the reference searches the tables linearly and takes the first match
  // (lib/fem/make_elem_em.c:98-109); absent flags leave eps = sigma = 0.
  // The first entry of each flag, looked up by hash: tables with one flag
  // per element (per-element materials) stay linear in the element count.
  std::unordered_map<int32_t, int32_t> eps_at, sigma_at;
  eps_at.reserve(2 * (size_t)std::max(0, mt->n_eps));
  sigma_at.reserve(2 * (size_t)std::max(0, mt->n_sigma));
  for (int i = 0; i < mt->n_eps; i++) eps_at.emplace(mt->eps_flag[i], i);
  for (int i = 0; i < mt->n_sigma; i++) sigma_at.emplace(mt->sigma_flag[i], i);
  for (int t = 0; t < m.nt; t++) {
    const int f = mesh->tet_flag[t];
    auto e = eps_at.find(f);
    if (e != eps_at.end()) {
      m.el_eps[t] = mt->eps[e->second];
      m.el_has_nu[t] = 1;
    }
    auto g = sigma_at.find(f);
    if (g != sigma_at.end()) m.el_sigma[t] = mt->sigma[g->second];
  }
  return FWGPU_OK;
}

int build_rhs(fwgpu_context *c, const fwgpu_source *src) {
  if (c->cojo_flag >= 0 && src && src->n_entries > 0)
    return set_error(FWGPU_ERR_ARG, "a correction-Jo context takes its right-hand side from the antenna current");
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  std::vector<double2> fI(p.sub_int_off[nsub], make_double2(0.0, 0.0));
  std::vector<double2> fG(p.sub_if_off[nsub], make_double2(0.0, 0.0));
  c->h_b_local.assign(p.sub_dof_off[nsub], make_double2(0.0, 0.0));
  if (src && src->n_entries > 0) {
    if (!src->edge || !src->value) return set_error(FWGPU_ERR_ARG, "source without edges or values");
    // owner subdomain and local DOF of every edge: the first subdomain holding it
    std::vector<int32_t> &owner = c->h_src_owner, &local = c->h_src_local;
    if (owner.empty()) {
      owner.assign(c->m.ne, -1);
      local.assign(c->m.ne, -1);
      for (int s = 0; s < nsub; s++) {
        const fw::SubHost &h = p.subs[s];
        for (int r = 0; r < h.nmp; r++) {
          const int e = h.edge_gid[r];
          if (owner[e] < 0) {
            owner[e] = s;
            local[e] = r;
          }
        }
      }
    }
    for (int k = 0; k < src->n_entries; k++) {
      const int e = src->edge[k];
      if (e < 0 || e >= c->m.ne) return set_error(FWGPU_ERR_ARG, "source edge out of range");
      const int s = owner[e], r = local[e];
      if (s < 0) continue;
      const double2 val = make_double2(src->value[2 * k], src->value[2 * k + 1]);
      double2 &b = c->h_b_local[p.sub_dof_off[s] + r];
      b.x += val.x;
      b.y += val.y;
      const fw::SubHost &h = p.subs[s];
      if (h.cidx[r] >= 0) {
        fI[p.sub_int_off[s] + h.cidx[r]] = b;
      } else if (h.slot[r] >= 0) {
        fG[p.sub_if_off[s] + h.slot[r]] = b;
      }
    }
  }
  if (!c->d_fI) {
    FW_TRY(c->alloc(&c->d_fI, fI.size()));
    FW_TRY(c->alloc(&c->d_fG, fG.size()));
  }
  if (!fI.empty())
    FW_CUDA(cudaMemcpyAsync(c->d_fI, fI.data(), fI.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  if (!fG.empty())
    FW_CUDA(cudaMemcpyAsync(c->d_fG, fG.data(), fG.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  if (c->el_src && !c->el_src_off) {
    // TMP_B = element contributions in element order, then the edge source;
    // the interior and interface right-hand sides are taken from it
    const int64_t ndof = p.sub_dof_off[nsub];
    if (!c->d_b_local) {
      FW_TRY(c->alloc(&c->d_b_local, ndof));
      FW_TRY(c->alloc(&c->d_b_edge, ndof));
    }
    if (ndof > 0)
      FW_CUDA(cudaMemcpyAsync(c->d_b_edge, c->h_b_local.data(), ndof * sizeof(double2), cudaMemcpyHostToDevice,
                              c->stream));
    fw::launch_rhs_gather(ndof, c->d_rhs_ptr, c->d_rhs_src, c->d_elrhs, c->d_b_edge, c->d_b_local, c->stream);
    fw::launch_rhs_split((int64_t)fI.size(), c->d_int_pos, c->d_b_local, c->d_fI, c->stream);
    fw::launch_rhs_split((int64_t)fG.size(), c->d_if_pos, c->d_b_local, c->d_fG, c->stream);
    c->launches += 3;
    FW_CUDA(cudaGetLastError());
  }
  FW_CUDA(cudaStreamSynchronize(c->stream));
  c->dp.fI = c->d_fI;
  c->dp.fG = c->d_fG;
  return FWGPU_OK;
}

// Gather lists of the element right-hand side: local DOF -> (element slot *
// 6 + element DOF), elements in subdomain order, and the local DOF of every
// interior and interface entry; built once per context.
int build_rhs_lists(fwgpu_context *c) {
  if (c->d_rhs_ptr) return FWGPU_OK;
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  const int nd = p.el_dofs;
  const int64_t ndof = p.sub_dof_off[nsub];
  std::vector<int64_t> ptr(ndof + 1, 0);
  for (int s = 0; s < nsub; s++) {
    const fw::SubHost &h = p.subs[s];
    for (size_t e = 0; e < h.els.size(); e++)
      for (int i = 0; i < nd; i++) ptr[p.sub_dof_off[s] + h.nop[10 * e + 4 + i] + 1]++;
  }
  for (int64_t r = 0; r < ndof; r++) ptr[r + 1] += ptr[r];
  std::vector<int32_t> src(ptr[ndof]);
  std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
  for (int s = 0; s < nsub; s++) {
    const fw::SubHost &h = p.subs[s];
    for (size_t e = 0; e < h.els.size(); e++)
      for (int i = 0; i < nd; i++)
        src[fill[p.sub_dof_off[s] + h.nop[10 * e + 4 + i]]++] = (int32_t)(6 * (p.sub_el_off[s] + (int64_t)e) + i);
  }
  std::vector<int64_t> int_pos(p.sub_int_off[nsub]), if_pos(p.sub_if_off[nsub]);
  for (int s = 0; s < nsub; s++) {
    for (int64_t k = p.sub_int_off[s]; k < p.sub_int_off[s + 1]; k++) int_pos[k] = p.sub_dof_off[s] + p.int_local[k];
    for (int64_t k = p.sub_if_off[s]; k < p.sub_if_off[s + 1]; k++) if_pos[k] = p.sub_dof_off[s] + p.if_local[k];
  }
  FW_TRY(c->upload(&c->d_rhs_ptr, ptr));
  FW_TRY(c->upload(&c->d_rhs_src, src));
  FW_TRY(c->upload(&c->d_int_pos, int_pos));
  FW_TRY(c->upload(&c->d_if_pos, if_pos));
  FW_TRY(c->alloc(&c->d_elrhs, 6 * std::max<size_t>(1, p.el_order.size())));
  return FWGPU_OK;
}

// Element sources: the per-element right-hand side is computed once (it
// depends on the geometry, the conductivity and the source only) and the
// gather lists from local DOFs to element contributions are built.
int set_element_source(fwgpu_context *c, const fwgpu_element_source *es) {
  const int64_t nv = c->m.nv, nt = c->m.nt;
  if (es->n_gaps < 0 || es->n_antennas < 0) return set_error(FWGPU_ERR_ARG, "negative count");
  if (es->n_gaps > 0 && (!es->gap_box || !es->gap_volt)) return set_error(FWGPU_ERR_ARG, "gaps without boxes");
  if (es->n_gaps == 0 && es->n_antennas > 0 && (!es->antenna_flag || !es->antenna_Jo || !es->antenna_Jor))
    return set_error(FWGPU_ERR_ARG, "antennas without flags or currents");
  for (void *q : {(void *)c->d_gap, (void *)c->d_el_ant, (void *)c->d_Jo, (void *)c->d_Jor}) c->release(q);
  c->d_gap = nullptr;
  c->d_el_ant = nullptr;
  c->d_Jo = c->d_Jor = nullptr;
  c->n_gaps = es->n_gaps;
  std::vector<double> gap(7 * (size_t)std::max(1, es->n_gaps), 0.0);
  for (int g = 0; g < es->n_gaps; g++) {
    for (int q = 0; q < 6; q++) gap[7 * g + q] = es->gap_box[6 * g + q];
    gap[7 * g + 6] = es->gap_volt[g];
  }
  FW_TRY(c->upload(&c->d_gap, gap));
  // first antenna whose flag matches (make_elem_em.c:110-115)
  const int nant = es->n_gaps > 0 ? 0 : es->n_antennas;
  std::vector<int32_t> el_ant(nt, -1);
  for (int64_t t = 0; t < nt; t++)
    for (int k = 0; k < nant; k++)
      if (c->m.flag[t] == es->antenna_flag[k]) {
        el_ant[t] = k;
        break;
      }
  FW_TRY(c->upload(&c->d_el_ant, el_ant));
  const size_t nj = 3 * (size_t)nv * std::max(1, nant);
  FW_TRY(c->alloc(&c->d_Jo, nj));
  FW_TRY(c->alloc(&c->d_Jor, nj));
  if (nant > 0) {
    FW_CUDA(cudaMemcpyAsync(c->d_Jo, es->antenna_Jo, nj * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    FW_CUDA(cudaMemcpyAsync(c->d_Jor, es->antenna_Jor, nj * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  FW_TRY(build_rhs_lists(c));
  fw::launch_element_rhs(nt, c->d_el_order, c->d_tv, c->d_crd, c->d_el_sigma, c->m.omega, es->n_gaps, c->d_gap,
                         c->d_el_ant, c->d_Jo, c->d_Jor, nv, c->d_elrhs, c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  c->el_src = true;
  return FWGPU_OK;
}

// The copy-timeout word is raised by the subdomain solves and cleared only
// here, at the start of a solve, so that no later launch hides it.
int clear_copy_timeout(fwgpu_context *c) {
  FW_CUDA(cudaMemsetAsync(&c->d_sc->copy_timeout, 0, sizeof(int32_t), c->stream));
  return FWGPU_OK;
}

int read_status(fwgpu_context *c, int32_t *status) {
  FW_CUDA(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(fw::CocgScalars), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  if (status) *status = c->h_sc->status;
  if (c->h_sc->copy_timeout != 0)
    return set_error(FWGPU_ERR_TIMEOUT, "subdomain solve gave up waiting for a staged copy");
  return FWGPU_OK;
}

}  // namespace

struct fwgpu_partition {
  fw::Model m;
  fw::Plan p;
  std::vector<int32_t> cojo_sub;  // correction-Jo partition: original id of each subdomain
};

static int copy_maps(const fw::Plan &p, int32_t s, int32_t *nel, int32_t *nmp, int32_t *nbc, int32_t *ninbc,
                     int32_t *nop, int32_t *ibc, int32_t *inbc_nfid, int32_t *inbc_ln_part, int32_t *edge_gid) {
  if (s < 0 || s >= (int32_t)p.subs.size()) return set_error(FWGPU_ERR_ARG, "bad subdomain");
  const fw::SubHost &h = p.subs[s];
  if (nel) *nel = (int32_t)h.els.size();
  if (nmp) *nmp = h.nmp;
  if (nbc) *nbc = (int32_t)h.ibc.size();
  if (ninbc) *ninbc = h.nG;
  if (nop) std::copy(h.nop.begin(), h.nop.end(), nop);
  if (ibc) std::copy(h.ibc.begin(), h.ibc.end(), ibc);
  if (inbc_nfid) std::copy(h.inbc_nfid.begin(), h.inbc_nfid.end(), inbc_nfid);
  if (inbc_ln_part) std::copy(h.inbc_ln.begin(), h.inbc_ln.end(), inbc_ln_part);
  if (edge_gid) std::copy(h.edge_gid.begin(), h.edge_gid.end(), edge_gid);
  return FWGPU_OK;
}

static int model_from_mesh(const fwgpu_mesh *mesh, fw::Model &m) {
  if (!mesh || mesh->n_vertices <= 0 || mesh->n_tets <= 0 || mesh->n_edges <= 0 || mesh->n_subdomains <= 0 ||
      !mesh->vertex_crd || !mesh->tet_vertices || !mesh->tet_edges || !mesh->tet_flag || !mesh->pec_edge ||
      !mesh->sub_of_tet)
    return set_error(FWGPU_ERR_ARG, "incomplete mesh");
  for (int64_t k = 0; k < 4 * (int64_t)mesh->n_tets; k++)
    if (mesh->tet_vertices[k] < 0 || mesh->tet_vertices[k] >= mesh->n_vertices)
      return set_error(FWGPU_ERR_ARG, "tet_vertices out of range");
  m.nv = mesh->n_vertices;
  m.nt = mesh->n_tets;
  m.ne = mesh->n_edges;
  m.nsub = mesh->n_subdomains;
  m.crd.assign(mesh->vertex_crd, mesh->vertex_crd + 3 * (int64_t)m.nv);
  m.tv.assign(mesh->tet_vertices, mesh->tet_vertices + 4 * (int64_t)m.nt);
  m.te.assign(mesh->tet_edges, mesh->tet_edges + 6 * (int64_t)m.nt);
  m.flag.assign(mesh->tet_flag, mesh->tet_flag + m.nt);
  m.sub_of_tet.assign(mesh->sub_of_tet, mesh->sub_of_tet + m.nt);
  m.pec.assign(mesh->pec_edge, mesh->pec_edge + m.ne);
  const bool any_order = mesh->sub_vertex_ptr || mesh->sub_vertex_order || mesh->sub_edge_ptr || mesh->sub_edge_order;
  if (any_order) {
    if (!mesh->sub_vertex_ptr || !mesh->sub_vertex_order || !mesh->sub_edge_ptr || !mesh->sub_edge_order)
      return set_error(FWGPU_ERR_ARG, "subdomain orders: give all four arrays or none");
    const int ns = m.nsub;
    for (int s = 0; s < ns; s++)
      if (mesh->sub_vertex_ptr[s + 1] < mesh->sub_vertex_ptr[s] || mesh->sub_edge_ptr[s + 1] < mesh->sub_edge_ptr[s])
        return set_error(FWGPU_ERR_ARG, "subdomain order offsets decrease");
    if (mesh->sub_vertex_ptr[0] != 0 || mesh->sub_edge_ptr[0] != 0)
      return set_error(FWGPU_ERR_ARG, "subdomain order offsets must start at 0");
    m.sub_vptr.assign(mesh->sub_vertex_ptr, mesh->sub_vertex_ptr + ns + 1);
    m.sub_eptr.assign(mesh->sub_edge_ptr, mesh->sub_edge_ptr + ns + 1);
    m.sub_vord.assign(mesh->sub_vertex_order, mesh->sub_vertex_order + m.sub_vptr[ns]);
    m.sub_eord.assign(mesh->sub_edge_order, mesh->sub_edge_order + m.sub_eptr[ns]);
  }
  return FWGPU_OK;
}

// The device side of a context whose model and plan are built: stream,
// uploads, operator structures, vectors and the per-entity solution map over
// c->n_out entities (edges, or vertices of the correction-Jo problem).  On a
// failure after the stream exists the context is handed out for release.
static int setup_device(fwgpu_context *c, const fwgpu_options *opts, fwgpu_context **out) {
  fw::Model &m = c->m;
  cudaError_t e = cudaSetDevice(opts->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return set_error(FWGPU_ERR_CUDA, std::string("device setup: ") + cudaGetErrorString(e));
  }
  for (auto &ev : c->ev) cudaEventCreate(&ev);
  *out = c;

  const fw::Plan &p = c->p;
  const int nsub = m.nsub;
  FW_TRY(c->upload(&c->d_crd, m.crd));
  FW_TRY(c->upload(&c->d_tv, m.tv));
  FW_TRY(c->upload(&c->d_el_order, p.el_order));
  FW_TRY(c->upload(&c->d_el_eps, m.el_eps));
  FW_TRY(c->upload(&c->d_el_sigma, m.el_sigma));
  FW_TRY(c->upload(&c->d_cptr, p.contrib_ptr));
  FW_TRY(c->upload(&c->d_contrib, p.contrib));
  FW_TRY(c->upload(&c->d_row_ptr, p.csr_row_ptr));
  FW_TRY(c->upload(&c->d_col, p.csr_col));
  FW_TRY(c->upload(&c->d_isbc, p.isbc));
  FW_TRY(c->upload(&c->d_dof_off, p.sub_dof_off));
  FW_TRY(c->upload(&c->d_nnz_off, p.sub_nnz_off));
  FW_TRY(c->alloc(&c->d_mesh_status, 4));
  FW_CUDA(cudaMemsetAsync(c->d_mesh_status, 0, 4 * sizeof(int32_t), c->stream));

  // the subdomains this context solves: all, or a shard's range
  int s_begin = 0, s_end = nsub;
  if (opts->shard_begin != 0 || opts->shard_end != 0) {
    if (opts->shard_begin < 0 || opts->shard_end > nsub || opts->shard_begin >= opts->shard_end)
      return set_error(FWGPU_ERR_ARG, "shard range outside the subdomains");
    s_begin = opts->shard_begin;
    s_end = opts->shard_end;
    // an explicit range, all subdomains included (one rank), runs the shard protocol
    c->sharded = true;
  }
  // subdomains largest first (by interior DOFs, then local DOFs)
  std::vector<int32_t> order(s_end - s_begin);
  for (int s = s_begin; s < s_end; s++) order[s - s_begin] = s;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const fw::SubHost &x = p.subs[a], &y = p.subs[b];
    return x.nI != y.nI ? x.nI > y.nI : x.nmp > y.nmp;
  });
  c->h_order = order;
  fw::DevProblem &dp = c->dp;
  dp.nsub = s_end - s_begin;
  dp.nfree = p.total_free;
  int32_t *d_order = nullptr;
  int64_t *d_int_off = nullptr, *d_if_off = nullptr;
  FW_TRY(c->upload(&d_order, order));
  FW_TRY(c->upload(&d_int_off, p.sub_int_off));
  FW_TRY(c->upload(&d_if_off, p.sub_if_off));
  dp.sub_order = d_order;
  dp.int_off = d_int_off;
  dp.if_off = d_if_off;
  // operator structures, and the global row pointers and column maps of the
  // grid-wide products of the staged solve
  fw::GlobalRows g;
  fw::global_rows(p, g);
  int32_t *ip = nullptr;
  int64_t *lp = nullptr;
  FW_TRY(c->upload(&ip, p.cpl_ptr));
  dp.cpl_ptr = ip;
  FW_TRY(c->upload(&lp, g.cpl_off));
  dp.cpl_off = lp;
  FW_TRY(c->upload(&ip, p.cpl_col));
  dp.cpl_col = ip;
  FW_TRY(c->upload(&ip, p.ifr_ptr));
  dp.ifr_ptr = ip;
  FW_TRY(c->upload(&lp, g.ifr_off));
  dp.ifr_off = lp;
  FW_TRY(c->upload(&ip, p.ifr_col));
  dp.ifr_col = ip;
  FW_TRY(c->upload(&ip, p.aii_ptr));
  dp.aii_ptr = ip;
  FW_TRY(c->upload(&lp, g.aii_off));
  dp.aii_off = lp;
  FW_TRY(c->upload(&ip, p.aii_col));
  dp.aii_col = ip;
  FW_TRY(c->upload(&ip, p.if_ln));
  dp.if_ln = ip;
  FW_TRY(c->upload(&ip, p.gq_ptr));
  dp.gq_ptr = ip;
  FW_TRY(c->upload(&lp, p.gq_slot));
  dp.gq_slot = lp;
  {
    FW_TRY(c->upload(&lp, g.cpl_rowptr));
    dp.cpl_rowptr = lp;
    FW_TRY(c->upload(&ip, g.cpl_gcol));
    dp.cpl_gcol = ip;
    FW_TRY(c->upload(&lp, g.ifr_rowptr));
    dp.ifr_rowptr = lp;
    FW_TRY(c->upload(&ip, g.ifr_gcol));
    dp.ifr_gcol = ip;
    FW_TRY(c->upload(&lp, g.aii_rowptr));
    dp.aii_rowptr = lp;
    FW_TRY(c->upload(&ip, g.aii_gcol));
    dp.aii_gcol = ip;
    dp.row0 = p.sub_int_off[s_begin];
    dp.n_interior = p.sub_int_off[s_end] - p.sub_int_off[s_begin];
    dp.slot0 = p.sub_if_off[s_begin];
    dp.n_slots = p.sub_if_off[s_end] - p.sub_if_off[s_begin];
    c->shard_lo = s_begin;
    c->shard_hi = s_end;
  }
  FW_TRY(c->alloc(&c->d_cpl_val, p.cpl_src.size()));
  FW_TRY(c->alloc(&c->d_ifr_val, p.ifr_src.size()));
  FW_TRY(c->alloc(&c->d_pcloc, p.if_diag_src.size()));
  dp.cpl_val = c->d_cpl_val;
  dp.ifr_val = c->d_ifr_val;
  if (opts->precision == FWGPU_PREC_FP32_IR) {
    FW_TRY(c->alloc(&c->d_aii_val, p.aii_src.size()));
    dp.aii_val = c->d_aii_val;
  }
  const int64_t nI_tot = p.sub_int_off[nsub], nG_tot = p.sub_if_off[nsub];
  FW_TRY(c->alloc(&dp.Y, nI_tot));
  FW_TRY(c->alloc(&dp.V, nG_tot));
  FW_TRY(c->alloc(&dp.qloc, nG_tot));
  if (opts->precision == FWGPU_PREC_FP32_IR) {
    FW_TRY(c->alloc(&dp.B, nI_tot));
    FW_TRY(c->alloc(&dp.Y32, nI_tot));
    FW_TRY(c->alloc(&dp.Rres, nI_tot));
  }
  const int64_t nf = std::max<int64_t>(1, p.total_free);
  FW_TRY(c->alloc(&dp.P, nf));
  FW_TRY(c->alloc(&dp.Q, nf));
  FW_TRY(c->alloc(&dp.R, nf));
  FW_TRY(c->alloc(&dp.Z, nf));
  FW_TRY(c->alloc(&dp.U, nf));
  FW_TRY(c->alloc(&dp.PC, nf));
  // COCG grid: at most 4 CTAs of 256 threads per SM (timed against 2, 8 and 16)
  int n_sm = 148;
  if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, opts->device) != cudaSuccess || n_sm <= 0)
    n_sm = 148;
  int nb = (int)std::min<int64_t>((p.total_free + 255) / 256, 4 * (int64_t)n_sm);
  if (nb < 1) nb = 1;
  dp.n_part_blocks = nb;
  FW_TRY(c->alloc(&dp.part, 8 * (size_t)nb));
  FW_TRY(c->alloc(&c->d_sc, 1));
  dp.sc = c->d_sc;
  FW_CUDA(cudaMallocHost(&c->h_sc, sizeof(fw::CocgScalars)));
  FW_TRY(c->alloc(&c->d_hist, (size_t)std::max(1, opts->hddm_max_loop) + 2));
  dp.hist = c->d_hist;
  dp.hist_cap = std::max(1, opts->hddm_max_loop) + 2;
  dp.ir_steps = c->opts.ir_max_steps;
  dp.ir_tol = c->opts.ir_tol;
  dp.ir_relax = c->opts.ir_relax;
  dp.stall_test = c->opts.stall_copy_test ? 1 : 0;
  {
    const bool fp32 = opts->precision == FWGPU_PREC_FP32_IR;
    const size_t smem = fw::subsolve_smem_bytes(p.max_interior, p.max_iface, fp32);
    dp.cta_smem = fw::configure_subsolve(smem, fp32) == 0 ? (int32_t)smem : 0;
    dp.max_interior = p.max_interior;
    dp.max_iface = p.max_iface;
    // the staged kernel's layout depends on the envelope: it is checked in solve_dom_1st
    switch (c->opts.solve_kernel) {
      case FWGPU_SOLVE_WARP:
        dp.solve_variant = fw::kSolveWarp;
        break;
      case FWGPU_SOLVE_CTA:
        if (dp.cta_smem == 0) return set_error(FWGPU_ERR_ARG, "CTA solve kernel: subdomains too large for shared memory");
        dp.solve_variant = fw::kSolveCta;
        break;
      case FWGPU_SOLVE_GLOBAL:
        dp.solve_variant = fw::kSolveGlobal;
        break;
      case FWGPU_SOLVE_BLOCKINV:
        dp.solve_variant = fw::kSolveInv;
        break;
      default:
        dp.solve_variant = dp.cta_smem > 0 ? fw::kSolveCta : fw::kSolveGlobal;
    }
    // AUTO and BLOCKINV time the warps per subdomain; WARP times its staging capacities too
    c->solve_tuned = c->opts.solve_kernel != FWGPU_SOLVE_AUTO && c->opts.solve_kernel != FWGPU_SOLVE_WARP &&
                     c->opts.solve_kernel != FWGPU_SOLVE_BLOCKINV;
  }
  // per-entity solution source: the first subdomain holding each edge (vertex)
  std::vector<int64_t> esrc(c->n_out, -1);
  std::vector<uint8_t> seen(c->n_out, 0);
  for (int s = 0; s < nsub; s++) {
    const fw::SubHost &h = p.subs[s];
    for (int r = 0; r < h.nmp; r++) {
      const int e = h.edge_gid[r];
      if (seen[e]) continue;
      seen[e] = 1;
      if (h.cidx[r] >= 0)
        esrc[e] = p.sub_int_off[s] + h.cidx[r];
      else if (h.slot[r] >= 0)
        esrc[e] = -(p.sub_if_off[s] + h.slot[r]) - 2;
      else
        esrc[e] = -1;
    }
  }
  FW_TRY(c->upload(&c->d_edge_src, esrc));
  FW_TRY(c->alloc(&c->d_xedge, c->n_out));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

extern "C" {

const char *fwgpu_last_error(void) { return g_last_error.c_str(); }
int fwgpu_abi_version(void) { return FWGPU_ABI_VERSION; }

int fwgpu_create(const fwgpu_mesh *mesh, const fwgpu_material *mt, const fwgpu_options *opts, fwgpu_context **out) {
  Trace trace("fwgpu_create");
  if (!mesh || !mt || !opts || !out) return set_error(FWGPU_ERR_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(FWGPU_ERR_CUDA, "no CUDA device");
  if (opts->device < 0 || opts->device >= ndev) return set_error(FWGPU_ERR_ARG, "bad device ordinal");

  fwgpu_context *c = new fwgpu_context();
  c->opts = *opts;
  if (c->opts.graph_iterations <= 0) c->opts.graph_iterations = 16;
  if (c->opts.ir_max_steps <= 0) c->opts.ir_max_steps = 1;
  if (c->opts.stage_warps != 0 && c->opts.stage_warps != 1 && c->opts.stage_warps != 2 && c->opts.stage_warps != 4) {
    delete c;
    return set_error(FWGPU_ERR_ARG, "stage_warps must be 0, 1, 2 or 4");
  }
  if (c->opts.solve_kernel < FWGPU_SOLVE_AUTO || c->opts.solve_kernel > FWGPU_SOLVE_BLOCKINV) {
    delete c;
    return set_error(FWGPU_ERR_ARG, "unknown solve_kernel");
  }
  fw::Model &m = c->m;
  {
    int rc = model_from_mesh(mesh, m);
    if (rc != FWGPU_OK) {
      delete c;
      return rc;
    }
  }
  m.omega = mt->omega;
  resolve_material(m, mesh, mt);
  std::string err = fw::build_plan(m, c->p);
  if (!err.empty()) {
    delete c;
    return set_error(FWGPU_ERR_ARG, err);
  }
  c->n_out = m.ne;
  return setup_device(c, opts, out);
}

int fwgpu_partition_build(const fwgpu_mesh *mesh, fwgpu_partition **out) {
  if (!out) return set_error(FWGPU_ERR_ARG, "null argument");
  *out = nullptr;
  fwgpu_partition *part = new fwgpu_partition();
  int rc = model_from_mesh(mesh, part->m);
  if (rc != FWGPU_OK) {
    delete part;
    return rc;
  }
  std::string err = fw::build_plan(part->m, part->p);
  if (!err.empty()) {
    delete part;
    return set_error(FWGPU_ERR_ARG, err);
  }
  *out = part;
  return FWGPU_OK;
}

// -- correction-Jo problem (main/fullwave/main.c:92-98) ------------------------

int fwgpu_cojo_create(const fwgpu_mesh *mesh, int32_t antenna_flag, const uint8_t *pec_vertex,
                      const fwgpu_options *opts, fwgpu_context **out) {
  Trace trace("fwgpu_cojo_create");
  if (!mesh || !opts || !out) return set_error(FWGPU_ERR_ARG, "null argument");
  *out = nullptr;
  if (opts->precision != FWGPU_PREC_FP64) return set_error(FWGPU_ERR_ARG, "the correction-Jo problem is solved in FP64");
  if (opts->shard_begin != 0 || opts->shard_end != 0)
    return set_error(FWGPU_ERR_ARG, "the correction-Jo problem is not sharded");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(FWGPU_ERR_CUDA, "no CUDA device");
  if (opts->device < 0 || opts->device >= ndev) return set_error(FWGPU_ERR_ARG, "bad device ordinal");
  if (opts->stage_warps != 0 && opts->stage_warps != 1 && opts->stage_warps != 2 && opts->stage_warps != 4)
    return set_error(FWGPU_ERR_ARG, "stage_warps must be 0, 1, 2 or 4");
  if (opts->solve_kernel < FWGPU_SOLVE_AUTO || opts->solve_kernel > FWGPU_SOLVE_BLOCKINV)
    return set_error(FWGPU_ERR_ARG, "unknown solve_kernel");
  fwgpu_context *c = new fwgpu_context();
  c->opts = *opts;
  if (c->opts.graph_iterations <= 0) c->opts.graph_iterations = 16;
  c->opts.ir_max_steps = 1;
  fw::Model &m = c->m;
  int rc = model_from_mesh(mesh, m);
  if (rc != FWGPU_OK) {
    delete c;
    return rc;
  }
  std::vector<uint8_t> pv;
  if (pec_vertex) pv.assign(pec_vertex, pec_vertex + m.nv);
  std::string err = fw::build_plan_cojo(m, antenna_flag, pv, c->p, c->cojo_sub);
  if (!err.empty()) {
    delete c;
    return set_error(FWGPU_ERR_ARG, err);
  }
  m.nsub = (int32_t)c->cojo_sub.size();  // the problem's own subdomains from here on
  c->cojo_flag = antenna_flag;
  c->n_out = m.nv;
  return setup_device(c, &c->opts, out);
}

int fwgpu_cojo_set_current(fwgpu_context *c, const double *current) {
  if (!c || !current) return set_error(FWGPU_ERR_ARG, "null argument");
  if (c->cojo_flag < 0) return set_error(FWGPU_ERR_STATE, "not a correction-Jo context");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const int64_t nv = c->m.nv;
  if (!c->d_cojo_J) FW_TRY(c->alloc(&c->d_cojo_J, 3 * (size_t)nv));
  FW_CUDA(cudaMemcpyAsync(c->d_cojo_J, current, 3 * (size_t)nv * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FW_TRY(build_rhs_lists(c));
  fw::launch_cojo_element_rhs((int64_t)c->p.el_order.size(), c->d_el_order, c->d_tv, c->d_crd, c->d_cojo_J,
                              c->d_elrhs, c->stream);
  FW_CUDA(cudaGetLastError());
  c->el_src = true;
  return FWGPU_OK;
}

int fwgpu_cojo_solve(fwgpu_context *c, const double *current, fwgpu_result *res, double *potential) {
  Trace trace("hddm_solver_RS correct_Jo");
  FW_TRY(fwgpu_cojo_set_current(c, current));
  const int64_t nv = c->m.nv;
  // the matrix does not depend on the current: the second pass reuses the factors
  const int rc = c->stage >= 2 && c->factor_fresh ? fwgpu_hddm_resolve(c, nullptr, res)
                                                   : fwgpu_hddm_solve(c, nullptr, res);
  if (rc != FWGPU_OK && rc != FWGPU_ERR_NOT_CONVERGED) return rc;
  if (potential) {
    std::vector<double2> x(nv);
    FW_CUDA(cudaMemcpy(x.data(), c->d_xedge, nv * sizeof(double2), cudaMemcpyDeviceToHost));
    for (int64_t v = 0; v < nv; v++) potential[v] = x[v].x;
  }
  if (res) res->kernel_launches += 1;
  return rc;
}

int fwgpu_cojo_subdomains(const fwgpu_context *c, int32_t *n, int32_t *sub_ids) {
  if (!c || !n) return set_error(FWGPU_ERR_ARG, "null argument");
  if (c->cojo_flag < 0) return set_error(FWGPU_ERR_STATE, "not a correction-Jo context");
  *n = (int32_t)c->cojo_sub.size();
  if (sub_ids) std::copy(c->cojo_sub.begin(), c->cojo_sub.end(), sub_ids);
  return FWGPU_OK;
}

int fwgpu_cojo_partition_build(const fwgpu_mesh *mesh, int32_t antenna_flag, const uint8_t *pec_vertex,
                               fwgpu_partition **out) {
  if (!out) return set_error(FWGPU_ERR_ARG, "null argument");
  *out = nullptr;
  fwgpu_partition *part = new fwgpu_partition();
  int rc = model_from_mesh(mesh, part->m);
  if (rc != FWGPU_OK) {
    delete part;
    return rc;
  }
  std::vector<uint8_t> pv;
  if (pec_vertex) pv.assign(pec_vertex, pec_vertex + part->m.nv);
  std::string err = fw::build_plan_cojo(part->m, antenna_flag, pv, part->p, part->cojo_sub);
  if (!err.empty()) {
    delete part;
    return set_error(FWGPU_ERR_ARG, err);
  }
  part->m.nsub = (int32_t)part->cojo_sub.size();
  *out = part;
  return FWGPU_OK;
}

int fwgpu_cojo_partition_subdomains(const fwgpu_partition *part, int32_t *sub_ids) {
  if (!part || !sub_ids) return set_error(FWGPU_ERR_ARG, "null argument");
  if (part->cojo_sub.empty()) return set_error(FWGPU_ERR_STATE, "not a correction-Jo partition");
  std::copy(part->cojo_sub.begin(), part->cojo_sub.end(), sub_ids);
  return FWGPU_OK;
}

int fwgpu_partition_destroy(fwgpu_partition *part) {
  delete part;
  return FWGPU_OK;
}

int fwgpu_partition_info(const fwgpu_partition *part, int32_t *n_subdomains, int32_t *total_free) {
  if (!part) return set_error(FWGPU_ERR_ARG, "null partition");
  if (n_subdomains) *n_subdomains = part->m.nsub;
  if (total_free) *total_free = part->p.total_free;
  return FWGPU_OK;
}

int fwgpu_partition_maps(const fwgpu_partition *part, int32_t s, int32_t *nel, int32_t *nmp, int32_t *nbc,
                         int32_t *ninbc, int32_t *nop, int32_t *ibc, int32_t *inbc_nfid, int32_t *inbc_ln_part,
                         int32_t *edge_gid) {
  if (!part) return set_error(FWGPU_ERR_ARG, "null partition");
  return copy_maps(part->p, s, nel, nmp, nbc, ninbc, nop, ibc, inbc_nfid, inbc_ln_part, edge_gid);
}

int fwgpu_destroy(fwgpu_context *c) {
  if (!c) return FWGPU_OK;
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->multi_graph) cudaGraphExecDestroy(c->multi_graph);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void *p : c->allocs) cudaFree(p);
  if (c->h_sc) cudaFreeHost(c->h_sc);
  if (c->h_ms) cudaFreeHost(c->h_ms);
  for (auto &ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return FWGPU_OK;
}

int fwgpu_get_sizes(const fwgpu_context *c, fwgpu_sizes *sz) {
  if (!c || !sz) return set_error(FWGPU_ERR_ARG, "null argument");
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  sz->n_subdomains = nsub;
  sz->total_free = p.total_free;
  sz->total_dofs = p.sub_dof_off[nsub];
  sz->total_interior = p.sub_int_off[nsub];
  sz->nlen_reference = c->nlen_ref;
  sz->nlen_interior = c->nlen_int;
  sz->nnz_lower = p.nnz_total;
  sz->nnz_interface_rows = (int64_t)p.ifr_src.size();
  sz->nnz_coupling = (int64_t)p.cpl_src.size();
  sz->nnz_interior = (int64_t)p.aii_src.size();
  sz->total_iface_slots = p.sub_if_off[nsub];
  sz->max_local_dofs = p.max_local;
  sz->max_interior = p.max_interior;
  return FWGPU_OK;
}

int fwgpu_set_element_source(fwgpu_context *c, const fwgpu_element_source *es) {
  if (c && c->cojo_flag >= 0) return set_error(FWGPU_ERR_STATE, "a correction-Jo context solves only fwgpu_cojo_solve");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (!es) {
    c->el_src = false;
    return FWGPU_OK;
  }
  FW_CUDA(cudaSetDevice(c->opts.device));
  return set_element_source(c, es);
}

int fwgpu_make_tmp_aij(fwgpu_context *c, const fwgpu_source *src) {
  Trace trace("make_TMP_AIJ");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const fw::Plan &p = c->p;
  FW_CUDA(cudaEventRecord(c->ev[0], c->stream));
  if (!c->d_elmat) {
    FW_TRY(c->alloc(&c->d_elmat, p.el_order.size() * 72));
    FW_TRY(c->alloc(&c->d_aval, p.nnz_total));
    FW_TRY(c->upload(&c->d_cpl_src, p.cpl_src));
    FW_TRY(c->upload(&c->d_ifr_src, p.ifr_src));
    if (c->d_aii_val) FW_TRY(c->upload(&c->d_aii_src, p.aii_src));
    FW_TRY(c->upload(&c->d_diag_src, p.if_diag_src));
  }
  c->launches += 2;
  if (c->cojo_flag >= 0)
    fw::launch_cojo_element_matrices((int64_t)p.el_order.size(), c->d_el_order, c->d_tv, c->d_crd, c->d_elmat,
                                     c->d_mesh_status, c->stream);
  else
    fw::launch_element_matrices(c->m.nt, c->d_el_order, c->d_tv, c->d_crd, c->d_el_eps, c->d_el_sigma, c->m.omega,
                                c->d_elmat, c->d_mesh_status, c->stream);
  fw::launch_gather_values(p.nnz_total, c->d_cptr, c->d_contrib, (const double2 *)c->d_elmat, c->d_aval, c->stream);
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  int32_t mesh_status = 0;
  FW_CUDA(cudaMemcpy(&mesh_status, c->d_mesh_status, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (mesh_status) return set_error(FWGPU_ERR_MESH, "non-positive element volume or degenerate edge");
  FW_TRY(build_rhs(c, src));
  // operators gathered from the assembled values
  c->launches += c->d_aii_val ? 4 : 3;
  fw::launch_gather_ops((int64_t)p.cpl_src.size(), c->d_cpl_src, c->d_aval, c->d_cpl_val, c->stream);
  fw::launch_gather_ops((int64_t)p.ifr_src.size(), c->d_ifr_src, c->d_aval, c->d_ifr_val, c->stream);
  if (c->d_aii_val) fw::launch_gather_ops((int64_t)p.aii_src.size(), c->d_aii_src, c->d_aval, c->d_aii_val, c->stream);
  fw::launch_diag_pc((int64_t)p.if_diag_src.size(), c->d_diag_src, c->d_aval, c->d_pcloc, c->stream);
  FW_CUDA(cudaGetLastError());
  c->stage = 1;
  c->factor_fresh = false;
  return FWGPU_OK;
}

// Row blocks of the staged solve: at most 32 rows, and stored entries that
// fit one staging buffer, so that one bulk copy brings a whole block in.
static int stage_max_row(const fwgpu_context *c) {
  const fw::Plan &p = c->p;
  int maxrow = 0;
  for (int s = 0; s < c->m.nsub; s++) {
    const int64_t io = p.sub_int_off[s];
    const int nI = (int)(p.sub_int_off[s + 1] - io);
    for (int r = 0; r < nI; r++) maxrow = std::max(maxrow, r - c->h_env_lo[io + r] + 1);
  }
  return maxrow;
}

// Block table for staging buffers of `cap` envelope elements.
static int build_stage_blocks(fwgpu_context *c, int cap, int *max_blocks_out) {
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  std::vector<int32_t> boff(nsub + 1, 0);
  std::vector<int2> btab;
  int max_blocks = 0;
  c->h_nblk.assign(nsub, 0);
  for (int s = 0; s < nsub; s++) {
    const int64_t io = p.sub_int_off[s];
    const int nI = (int)(p.sub_int_off[s + 1] - io);
    const int64_t base = nI > 0 ? c->h_env_ptr[io] : 0;
    boff[s] = (int32_t)btab.size();
    auto row_end = [&](int r) { return (int)(c->h_env_ptr[io + r] - base) + (r - c->h_env_lo[io + r]) + 1; };
    int r = 0, nb = 0;
    while (r < nI) {
      const int r_start = r;
      const int e0 = (int)(c->h_env_ptr[io + r] - base);
      int rows = 0;
      while (r < nI && rows < 32) {
        if (rows > 0 && row_end(r) - e0 > cap - 2) break;
        r++;
        rows++;
      }
      btab.push_back(make_int2(r_start, e0));
      nb++;
    }
    btab.push_back(make_int2(nI, nI > 0 ? row_end(nI - 1) : 0));
    max_blocks = std::max(max_blocks, nb);
    c->h_nblk[s] = nb;
  }
  boff[nsub] = (int32_t)btab.size();
  c->release(c->d_blk_off);
  c->release(c->d_blk_tab);
  c->d_blk_off = nullptr;
  c->d_blk_tab = nullptr;
  FW_TRY(c->upload(&c->d_blk_off, boff));
  FW_TRY(c->upload(&c->d_blk_tab, btab));
  c->dp.blk_off = c->d_blk_off;
  c->dp.blk_tab = c->d_blk_tab;
  c->dp.max_blocks = max_blocks;
  c->dp.stage_cap = cap;
  if (c->dp.stage_warps < 1) c->dp.stage_warps = c->opts.stage_warps > 0 ? c->opts.stage_warps : 1;
  if (max_blocks_out) *max_blocks_out = max_blocks;
  return FWGPU_OK;
}

// Block-inverse layout: row blocks of at most 32 rows whose stored elements
// (the rows' entries left of the block, the block's N = (I + L_bb)^-1 - I as
// a dense strict lower triangle, and its pivots) fit one staging buffer of
// `cap` elements, each subdomain's elements from a 16-byte boundary.
static int build_inv_blocks(fwgpu_context *c, int cap) {
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  std::vector<int32_t> boff(nsub + 1, 0);
  std::vector<int2> btab;
  std::vector<int64_t> iptr(p.sub_int_off[nsub], 0);
  int max_blocks = 0, max_nI = 0;
  int64_t pos = 0;
  for (int s = 0; s < nsub; s++) {
    const int64_t io = p.sub_int_off[s];
    const int nI = (int)(p.sub_int_off[s + 1] - io);
    max_nI = std::max(max_nI, nI);
    pos = (pos + 1) & ~(int64_t)1;
    const int64_t base = pos;
    boff[s] = (int32_t)btab.size();
    auto left = [&](int r, int r0) { return std::max(0, r0 - c->h_env_lo[io + r]); };
    int r = 0, nb = 0;
    while (r < nI) {
      const int r0 = r;
      int64_t lsum = 0;
      int rows = 0;
      while (r < nI && rows < 32) {
        const int64_t size = lsum + left(r, r0) + (int64_t)(rows + 1) * rows / 2 + rows + 1;
        if (rows > 0 && size > cap - 2) break;
        lsum += left(r, r0);
        r++;
        rows++;
      }
      if (lsum + (int64_t)rows * (rows - 1) / 2 + rows > cap - 2)
        return set_error(FWGPU_ERR_ARG, "block-inverse layout: a row exceeds the staging capacity");
      btab.push_back(make_int2(r0, (int)(pos - base)));
      for (int t = r0; t < r; t++) {
        iptr[io + t] = pos;
        pos += left(t, r0);
      }
      pos += (int64_t)rows * (rows - 1) / 2 + rows;
      nb++;
    }
    btab.push_back(make_int2(nI, (int)(pos - base)));
    if (pos - base > INT32_MAX) return set_error(FWGPU_ERR_ARG, "block-inverse layout: a subdomain over 2^31 elements");
    if (nI > 0) iptr[io] = base;
    max_blocks = std::max(max_blocks, nb);
  }
  boff[nsub] = (int32_t)btab.size();
  const size_t smem = fw::subsolve_staged_smem_bytes(max_nI, max_blocks, cap, fp32);
  if (smem > 227 * 1024 || fw::configure_subsolve_inv(smem, fp32) != 0) {
    c->inv_ok = false;
    return FWGPU_OK;
  }
  FW_TRY(c->upload(&c->d_inv_blk_off, boff));
  FW_TRY(c->upload(&c->d_inv_blk_tab, btab));
  FW_TRY(c->upload(&c->d_inv_ptr, iptr));
  // padding: bulk copies of a block may read up to 16 bytes past its end
  if (fp32)
    FW_TRY(c->alloc(&c->d_Linv32, pos + 64));
  else
    FW_TRY(c->alloc(&c->d_Linv64, pos + 64));
  c->inv_len = pos;
  c->dp.inv_ptr = c->d_inv_ptr;
  c->dp.inv_blk_off = c->d_inv_blk_off;
  c->dp.inv_blk_tab = c->d_inv_blk_tab;
  c->dp.Linv64 = c->d_Linv64;
  c->dp.Linv32 = c->d_Linv32;
  c->dp.inv_max_blocks = max_blocks;
  c->dp.inv_cap = cap;
  c->inv_ok = true;
  return FWGPU_OK;
}

// Staging capacities the staged kernel can run with (shared memory of one
// warp <= 227 KB), the default one's block table, and the kernel's shared
// memory limit set for the largest of them.
static int setup_stage(fwgpu_context *c) {
  const fw::Plan &p = c->p;
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  const int min_cap = (stage_max_row(c) + 2 + 7) & ~7;
  std::vector<int> cand = fp32 ? std::vector<int>{1024, 1536, 2048, 3072} : std::vector<int>{512, 768, 1024, 1536};
  if (c->opts.stage_cap > 0) cand = {c->opts.stage_cap};
  c->stage_caps.clear();
  size_t smem_max = 0;
  for (int cap : cand) {
    cap = std::max(cap, min_cap);
    if (std::find(c->stage_caps.begin(), c->stage_caps.end(), cap) != c->stage_caps.end()) continue;
    int mb = 0;
    FW_TRY(build_stage_blocks(c, cap, &mb));
    const size_t smem = fw::subsolve_staged_smem_bytes(p.max_interior, mb, cap, fp32);
    if (smem > 227 * 1024) continue;
    c->stage_caps.push_back(cap);
    smem_max = std::max(smem_max, smem);
  }
  c->warp_ok = !c->stage_caps.empty() && fw::configure_subsolve_staged(smem_max, fp32) == 0;
  if (c->warp_ok) {
    // the default: the middle capacity
    FW_TRY(build_stage_blocks(c, c->stage_caps[(c->stage_caps.size() - 1) / 2 + (c->stage_caps.size() > 2 ? 1 : 0)],
                              nullptr));
  }
  return FWGPU_OK;
}

// Times the candidate subdomain-solve kernels on the factors just computed
// (first-solve mode, whose outputs the real first solve then overwrites) and
// keeps the fastest.
//
// The timed choice never changes the arithmetic, so that a solve gives the
// same bits on every run: AUTO times only variants that sum in the same
// order.  The staging capacity sets the row blocks, and with them the
// order of the sums, so AUTO keeps the default capacity (a rule on the
// model's envelope, setup_stage) and times one, two and four warps per
// subdomain, which share out whole row groups and column chunks and so sum
// alike.  With FP32 factors AUTO runs the block-inverse sweep (a rule, not
// a timed choice), with FP64 factors the staged sweep.  The CTA kernel sums
// in another order and runs only when asked for.  An explicit WARP choice
// times the staging capacities too.
static int tune_solve_kernel(fwgpu_context *c) {
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  struct Cand {
    int variant, cap, warps;
  };
  std::vector<Cand> cand;
  const bool any = c->opts.solve_kernel == FWGPU_SOLVE_AUTO;
  // AUTO runs the block-inverse sweep where it built that layout (FP32 factors)
  const bool any_inv = any && c->inv_ok;
  if (any && c->warp_ok && !any_inv) {
    for (int warps = 1; warps <= 4; warps *= 2)
      if (c->opts.stage_warps == 0 || c->opts.stage_warps == warps)
        cand.push_back({fw::kSolveWarp, c->dp.stage_cap, warps});
    if (cand.empty()) cand.push_back({fw::kSolveWarp, c->dp.stage_cap, c->opts.stage_warps});
  }
  if (c->opts.solve_kernel == FWGPU_SOLVE_WARP && c->warp_ok)
    for (int cap : c->stage_caps)
      for (int warps = 1; warps <= 4; warps *= 2)
        if (c->opts.stage_warps == 0 || c->opts.stage_warps == warps) cand.push_back({fw::kSolveWarp, cap, warps});
  if (any && !c->warp_ok && c->dp.cta_smem > 0) cand.push_back({fw::kSolveCta, 0, 1});
  if ((c->opts.solve_kernel == FWGPU_SOLVE_BLOCKINV || any_inv) && c->inv_ok)
    for (int warps = 1; warps <= 4; warps *= 2)
      if (c->opts.stage_warps == 0 || c->opts.stage_warps == warps)
        cand.push_back({fw::kSolveInv, c->dp.inv_cap, warps});
  if (cand.empty()) {
    c->solve_tuned = true;
    return FWGPU_OK;
  }
  float best = -1.f;
  Cand pick = cand[0];
  for (const Cand &k : cand) {
    c->dp.solve_variant = k.variant;
    c->dp.stage_warps = k.warps;
    if (k.variant == fw::kSolveWarp && c->dp.stage_cap != k.cap) FW_TRY(build_stage_blocks(c, k.cap, nullptr));
    fw::launch_subsolve(c->dp, fw::kModeFirst, fp32, c->stream);
    FW_CUDA(cudaEventRecord(c->ev[4], c->stream));
    for (int r = 0; r < 3; r++) fw::launch_subsolve(c->dp, fw::kModeFirst, fp32, c->stream);
    FW_CUDA(cudaEventRecord(c->ev[5], c->stream));
    FW_CUDA(cudaEventSynchronize(c->ev[5]));
    c->launches += 4 * fw::subsolve_launches(c->dp, fp32);
    float ms = 0.f;
    FW_CUDA(cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]));
    if (best < 0.f || ms < best) {
      best = ms;
      pick = k;
    }
  }
  c->dp.solve_variant = pick.variant;
  c->dp.stage_warps = pick.warps;
  if (pick.variant == fw::kSolveWarp && c->dp.stage_cap != pick.cap) FW_TRY(build_stage_blocks(c, pick.cap, nullptr));
  c->solve_tuned = true;
  return FWGPU_OK;
}

int fwgpu_solve_dom_1st(fwgpu_context *c) {
  Trace trace("solve_dom_1st");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->stage < 1) return set_error(FWGPU_ERR_STATE, "solve_dom_1st before make_tmp_aij");
  FW_CUDA(cudaSetDevice(c->opts.device));
  FW_TRY(clear_copy_timeout(c));
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  const int64_t ndof = p.sub_dof_off[nsub];
  if (!c->d_L64) {
    // skyline profile on the device, envelope layout on the host
    FW_TRY(c->alloc(&c->d_idx1, ndof));
    c->launches += 1;
    fw::launch_profile(nsub, c->d_dof_off, c->d_nnz_off, c->d_row_ptr, c->d_col, c->d_aval, c->d_isbc, c->d_idx1,
                       c->stream);
    c->h_idx1.resize(ndof);
    FW_CUDA(cudaMemcpyAsync(c->h_idx1.data(), c->d_idx1, ndof * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(cudaStreamSynchronize(c->stream));
    // the interior envelope of every subdomain, laid out on all host threads
    fw::EnvelopeLayout env;
    fw::envelope_layout(p, c->h_idx1.data(), env);
    c->h_env_lo.swap(env.env_lo);
    c->h_env_ptr.swap(env.env_ptr);
    const int64_t pos = env.nlen;
    c->nlen_int = env.nlen;
    c->nlen_ref = env.nlen_ref;
    FW_TRY(c->upload(&c->d_env_lo, c->h_env_lo));
    FW_TRY(c->upload(&c->d_env_ptr, c->h_env_ptr));
    FW_TRY(c->upload(&c->d_env_dst, env.dst));
    // padding: bulk copies of a block may read up to 16 bytes past its end
    FW_TRY(c->alloc(&c->d_L64, pos + 64));
    c->dp.env_lo = c->d_env_lo;
    c->dp.env_ptr = c->d_env_ptr;
    if (c->opts.precision == FWGPU_PREC_FP32_IR) FW_TRY(c->alloc(&c->d_L32, pos + 64));
    FW_TRY(setup_stage(c));
    if (c->opts.solve_kernel == FWGPU_SOLVE_WARP && !c->warp_ok)
      return set_error(FWGPU_ERR_ARG, "staged solve kernel: subdomains too large for shared memory");
    // the block-inverse layout: asked for, or AUTO with FP32 factors, where
    // it is the faster sweep (C2 12 %, C3 3 %; with FP64 factors the two
    // sweeps take the same time)
    const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
    const bool inv = c->opts.solve_kernel == FWGPU_SOLVE_BLOCKINV || (c->opts.solve_kernel == FWGPU_SOLVE_AUTO && fp32);
    if (inv && c->warp_ok) {
      // staging capacity: the caller's, else the staged kernel's, whose rule
      // was also the fastest of 1, 1.5 and 2 times it for this layout
      FW_TRY(build_inv_blocks(c, c->opts.stage_cap > 0 ? c->opts.stage_cap : c->dp.stage_cap));
    }
    if (c->opts.solve_kernel == FWGPU_SOLVE_BLOCKINV && !c->inv_ok)
      return set_error(FWGPU_ERR_ARG, "block-inverse solve kernel: subdomains too large for shared memory");
  }
  if (!c->factor_fresh) {
    // envelope values and LDL^T factor (the layout is fixed by the model)
    const int64_t pos = c->nlen_int;
    FW_CUDA(cudaMemsetAsync(c->d_L64, 0, (pos + 64) * sizeof(double2), c->stream));
    c->launches += c->opts.precision == FWGPU_PREC_FP32_IR ? 3 : 2;
    fw::launch_scatter_envelope(p.nnz_total, c->d_env_dst, c->d_aval, c->d_L64, c->stream);
    c->dp.L64 = c->d_L64;
    FW_CUDA(cudaMemsetAsync(c->d_mesh_status + 1, 0, sizeof(int32_t), c->stream));
    fw::launch_factor(c->dp, c->dp.int_off, c->d_env_lo, c->d_env_ptr, c->d_L64, c->d_mesh_status + 1, c->stream);
    FW_CUDA(cudaGetLastError());
    if (c->opts.precision == FWGPU_PREC_FP32_IR) {
      fw::launch_to_fp32(pos + 64, c->d_L64, c->d_L32, c->stream);
      c->dp.L32 = c->d_L32;
      c->dp.L64 = nullptr;
    }
    if (c->inv_ok) {
      fw::launch_inv_relayout(c->dp, c->d_L64, c->opts.precision == FWGPU_PREC_FP32_IR, c->stream);
      c->launches += 1;
    }
    int32_t fstat = 0;
    FW_CUDA(cudaMemcpyAsync(&fstat, c->d_mesh_status + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(cudaStreamSynchronize(c->stream));
    c->factor_bad = fstat != 0;
    c->factor_fresh = true;
    if (!c->solve_tuned) FW_TRY(tune_solve_kernel(c));
  }
  fw::launch_subsolve(c->dp, fw::kModeFirst, c->opts.precision == FWGPU_PREC_FP32_IR, c->stream);
  c->launches += fw::subsolve_launches(c->dp, c->opts.precision == FWGPU_PREC_FP32_IR);
  FW_CUDA(cudaGetLastError());
  c->stage = 2;
  if (c->factor_bad) return set_error(FWGPU_ERR_BREAKDOWN, "zero or non-finite pivot in a subdomain factor");
  // the timing launches and the first solve above
  FW_TRY(read_status(c, nullptr));
  return FWGPU_OK;
}

// kernels of one interface iteration: the subdomain solve and 3 COCG kernels
static int64_t iteration_launches(const fwgpu_context *c) {
  return 3 + fw::subsolve_launches(c->dp, c->opts.precision == FWGPU_PREC_FP32_IR);
}

int fwgpu_iteration_s_1st(fwgpu_context *c, int32_t *status) {
  Trace trace("iteration_s_1st");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->sharded) return set_error(FWGPU_ERR_STATE, "sharded context: use the fwgpu_shard_* calls");
  if (c->stage < 2) return set_error(FWGPU_ERR_STATE, "iteration_s_1st before solve_dom_1st");
  FW_CUDA(cudaSetDevice(c->opts.device));
  fw::launch_set_status(c->d_sc, c->opts.hddm_eps, c->opts.hddm_max_loop, c->stream);
  fw::launch_cocg_first(c->dp, c->d_pcloc, c->stream);
  c->launches += 3;
  FW_CUDA(cudaGetLastError());
  FW_TRY(read_status(c, status));
  c->stage = 3;
  return FWGPU_OK;
}

int fwgpu_iteration_s(fwgpu_context *c, int32_t *status) {
  Trace trace("iteration_s");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->sharded) return set_error(FWGPU_ERR_STATE, "sharded context: use the fwgpu_shard_* calls");
  if (c->stage != 3) return set_error(FWGPU_ERR_STATE, "iteration_s outside the interface loop");
  FW_CUDA(cudaSetDevice(c->opts.device));
  fw::launch_cocg_iteration(c->dp, c->stream);
  c->launches += iteration_launches(c);
  FW_CUDA(cudaGetLastError());
  FW_TRY(read_status(c, status));
  return FWGPU_OK;
}

// Buffers of the batched-source solve, allocated on first use.
static int multi_setup(fwgpu_context *c) {
  if (c->mp.ms) return FWGPU_OK;
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  const fw::DevProblem &dp = c->dp;
  const int64_t R = fw::kMaxRhs;
  const int64_t nI = c->p.sub_int_off[c->m.nsub], nG = c->p.sub_if_off[c->m.nsub];
  const int64_t nf = std::max<int64_t>(1, dp.nfree);
  fw::MultiProblem &m = c->mp;
  double2 *d = nullptr;
  FW_TRY(c->alloc(&d, nI * R));
  m.fI = d;
  FW_TRY(c->alloc(&d, nG * R));
  m.fG = d;
  FW_TRY(c->alloc(&m.Y, nI * R));
  FW_TRY(c->alloc(&m.V, nG * R));
  FW_TRY(c->alloc(&m.qloc, nG * R));
  FW_CUDA(cudaMemsetAsync(m.qloc, 0, nG * R * sizeof(double2), c->stream));
  if (fp32) {
    FW_TRY(c->alloc(&m.B, nI * R));
    FW_TRY(c->alloc(&m.Rres, nI * R));
    float2 *z = nullptr;
    FW_TRY(c->alloc(&z, nI * R));
    m.Zs = z;
  } else {
    double2 *z = nullptr;
    FW_TRY(c->alloc(&z, nI * R));
    m.Zs = z;
  }
  FW_TRY(c->alloc(&m.P, nf * R));
  FW_TRY(c->alloc(&m.Q, nf * R));
  FW_TRY(c->alloc(&m.R, nf * R));
  FW_TRY(c->alloc(&m.Z, nf * R));
  FW_TRY(c->alloc(&m.U, nf * R));
  FW_TRY(c->alloc(&m.PC, nf));
  FW_TRY(c->alloc(&m.part, (size_t)8 * dp.n_part_blocks * R));
  FW_TRY(c->alloc(&m.ms, 1));
  FW_CUDA(cudaMallocHost(&c->h_ms, sizeof(fw::MultiScalars)));
  return FWGPU_OK;
}

// Size buckets of the batched sweep: the subdomains in interior-size order,
// a new bucket where the size falls below 0.6 of the bucket's largest, so a
// warp's vectors of many right-hand sides take shared memory for its own size
// class, not for the largest subdomain of the model.
static void set_multi_buckets(fwgpu_context *c) {
  fw::MultiProblem &m = c->mp;
  const fw::Plan &p = c->p;
  const int n = (int)c->h_order.size();
  m.n_buckets = 0;
  int i = 0;
  while (i < n) {
    const int k = m.n_buckets;
    const int lead = p.subs[c->h_order[i]].nI;
    int j = i, mb = 0;
    const bool last = k == fw::kMaxBuckets - 1;
    while (j < n && (last || p.subs[c->h_order[j]].nI * 10 >= lead * 6 || j == i)) {
      mb = std::max(mb, c->h_nblk[c->h_order[j]]);
      j++;
    }
    m.bucket_first[k] = i;
    m.bucket_count[k] = j - i;
    m.bucket_max_interior[k] = std::max(1, lead);
    m.bucket_max_blocks[k] = std::max(1, mb);
    m.n_buckets++;
    i = j;
  }
}

static int read_multi_status(fwgpu_context *c) {
  FW_CUDA(cudaMemcpyAsync(c->h_ms, c->mp.ms, sizeof(fw::MultiScalars), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  if (c->h_ms->err != 0) return set_error(FWGPU_ERR_TIMEOUT, "subdomain solve gave up waiting for a staged copy");
  return FWGPU_OK;
}

// The batched solve of n_src sources on the context's factors (assembled and
// factored already): right-hand sides, first solves, the COCGs in lockstep,
// last solves.
static int multi_run(fwgpu_context *c, int32_t n_src, const fwgpu_source *srcs, fwgpu_result *res) {
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  c->multi_n = 0;
  if (!c->warp_ok) return set_error(FWGPU_ERR_ARG, "batched sources need the staged solve kernel");
  const size_t smem = fw::multi_smem_bytes(c->dp.max_interior, c->dp.max_blocks, c->dp.stage_cap, fp32);
  if (fw::configure_multi(smem, fp32) != 0)
    return set_error(FWGPU_ERR_ARG, "batched sources: subdomains too large for shared memory");
  set_multi_buckets(c);
  FW_TRY(multi_setup(c));
  fw::MultiProblem &m = c->mp;
  m.p = c->dp;
  // right-hand sides: column k of [row][kMaxRhs] is source k (the others zero)
  const int64_t R = fw::kMaxRhs;
  const int64_t nI = c->p.sub_int_off[c->m.nsub], nG = c->p.sub_if_off[c->m.nsub];
  FW_CUDA(cudaMemsetAsync((void *)m.fI, 0, nI * R * sizeof(double2), c->stream));
  FW_CUDA(cudaMemsetAsync((void *)m.fG, 0, nG * R * sizeof(double2), c->stream));
  for (int k = 0; k < n_src; k++) {
    FW_TRY(build_rhs(c, &srcs[k]));
    if (nI > 0)
      FW_CUDA(cudaMemcpy2DAsync((double2 *)m.fI + k, R * sizeof(double2), c->d_fI, sizeof(double2), sizeof(double2),
                                nI, cudaMemcpyDeviceToDevice, c->stream));
    if (nG > 0)
      FW_CUDA(cudaMemcpy2DAsync((double2 *)m.fG + k, R * sizeof(double2), c->d_fG, sizeof(double2), sizeof(double2),
                                nG, cudaMemcpyDeviceToDevice, c->stream));
  }
  FW_CUDA(cudaEventRecord(c->ev[0], c->stream));
  FW_CUDA(cudaMemsetAsync(&m.ms->err, 0, sizeof(int32_t), c->stream));
  fw::launch_multi_subsolve(m, fw::kModeFirst, fp32, c->stream);
  fw::launch_multi_set_status(m.ms, c->opts.hddm_eps, c->opts.hddm_max_loop, c->stream);
  fw::launch_multi_first(m, c->d_pcloc, c->stream);
  const int per_iter = fw::multi_iteration_launches(fp32, c->dp.ir_steps, c->mp.n_buckets);
  c->launches += per_iter - 3 + 2;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaEventRecord(c->ev[1], c->stream));
  if (!c->multi_graph) {
    cudaGraph_t g;
    FW_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < c->opts.graph_iterations; k++) fw::launch_multi_iteration(m, fp32, c->stream);
    FW_CUDA(cudaStreamEndCapture(c->stream, &g));
    FW_CUDA(cudaGraphInstantiate(&c->multi_graph, g, 0));
    cudaGraphDestroy(g);
  }
  FW_TRY(read_multi_status(c));
  while (c->h_ms->all_status == 0) {
    FW_CUDA(cudaGraphLaunch(c->multi_graph, c->stream));
    c->launches += (int64_t)per_iter * c->opts.graph_iterations;
    FW_TRY(read_multi_status(c));
  }
  FW_CUDA(cudaEventRecord(c->ev[2], c->stream));
  fw::launch_multi_subsolve(m, fw::kModeLast, fp32, c->stream);
  c->launches += per_iter - 3;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaEventRecord(c->ev[3], c->stream));
  FW_TRY(read_multi_status(c));
  float ms0 = 0.f, ms1 = 0.f, ms2 = 0.f;
  cudaEventElapsedTime(&ms0, c->ev[0], c->ev[1]);
  cudaEventElapsedTime(&ms1, c->ev[1], c->ev[2]);
  cudaEventElapsedTime(&ms2, c->ev[2], c->ev[3]);
  int all_conv = 1, any_bad = 0;
  for (int k = 0; k < n_src; k++) {
    const fw::CocgScalars &sc = c->h_ms->s[k];
    res[k].iterations = sc.loop - 1;
    res[k].converged = sc.converged;
    res[k].initial_norm = sc.norm0;
    res[k].final_resi = sc.resi;
    res[k].final_resi_l2 = sc.resi_l2;
    res[k].t_setup_ms = ms0;
    res[k].t_iterate_ms = ms1;
    res[k].t_last_ms = ms2;
    res[k].kernel_launches = c->launches;
    res[k].solve_kernel = fw::kSolveWarp + 1;
    res[k].stage_cap = c->dp.stage_cap;
    res[k].stage_warps = c->dp.stage_warps;
    res[k].reserved = 0;
    all_conv &= sc.converged;
    any_bad |= sc.nonfinite;
  }
  c->multi_n = n_src;
  if (any_bad) return set_error(FWGPU_ERR_NONFINITE, "an interface residual became NaN or infinite");
  return all_conv ? FWGPU_OK : set_error(FWGPU_ERR_NOT_CONVERGED, "hddm_max_loop reached before hddm_eps");
}

int fwgpu_hddm_solve_multi(fwgpu_context *c, int32_t n_src, const fwgpu_source *srcs, fwgpu_result *res) {
  Trace trace("hddm_solve_multi");
  if (c && c->cojo_flag >= 0) return set_error(FWGPU_ERR_STATE, "a correction-Jo context solves only fwgpu_cojo_solve");
  if (!c || !srcs || !res) return set_error(FWGPU_ERR_ARG, "null argument");
  if (n_src < 1 || n_src > fw::kMaxRhs) return set_error(FWGPU_ERR_ARG, "n_src outside 1..FWGPU_MAX_RHS");
  if (c->sharded) return set_error(FWGPU_ERR_STATE, "sharded context: use the fwgpu_shard_* calls");
  if (c->opts.hddm_max_loop == 0) return set_error(FWGPU_ERR_ARG, "hddm_max_loop is 0");
  c->launches = 0;
  c->multi_n = 0;
  FW_TRY(fwgpu_make_tmp_aij(c, &srcs[0]));
  FW_TRY(fwgpu_solve_dom_1st(c));
  return multi_run(c, n_src, srcs, res);
}

int fwgpu_adjoint_gradient_multi(fwgpu_context *c, int32_t n_probe, const int32_t *probe_edges, int32_t n_design,
                                 const int32_t *design_tets, double *J, double *grad_eps, double *grad_sigma,
                                 fwgpu_result *adjoint_results) {
  Trace trace("adjoint_gradient_multi");
  if (c && c->cojo_flag >= 0) return set_error(FWGPU_ERR_STATE, "a correction-Jo context solves only fwgpu_cojo_solve");
  if (!c || n_probe < 0 || n_design < 0 || (n_probe > 0 && !probe_edges) || (n_design > 0 && !design_tets))
    return set_error(FWGPU_ERR_ARG, "bad argument");
  const int n_src = c->multi_n;
  if (n_src < 1) return set_error(FWGPU_ERR_STATE, "the batched adjoint needs a batched forward solve");
  for (int k = 0; k < n_probe; k++)
    if (probe_edges[k] < 0 || probe_edges[k] >= c->m.ne) return set_error(FWGPU_ERR_ARG, "probe edge out of range");
  for (int k = 0; k < n_design; k++)
    if (design_tets[k] < 0 || design_tets[k] >= c->m.nt) return set_error(FWGPU_ERR_ARG, "design element out of range");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const int64_t ne = c->m.ne;
  if (!c->d_te) FW_TRY(c->upload(&c->d_te, c->m.te));
  // every source's forward solution, and its probe values on the host
  double2 *d_xf = nullptr;
  FW_TRY(c->alloc(&d_xf, (size_t)ne * n_src));
  std::vector<double2> probe_x((size_t)n_src * std::max(1, n_probe));
  for (int k = 0; k < n_src; k++) {
    fw::launch_multi_edge_solution(c->mp, k, ne, c->d_edge_src, d_xf + (size_t)k * ne, c->stream);
    for (int q = 0; q < n_probe; q++)
      FW_CUDA(cudaMemcpyAsync(&probe_x[(size_t)k * n_probe + q], d_xf + (size_t)k * ne + probe_edges[q],
                              sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  }
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  c->launches += n_src;
  // J_k and the adjoint sources dJ_k/dx = conj(x_k at the probes)
  std::vector<int32_t> pe(probe_edges, probe_edges + n_probe);
  std::vector<double> pv(2 * (size_t)n_src * std::max(1, n_probe));
  std::vector<fwgpu_source> srcs(n_src);
  for (int k = 0; k < n_src; k++) {
    double Jv = 0.0;
    for (int q = 0; q < n_probe; q++) {
      const double2 v = probe_x[(size_t)k * n_probe + q];
      Jv += v.x * v.x + v.y * v.y;
      pv[2 * ((size_t)k * n_probe + q)] = v.x;
      pv[2 * ((size_t)k * n_probe + q) + 1] = -v.y;
    }
    if (J) J[k] = Jv;
    srcs[k] = fwgpu_source{n_probe, pe.data(), pv.data() + 2 * (size_t)k * n_probe};
  }
  std::vector<fwgpu_result> ares(n_src);
  // the adjoint right-hand sides are dJ_k/dx alone, on the forward factors
  c->el_src_off = true;
  const int rc = multi_run(c, n_src, srcs.data(), ares.data());
  c->el_src_off = false;
  if (adjoint_results)
    for (int k = 0; k < n_src; k++) adjoint_results[k] = ares[k];
  if (rc != FWGPU_OK && rc != FWGPU_ERR_NOT_CONVERGED) {
    c->release(d_xf);
    return rc;
  }
  int32_t *d_design = nullptr;
  double *d_g = nullptr;
  std::vector<int32_t> dt(design_tets, design_tets + n_design);
  const int nd1 = std::max(1, n_design);
  FW_TRY(c->upload(&d_design, dt));
  FW_TRY(c->alloc(&d_g, 2 * (size_t)nd1));
  if (!c->d_xedge) FW_TRY(c->alloc(&c->d_xedge, ne));
  std::vector<double> gh(2 * (size_t)nd1);
  for (int k = 0; k < n_src; k++) {
    fw::launch_multi_edge_solution(c->mp, k, ne, c->d_edge_src, c->d_xedge, c->stream);
    fw::launch_adjoint_gradient(n_design, d_design, c->d_tv, c->d_te, c->d_crd, c->m.omega, d_xf + (size_t)k * ne,
                                c->d_xedge, d_g, d_g + nd1, c->stream);
    FW_CUDA(cudaGetLastError());
    FW_CUDA(cudaMemcpyAsync(gh.data(), d_g, gh.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < n_design; i++) {
      if (grad_eps) grad_eps[(size_t)k * n_design + i] = gh[i];
      if (grad_sigma) grad_sigma[(size_t)k * n_design + i] = gh[nd1 + i];
    }
  }
  c->launches += 2 * n_src;
  c->xedge_ok = false;
  c->release(d_design);
  c->release(d_g);
  c->release(d_xf);
  return rc;
}

int fwgpu_get_edge_solution_multi(fwgpu_context *c, int32_t k, double *x) {
  if (!c || !x) return set_error(FWGPU_ERR_ARG, "null argument");
  if (k < 0 || k >= c->multi_n) return set_error(FWGPU_ERR_ARG, "no such source in the last batched solve");
  FW_CUDA(cudaSetDevice(c->opts.device));
  fw::launch_multi_edge_solution(c->mp, k, c->m.ne, c->d_edge_src, c->d_xedge, c->stream);
  FW_CUDA(cudaGetLastError());
  c->xedge_ok = true;
  FW_CUDA(cudaMemcpyAsync(x, c->d_xedge, c->m.ne * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_set_layout(fwgpu_context *c, int32_t n_shards, const int32_t *shard_first, int32_t *n_shared) {
  if (c && c->cojo_flag >= 0) return set_error(FWGPU_ERR_STATE, "a correction-Jo context solves only fwgpu_cojo_solve");
  if (!c || !shard_first || n_shards < 1) return set_error(FWGPU_ERR_ARG, "bad argument");
  if (!c->sharded) return set_error(FWGPU_ERR_STATE, "not a sharded context");
  const fw::Plan &p = c->p;
  const int nsub = c->m.nsub;
  if (shard_first[0] != 0 || shard_first[n_shards] != nsub) return set_error(FWGPU_ERR_ARG, "shard ranges must cover the subdomains");
  int me = -1;
  for (int k = 0; k < n_shards; k++) {
    if (shard_first[k + 1] <= shard_first[k]) return set_error(FWGPU_ERR_ARG, "empty or decreasing shard range");
    if (shard_first[k] == c->shard_lo && shard_first[k + 1] == c->shard_hi) me = k;
  }
  if (me < 0) return set_error(FWGPU_ERR_ARG, "this context's range is not one of the shards");
  FW_CUDA(cudaSetDevice(c->opts.device));
  std::vector<int32_t> shard_of(nsub), slot_shard(p.sub_if_off[nsub]);
  for (int k = 0; k < n_shards; k++)
    for (int s = shard_first[k]; s < shard_first[k + 1]; s++) shard_of[s] = k;
  for (int s = 0; s < nsub; s++)
    for (int64_t q = p.sub_if_off[s]; q < p.sub_if_off[s + 1]; q++) slot_shard[q] = shard_of[s];
  // the slots of a DOF are in subdomain order, so its shards come in
  // ascending order: the first is its owner
  std::vector<int32_t> dof, pos;
  std::vector<uint8_t> own;
  int32_t shared = 0;
  for (int g = 0; g < p.total_free; g++) {
    int first = -1, last = -1, distinct = 0;
    bool mine = false;
    for (int t = p.gq_ptr[g]; t < p.gq_ptr[g + 1]; t++) {
      const int k = slot_shard[p.gq_slot[t]];
      if (k != last) distinct++;
      if (first < 0) first = k;
      last = k;
      mine |= k == me;
    }
    const int ps = distinct >= 2 ? shared++ : -1;
    if (mine) {
      dof.push_back(g);
      own.push_back(first == me ? 1 : 0);
      pos.push_back(ps);
    }
  }
  int32_t *d_dof = nullptr, *d_pos = nullptr;
  uint8_t *d_own = nullptr;
  FW_TRY(c->upload(&d_dof, dof));
  FW_TRY(c->upload(&d_pos, pos));
  FW_TRY(c->upload(&d_own, own));
  c->dp.dist_dof = d_dof;
  c->dp.dist_pos = d_pos;
  c->dp.dist_own = d_own;
  c->dp.dist_n = (int32_t)dof.size();
  c->dp.n_shared = shared;
  c->n_shared = shared;
  if (n_shared) *n_shared = shared;
  return FWGPU_OK;
}

int fwgpu_shard_set_exchange(fwgpu_context *c, double *d_pack, double *d_scal) {
  if (!c || !d_pack || !d_scal) return set_error(FWGPU_ERR_ARG, "null argument");
  c->d_pack = (double2 *)d_pack;
  c->d_scal = d_scal;
  c->dp.dist_pack = c->d_pack;
  c->dp.dist_scal = d_scal;
  return FWGPU_OK;
}

static int shard_ready(fwgpu_context *c) {
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->n_shared < 0) return set_error(FWGPU_ERR_STATE, "no shard layout (fwgpu_shard_set_layout)");
  if (!c->d_pack) return set_error(FWGPU_ERR_STATE, "no exchange buffers (fwgpu_shard_set_exchange)");
  FW_CUDA(cudaSetDevice(c->opts.device));
  return FWGPU_OK;
}

static int zero_pack(fwgpu_context *c, int vectors) {
  if (c->n_shared > 0)
    FW_CUDA(cudaMemsetAsync(c->d_pack, 0, (size_t)vectors * c->n_shared * sizeof(double2), c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_first(fwgpu_context *c) {
  FW_TRY(shard_ready(c));
  FW_TRY(fwgpu_solve_dom_1st(c));
  FW_TRY(zero_pack(c, 2));
  fw::launch_dist_pack(c->dp, c->d_pcloc, true, false, c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_first_sums(fwgpu_context *c) {
  FW_TRY(shard_ready(c));
  if (c->stage < 2) return set_error(FWGPU_ERR_STATE, "shard_first_sums before shard_first");
  fw::launch_set_status(c->d_sc, c->opts.hddm_eps, c->opts.hddm_max_loop, c->stream);
  fw::launch_dist_first(c->dp, c->d_pcloc, c->stream);
  c->launches += 2;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_first_finish(fwgpu_context *c, int32_t *status) {
  FW_TRY(shard_ready(c));
  if (c->stage < 2) return set_error(FWGPU_ERR_STATE, "shard_first_finish before shard_first");
  fw::launch_dist_first_finish(c->dp, c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  FW_TRY(read_status(c, status));
  c->stage = 3;
  return FWGPU_OK;
}

int fwgpu_shard_iterate(fwgpu_context *c) {
  Trace trace("shard iterate");
  FW_TRY(shard_ready(c));
  if (c->stage != 3) return set_error(FWGPU_ERR_STATE, "shard_iterate outside the interface loop");
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  fw::launch_subsolve(c->dp, fw::kModeIter, fp32, c->stream);
  FW_TRY(zero_pack(c, 1));
  fw::launch_dist_pack(c->dp, c->d_pcloc, false, true, c->stream);
  c->launches += 1 + fw::subsolve_launches(c->dp, fp32);
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_iterate_pq(fwgpu_context *c) {
  FW_TRY(shard_ready(c));
  if (c->stage != 3) return set_error(FWGPU_ERR_STATE, "shard_iterate_pq outside the interface loop");
  fw::launch_dist_pq(c->dp, c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_iterate_update(fwgpu_context *c) {
  FW_TRY(shard_ready(c));
  if (c->stage != 3) return set_error(FWGPU_ERR_STATE, "shard_iterate_update outside the interface loop");
  fw::launch_dist_update(c->dp, c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return FWGPU_OK;
}

int fwgpu_shard_iterate_finish(fwgpu_context *c, int32_t *status) {
  FW_TRY(shard_ready(c));
  if (c->stage != 3) return set_error(FWGPU_ERR_STATE, "shard_iterate_finish outside the interface loop");
  fw::launch_dist_finish(c->dp, c->stream);
  c->launches += 2;
  FW_CUDA(cudaGetLastError());
  FW_TRY(read_status(c, status));
  return FWGPU_OK;
}

int fwgpu_solve_dom_last(fwgpu_context *c) {
  Trace trace("solve_dom_last");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->stage < 3) return set_error(FWGPU_ERR_STATE, "solve_dom_last before the interface loop");
  FW_CUDA(cudaSetDevice(c->opts.device));
  fw::launch_subsolve(c->dp, fw::kModeLast, c->opts.precision == FWGPU_PREC_FP32_IR, c->stream);
  fw::launch_edge_solution(c->dp, c->n_out, c->d_edge_src, c->dp.Y, c->dp.V, c->d_xedge, c->stream);
  c->launches += 1 + fw::subsolve_launches(c->dp, c->opts.precision == FWGPU_PREC_FP32_IR);
  FW_CUDA(cudaGetLastError());
  c->stage = 4;
  FW_TRY(read_status(c, nullptr));
  c->xedge_ok = !c->sharded;
  return FWGPU_OK;
}

static int run_loop(fwgpu_context *c, fwgpu_result *res) {
  Trace trace("interface iterations");
  // interface iterations captured in a CUDA graph, graph_iterations per launch
  if (!c->graph) {
    cudaGraph_t g;
    FW_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < c->opts.graph_iterations; k++) fw::launch_cocg_iteration(c->dp, c->stream);
    FW_CUDA(cudaStreamEndCapture(c->stream, &g));
    FW_CUDA(cudaGraphInstantiate(&c->graph, g, 0));
    cudaGraphDestroy(g);
    c->graph_iters = c->opts.graph_iterations;
  }
  int32_t st = c->h_sc->status;
  while (st == 0) {
    FW_CUDA(cudaGraphLaunch(c->graph, c->stream));
    c->launches += iteration_launches(c) * (int64_t)c->graph_iters;
    FW_TRY(read_status(c, &st));
  }
  (void)res;
  return FWGPU_OK;
}

static int fill_result(fwgpu_context *c, fwgpu_result *res) {
  FW_TRY(read_status(c, nullptr));
  const fw::CocgScalars &sc = *c->h_sc;
  if (res) {
    res->iterations = sc.loop - 1;
    res->converged = sc.converged;
    res->initial_norm = sc.norm0;
    res->final_resi = sc.resi;
    res->final_resi_l2 = sc.resi_l2;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    res->t_setup_ms = ms;
    cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]);
    res->t_iterate_ms = ms;
    cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
    res->t_last_ms = ms;
    res->kernel_launches = c->launches;
    res->solve_kernel = c->dp.solve_variant + 1;
    res->stage_cap = c->dp.solve_variant == fw::kSolveWarp  ? c->dp.stage_cap
                     : c->dp.solve_variant == fw::kSolveInv ? c->dp.inv_cap
                                                            : 0;
    res->stage_warps =
        c->dp.solve_variant == fw::kSolveWarp || c->dp.solve_variant == fw::kSolveInv ? c->dp.stage_warps : 0;
    res->reserved = 0;
  }
  if (sc.nonfinite) return set_error(FWGPU_ERR_NONFINITE, "the interface residual became NaN or infinite");
  return sc.converged ? FWGPU_OK : set_error(FWGPU_ERR_NOT_CONVERGED, "hddm_max_loop reached before hddm_eps");
}

int fwgpu_hddm_solve(fwgpu_context *c, const fwgpu_source *src, fwgpu_result *res) {
  Trace trace("hddm_solver_CS");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->sharded) return set_error(FWGPU_ERR_STATE, "sharded context: use the fwgpu_shard_* calls");
  if (c->opts.hddm_max_loop == 0) return set_error(FWGPU_ERR_ARG, "hddm_max_loop is 0");
  c->launches = 0;
  FW_TRY(fwgpu_make_tmp_aij(c, src));
  FW_TRY(fwgpu_solve_dom_1st(c));
  int32_t st = 0;
  FW_TRY(fwgpu_iteration_s_1st(c, &st));
  FW_CUDA(cudaEventRecord(c->ev[1], c->stream));
  FW_TRY(run_loop(c, res));
  FW_CUDA(cudaEventRecord(c->ev[2], c->stream));
  FW_TRY(fwgpu_solve_dom_last(c));
  FW_CUDA(cudaEventRecord(c->ev[3], c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return fill_result(c, res);
}

int fwgpu_hddm_resolve(fwgpu_context *c, const fwgpu_source *src, fwgpu_result *res) {
  Trace trace("hddm_resolve");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (c->sharded) return set_error(FWGPU_ERR_STATE, "sharded context: use the fwgpu_shard_* calls");
  if (c->stage < 2) return set_error(FWGPU_ERR_STATE, "resolve before the factors exist");
  FW_CUDA(cudaSetDevice(c->opts.device));
  FW_CUDA(cudaEventRecord(c->ev[0], c->stream));
  FW_TRY(clear_copy_timeout(c));
  c->launches = 1;
  FW_TRY(build_rhs(c, src));
  fw::launch_subsolve(c->dp, fw::kModeFirst, c->opts.precision == FWGPU_PREC_FP32_IR, c->stream);
  c->launches += fw::subsolve_launches(c->dp, c->opts.precision == FWGPU_PREC_FP32_IR);
  int32_t st = 0;
  FW_TRY(fwgpu_iteration_s_1st(c, &st));
  FW_CUDA(cudaEventRecord(c->ev[1], c->stream));
  FW_TRY(run_loop(c, res));
  FW_CUDA(cudaEventRecord(c->ev[2], c->stream));
  FW_TRY(fwgpu_solve_dom_last(c));
  FW_CUDA(cudaEventRecord(c->ev[3], c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  return fill_result(c, res);
}

int fwgpu_adjoint_gradient(fwgpu_context *c, int32_t n_probe, const int32_t *probe_edges, int32_t n_design,
                           const int32_t *design_tets, double *J, double *grad_eps, double *grad_sigma,
                           fwgpu_result *adjoint_result) {
  Trace trace("adjoint_gradient");
  if (c && c->cojo_flag >= 0) return set_error(FWGPU_ERR_STATE, "a correction-Jo context solves only fwgpu_cojo_solve");
  if (!c || n_probe < 0 || n_design < 0 || (n_probe > 0 && !probe_edges) || (n_design > 0 && !design_tets))
    return set_error(FWGPU_ERR_ARG, "bad argument");
  if (c->stage < 4) return set_error(FWGPU_ERR_STATE, "adjoint needs a forward solve");
  for (int k = 0; k < n_probe; k++)
    if (probe_edges[k] < 0 || probe_edges[k] >= c->m.ne) return set_error(FWGPU_ERR_ARG, "probe edge out of range");
  for (int k = 0; k < n_design; k++)
    if (design_tets[k] < 0 || design_tets[k] >= c->m.nt) return set_error(FWGPU_ERR_ARG, "design element out of range");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const int64_t ne = c->m.ne;
  if (!c->d_xfwd) FW_TRY(c->alloc(&c->d_xfwd, ne));
  if (!c->d_te) FW_TRY(c->upload(&c->d_te, c->m.te));
  FW_CUDA(cudaMemcpyAsync(c->d_xfwd, c->d_xedge, ne * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
  std::vector<double2> xh(ne);
  FW_CUDA(cudaMemcpyAsync(xh.data(), c->d_xedge, ne * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  // J and the adjoint source dJ/dx = conj(x_P)
  double Jv = 0.0;
  std::vector<int32_t> pe(probe_edges, probe_edges + n_probe);
  std::vector<double> pv(2 * (size_t)n_probe);
  for (int k = 0; k < n_probe; k++) {
    const double2 v = xh[pe[k]];
    Jv += v.x * v.x + v.y * v.y;
    pv[2 * k] = v.x;
    pv[2 * k + 1] = -v.y;
  }
  if (J) *J = Jv;
  fwgpu_source src{n_probe, pe.data(), pv.data()};
  fwgpu_result res{};
  // the adjoint right-hand side is dJ/dx alone
  c->el_src_off = true;
  const int rc = fwgpu_hddm_resolve(c, &src, &res);
  c->el_src_off = false;
  if (adjoint_result) *adjoint_result = res;
  if (rc != FWGPU_OK && rc != FWGPU_ERR_NOT_CONVERGED) return rc;
  // gradient from the forward solution and the adjoint solution
  int32_t *d_design = nullptr;
  double *d_g = nullptr;
  std::vector<int32_t> dt(design_tets, design_tets + n_design);
  FW_TRY(c->upload(&d_design, dt));
  FW_TRY(c->alloc(&d_g, 2 * (size_t)std::max(1, n_design)));
  fw::launch_adjoint_gradient(n_design, d_design, c->d_tv, c->d_te, c->d_crd, c->m.omega, c->d_xfwd, c->d_xedge, d_g,
                              d_g + std::max(1, n_design), c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  std::vector<double> gh(2 * (size_t)std::max(1, n_design));
  FW_CUDA(cudaMemcpyAsync(gh.data(), d_g, gh.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  // the forward solution stays the context's result
  FW_CUDA(cudaMemcpyAsync(c->d_xedge, c->d_xfwd, ne * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  c->release(d_design);
  c->release(d_g);
  for (int k = 0; k < n_design; k++) {
    if (grad_eps) grad_eps[k] = gh[k];
    if (grad_sigma) grad_sigma[k] = gh[std::max(1, n_design) + k];
  }
  return rc;
}

namespace {

// Device memory of the context's device, 16-byte aligned: a kernel may read
// or write it in place.  Host memory (pageable or pinned) is not.
bool usable_on_device(const fwgpu_context *c, const void *p) {
  if (!p || ((uintptr_t)p & 15u)) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == c->opts.device;
}

int post_static_data(fwgpu_context *c) {
  if (!c->d_te) FW_TRY(c->upload(&c->d_te, c->m.te));
  if (!c->d_el_has_nu) FW_TRY(c->upload(&c->d_el_has_nu, c->m.el_has_nu));
  return FWGPU_OK;
}

}  // namespace

int fwgpu_post_em_E(fwgpu_context *c, const double *x, double *el_B, double *el_E, double *el_Je) {
  Trace trace("post_em_E");
  if (c && c->cojo_flag >= 0) return set_error(FWGPU_ERR_STATE, "a correction-Jo context solves only fwgpu_cojo_solve");
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  if (!x && !c->xedge_ok)
    return set_error(FWGPU_ERR_STATE, c->sharded ? "a sharded context needs the whole edge solution x"
                                                 : "no edge solution yet: solve first or pass x");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const int64_t nt = c->m.nt, ne = c->m.ne;
  FW_TRY(post_static_data(c));
  const double2 *dx = c->d_xedge;
  if (x) {
    if (usable_on_device(c, x)) {
      dx = reinterpret_cast<const double2 *>(x);
    } else {
      if (!c->d_post_x) FW_TRY(c->alloc(&c->d_post_x, ne));
      FW_CUDA(cudaMemcpyAsync(c->d_post_x, x, ne * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
      dx = c->d_post_x;
    }
  }
  double *user[3] = {el_B, el_E, el_Je};
  double2 *out[3] = {nullptr, nullptr, nullptr};
  bool staged[3] = {false, false, false};
  for (int k = 0; k < 3; k++) {
    if (!user[k]) continue;
    if (usable_on_device(c, user[k])) {
      out[k] = reinterpret_cast<double2 *>(user[k]);
    } else {
      if (!c->d_post) FW_TRY(c->alloc(&c->d_post, 9 * (size_t)std::max<int64_t>(1, nt)));
      out[k] = c->d_post + 3 * nt * k;
      staged[k] = true;
    }
  }
  FW_CUDA(cudaMemsetAsync(c->d_mesh_status + 2, 0, sizeof(int32_t), c->stream));
  fw::launch_post_em_E(nt, c->d_tv, c->d_te, c->d_crd, c->d_el_has_nu, c->d_el_sigma, c->m.omega, dx, out[0], out[1],
                       out[2], c->d_mesh_status + 2, c->stream);
  c->launches += 1;
  FW_CUDA(cudaGetLastError());
  for (int k = 0; k < 3; k++)
    if (staged[k])
      FW_CUDA(cudaMemcpyAsync(user[k], out[k], 3 * nt * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  int32_t bad = 0;
  FW_CUDA(cudaMemcpyAsync(&bad, c->d_mesh_status + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(cudaStreamSynchronize(c->stream));
  if (bad) return set_error(FWGPU_ERR_MESH, "degenerate element in the post step");
  return FWGPU_OK;
}

int fwgpu_profile_post(fwgpu_context *c, int32_t reps, double *kernel_ms) {
  if (!c || !kernel_ms || reps <= 0) return set_error(FWGPU_ERR_ARG, "bad argument");
  if (!c->xedge_ok) return set_error(FWGPU_ERR_STATE, "profile needs an edge solution");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const int64_t nt = c->m.nt;
  FW_TRY(post_static_data(c));
  if (!c->d_post) FW_TRY(c->alloc(&c->d_post, 9 * (size_t)std::max<int64_t>(1, nt)));
  const size_t flush_bytes = (size_t)256 << 20;
  uint8_t *flush = nullptr;
  FW_TRY(c->alloc(&flush, flush_bytes));
  cudaEvent_t a, b;
  FW_CUDA(cudaEventCreate(&a));
  FW_CUDA(cudaEventCreate(&b));
  double total = 0.0;
  int rc = FWGPU_OK;
  for (int r = 0; r <= reps && rc == FWGPU_OK; r++) {  // r = 0 is a warm-up
    cudaError_t e = cudaMemsetAsync(flush, r & 0xff, flush_bytes, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(a, c->stream);
    fw::launch_post_em_E(nt, c->d_tv, c->d_te, c->d_crd, c->d_el_has_nu, c->d_el_sigma, c->m.omega, c->d_xedge,
                         c->d_post, c->d_post + 3 * nt, c->d_post + 6 * nt, nullptr, c->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(b, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e != cudaSuccess) rc = set_error(FWGPU_ERR_CUDA, std::string("profile_post: ") + cudaGetErrorString(e));
    if (r > 0) total += ms;
  }
  c->launches += reps + 1;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  c->release(flush);
  if (rc) return rc;
  *kernel_ms = total / reps;
  return FWGPU_OK;
}

int fwgpu_profile_iteration(fwgpu_context *c, int32_t reps, fwgpu_kernel_profile *out) {
  if (!c || !out || reps <= 0) return set_error(FWGPU_ERR_ARG, "bad argument");
  if (c->stage < 3 || !c->graph) return set_error(FWGPU_ERR_STATE, "profile needs a finished solve");
  FW_CUDA(cudaSetDevice(c->opts.device));
  const bool fp32 = c->opts.precision == FWGPU_PREC_FP32_IR;
  cudaEvent_t a, b;
  FW_CUDA(cudaEventCreate(&a));
  FW_CUDA(cudaEventCreate(&b));
  fw::launch_profile_reset(c->d_sc, c->stream);
  // warm-up
  fw::launch_cocg_iteration(c->dp, c->stream);
  float ms = 0.f;
  FW_CUDA(cudaEventRecord(a, c->stream));
  for (int r = 0; r < reps; r++) fw::launch_subsolve(c->dp, fw::kModeIter, fp32, c->stream);
  FW_CUDA(cudaEventRecord(b, c->stream));
  FW_CUDA(cudaEventSynchronize(b));
  FW_CUDA(cudaEventElapsedTime(&ms, a, b));
  out->subsolve_ms = ms / reps;
  FW_CUDA(cudaEventRecord(a, c->stream));
  for (int r = 0; r < reps; r++) fw::launch_cocg_iteration(c->dp, c->stream);
  FW_CUDA(cudaEventRecord(b, c->stream));
  FW_CUDA(cudaEventSynchronize(b));
  FW_CUDA(cudaEventElapsedTime(&ms, a, b));
  out->interface_ms = ms / reps - out->subsolve_ms;
  const int launches = std::max(1, reps / std::max(1, c->graph_iters));
  FW_CUDA(cudaEventRecord(a, c->stream));
  for (int r = 0; r < launches; r++) FW_CUDA(cudaGraphLaunch(c->graph, c->stream));
  FW_CUDA(cudaEventRecord(b, c->stream));
  FW_CUDA(cudaEventSynchronize(b));
  FW_CUDA(cudaEventElapsedTime(&ms, a, b));
  out->iteration_ms = ms / (launches * c->graph_iters);
  out->reps = reps;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  FW_CUDA(cudaGetLastError());
  c->stage = 2;
  return FWGPU_OK;
}

int fwgpu_get_edge_solution(fwgpu_context *c, double *x) {
  if (!c || !x) return set_error(FWGPU_ERR_ARG, "null argument");
  if (c->stage < 4) return set_error(FWGPU_ERR_STATE, "no solution yet");
  FW_CUDA(cudaMemcpy(x, c->d_xedge, (size_t)c->n_out * sizeof(double2), cudaMemcpyDeviceToHost));
  return FWGPU_OK;
}

int fwgpu_get_history(fwgpu_context *c, double *resi, int32_t max_n, int32_t *n_out) {
  if (!c || !n_out) return set_error(FWGPU_ERR_ARG, "null argument");
  FW_TRY(read_status(c, nullptr));
  int n = std::max(0, c->h_sc->loop - 1);
  n = std::min(n, std::max(1, c->opts.hddm_max_loop));
  *n_out = n;
  if (resi && max_n > 0) FW_CUDA(cudaMemcpy(resi, c->d_hist, std::min(n, max_n) * sizeof(double), cudaMemcpyDeviceToHost));
  return FWGPU_OK;
}

int fwgpu_get_subdomain_maps(const fwgpu_context *c, int32_t s, int32_t *nel, int32_t *nmp, int32_t *nbc,
                             int32_t *ninbc, int32_t *nop, int32_t *ibc, int32_t *inbc_nfid, int32_t *inbc_ln_part,
                             int32_t *edge_gid) {
  if (!c) return set_error(FWGPU_ERR_ARG, "null context");
  return copy_maps(c->p, s, nel, nmp, nbc, ninbc, nop, ibc, inbc_nfid, inbc_ln_part, edge_gid);
}

int fwgpu_get_skyline_profile(fwgpu_context *c, int32_t s, int32_t *idx1, int32_t *idx2, int32_t *nlen) {
  if (!c || s < 0 || s >= c->m.nsub) return set_error(FWGPU_ERR_ARG, "bad subdomain");
  if (c->h_idx1.empty()) return set_error(FWGPU_ERR_STATE, "no profile yet");
  const fw::SubHost &h = c->p.subs[s];
  const int32_t *src = c->h_idx1.data() + c->p.sub_dof_off[s];
  int32_t acc = 0;
  for (int i = 0; i < h.nmp; i++) {
    if (idx1) idx1[i] = src[i];
    if (i > 0) acc += i - src[i];
    if (idx2) idx2[i] = acc;
  }
  if (nlen) *nlen = acc + h.nmp;
  return FWGPU_OK;
}

int fwgpu_get_tmp_aij(fwgpu_context *c, int32_t s, int32_t *nnz, int32_t *row_ptr, int32_t *col, double *val,
                      double *b) {
  if (!c || s < 0 || s >= c->m.nsub || !nnz) return set_error(FWGPU_ERR_ARG, "bad argument");
  if (c->stage < 1) return set_error(FWGPU_ERR_STATE, "not assembled");
  const fw::Plan &p = c->p;
  const fw::SubHost &h = p.subs[s];
  const int64_t z0 = p.sub_nnz_off[s];
  const int64_t n = p.sub_nnz_off[s + 1] - z0;
  std::vector<double2> v(n);
  FW_CUDA(cudaMemcpy(v.data(), c->d_aval + z0, n * sizeof(double2), cudaMemcpyDeviceToHost));
  // rows after DeleteZero (aij_matrix_func.h:342-391)
  int32_t k = 0;
  if (row_ptr) row_ptr[0] = 0;
  for (int r = 0; r < h.nmp; r++) {
    for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++) {
      if (v[q].x == 0.0 && v[q].y == 0.0) continue;
      if (col) col[k] = h.col[q];
      if (val) {
        val[2 * k] = v[q].x;
        val[2 * k + 1] = v[q].y;
      }
      k++;
    }
    if (row_ptr) row_ptr[r + 1] = k;
  }
  *nnz = k;
  if (b) {
    std::vector<double2> bl(c->h_b_local.begin() + p.sub_dof_off[s], c->h_b_local.begin() + p.sub_dof_off[s + 1]);
    if (c->el_src && c->d_b_local)
      FW_CUDA(cudaMemcpy(bl.data(), c->d_b_local + p.sub_dof_off[s], h.nmp * sizeof(double2), cudaMemcpyDeviceToHost));
    for (int r = 0; r < h.nmp; r++) {
      b[2 * r] = bl[r].x;
      b[2 * r + 1] = bl[r].y;
    }
  }
  return FWGPU_OK;
}

int fwgpu_get_factor(fwgpu_context *c, int32_t s, double *mat) {
  if (!c || s < 0 || s >= c->m.nsub || !mat) return set_error(FWGPU_ERR_ARG, "bad argument");
  if (c->stage < 2 || !c->d_L64) return set_error(FWGPU_ERR_STATE, "no FP64 factor");
  const fw::Plan &p = c->p;
  const fw::SubHost &h = p.subs[s];
  const int64_t io = p.sub_int_off[s];
  const int64_t b0 = h.nI > 0 ? c->h_env_ptr[io] : 0;
  const int64_t b1 = h.nI > 0 ? c->h_env_ptr[io + h.nI - 1] + (h.nI - 1 - c->h_env_lo[io + h.nI - 1]) + 1 : 0;
  std::vector<double2> L(b1 - b0);
  if (b1 > b0) FW_CUDA(cudaMemcpy(L.data(), c->d_L64 + b0, (b1 - b0) * sizeof(double2), cudaMemcpyDeviceToHost));
  const int32_t *idx1 = c->h_idx1.data() + p.sub_dof_off[s];
  int64_t idx2 = 0;
  for (int i = 0; i < h.nmp; i++) {
    if (i > 0) idx2 += i - idx1[i];
    for (int j = idx1[i]; j <= i; j++) {
      double2 val = make_double2(0.0, 0.0);
      if (h.cidx[i] < 0) {
        if (j == i) val = make_double2(1.0, 0.0);
      } else if (h.cidx[j] >= 0) {
        const int cI = h.cidx[i];
        val = L[c->h_env_ptr[io + cI] - b0 + (h.cidx[j] - c->h_env_lo[io + cI])];
      }
      mat[2 * (idx2 + j)] = val.x;
      mat[2 * (idx2 + j) + 1] = val.y;
    }
  }
  return FWGPU_OK;
}

}  // extern "C"
