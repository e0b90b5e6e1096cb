// Host-side integer setup of the HDDM hot path: subdomain-local numbering,
// Dirichlet lists, interface maps and the index lists the device gathers use.
//
// For one part this is what the reference's make_PartMesh_FW
// (lib/hddm/make_PartMesh.c:1201-1241) leaves in every DomMesh:
//   - local vertex ids ("ap") are ranks of the subdomain's vertex nodes and
//     local edge DOF ids are ranks of its mid-edge nodes, both in subdomain
//     node order (make_MESH_make_ap / make_MESH_change_ap,
//     lib/fem/make_MESH.c:237-272,539-552); subdomain node order is the
//     caller's (the part file's node order, fwgpu_mesh sub_*_order) or else
//     ascending global node id;
//   - nop holds local ids with the mid-node slots 8 and 9 swapped
//     (make_MESH_change_nop, lib/fem/make_MESH.c:556-585);
//   - interface DOFs are the mid-edge nodes shared by two or more subdomains
//     that are not on the PEC wall (Pinbc 1st-4th passes and change_Inbc,
//     make_PartMesh.c:158-248,393-748 with make_nf_A_Method :1603-1624),
//     numbered in part-interface order (ascending global node id);
//   - inbc is sorted by local DOF id and the Dirichlet list is the sorted PEC
//     DOFs followed by the interface DOFs (change_dbc_Axn0_2nd/3rd,
//     make_PartMesh.c:1068-1163, sort_inbc :1167-1194).
#include <algorithm>
#include <array>
#include <atomic>
#include <numeric>
#include <string>
#include <thread>

#include "fw_internal.h"

namespace fw {

namespace {

// Index lists of one subdomain, with positions local to it: src entries
// count from the subdomain's first lower-CSR entry, contrib_cnt gives the
// contributions of each of its entries.  build_plan concatenates them.
struct SubLists {
  std::vector<int64_t> contrib;
  std::vector<int32_t> contrib_cnt;
  std::vector<int32_t> int_local, cpl_ptr, cpl_col, aii_ptr, aii_col, if_ln, if_local, ifr_ptr, ifr_col;
  std::vector<int64_t> int_diag_src, cpl_src, aii_src, if_diag_src, ifr_src;
  std::string err;  // non-empty: the subdomain's given local order is not a permutation of its nodes
};

// per-thread scratch: global edge / vertex id -> local id, -1 elsewhere
struct Scratch {
  std::vector<int32_t> eloc, vloc;
  struct Ent {
    int32_t row, col;
    int64_t contrib;
  };
  std::vector<Ent> ents, tmp;
  std::vector<int32_t> count;
};

void build_lists(SubHost &h, SubLists &L, Scratch &w, int64_t e0, int nel, int nd);

void build_sub(const Model &m, const Plan &p, const std::vector<int32_t> &iface_of_edge, int s, SubHost &h,
               SubLists &L, Scratch &w) {
  const int64_t e0 = p.sub_el_off[s], e1 = p.sub_el_off[s + 1];
  const int nel = (int)(e1 - e0);
  h.els.assign(p.el_order.begin() + e0, p.el_order.begin() + e1);
  // the subdomain's edges and vertices once each (the scratch maps mark
  // them; the marks are overwritten by the local ids below), ascending
  std::vector<int32_t> ve, vv;
  ve.reserve(nel * 2);
  vv.reserve(nel);
  for (int k = 0; k < nel; k++) {
    int t = h.els[k];
    for (int i = 0; i < 6; i++) {
      const int32_t e = m.te[6 * (int64_t)t + i];
      if (w.eloc[e] < 0) {
        w.eloc[e] = 0;
        ve.push_back(e);
      }
    }
    for (int i = 0; i < 4; i++) {
      const int32_t v = m.tv[4 * (int64_t)t + i];
      if (w.vloc[v] < 0) {
        w.vloc[v] = 0;
        vv.push_back(v);
      }
    }
  }
  std::sort(ve.begin(), ve.end());
  std::sort(vv.begin(), vv.end());
  if (!m.sub_eptr.empty()) {
    // the caller's local order (the part file's node order): the same sets
    std::vector<int32_t> ge(m.sub_eord.begin() + m.sub_eptr[s], m.sub_eord.begin() + m.sub_eptr[s + 1]);
    std::vector<int32_t> gv(m.sub_vord.begin() + m.sub_vptr[s], m.sub_vord.begin() + m.sub_vptr[s + 1]);
    std::vector<int32_t> se(ge), sv(gv);
    std::sort(se.begin(), se.end());
    std::sort(sv.begin(), sv.end());
    if (se != ve || sv != vv) {
      L.err = "subdomain " + std::to_string(s) + ": the given local order does not list its vertices and edges once each";
      for (int32_t e : ve) w.eloc[e] = -1;
      for (int32_t v : vv) w.vloc[v] = -1;
      return;
    }
    ve.swap(ge);
    vv.swap(gv);
  }
  h.nmp = (int32_t)ve.size();
  h.nap = (int32_t)vv.size();
  h.edge_gid = ve;
  for (int i = 0; i < h.nmp; i++) w.eloc[ve[i]] = i;
  for (int i = 0; i < h.nap; i++) w.vloc[vv[i]] = i;
  h.nop.resize((size_t)nel * 10);
  for (int k = 0; k < nel; k++) {
    int t = h.els[k];
    for (int i = 0; i < 4; i++) h.nop[10 * k + i] = w.vloc[m.tv[4 * (int64_t)t + i]];
    for (int i = 0; i < 6; i++) h.nop[10 * k + 4 + i] = w.eloc[m.te[6 * (int64_t)t + kFileSlot[i]]];
  }
  for (int i = 0; i < h.nmp; i++) w.eloc[ve[i]] = -1;
  for (int i = 0; i < h.nap; i++) w.vloc[vv[i]] = -1;
  // Dirichlet list: PEC then interface (both ascending local id)
  h.isbc.assign(h.nmp, 0);
  h.cidx.assign(h.nmp, -1);
  h.slot.assign(h.nmp, -1);
  std::vector<int32_t> pecl;
  for (int i = 0; i < h.nmp; i++) {
    int e = ve[i];
    if (m.pec[e]) {
      pecl.push_back(i);
      h.isbc[i] = 1;
    } else if (iface_of_edge[e] >= 0) {
      h.slot[i] = (int32_t)h.inbc_nfid.size();
      h.inbc_nfid.push_back(i);
      h.inbc_ln.push_back(iface_of_edge[e]);
      h.isbc[i] = 1;
    }
  }
  h.npec = (int32_t)pecl.size();
  h.ibc = pecl;
  h.ibc.insert(h.ibc.end(), h.inbc_nfid.begin(), h.inbc_nfid.end());
  h.nG = (int32_t)h.inbc_nfid.size();
  int nI = 0;
  for (int i = 0; i < h.nmp; i++)
    if (!h.isbc[i]) h.cidx[i] = nI++;
  h.nI = nI;
  build_lists(h, L, w, e0, nel, 6);
}

// The lower-row structure, the element contributions of every lower entry
// and the per-iteration operator lists of one subdomain whose element k
// holds the nd local DOFs h.nop[10k+4 .. 10k+4+nd-1] (nd = 6 edges, or 4
// vertices for the correction-Jo problem); the element matrix of slot e0+k
// is stored as 6x6 complex entries from (e0+k)*36, DOF pair (i, j) at i*6+j.
void build_lists(SubHost &h, SubLists &L, Scratch &w, int64_t e0, int nel, int nd) {
  // structural lower rows: entry (row = larger DOF, col = smaller DOF) of
  // every element, value M[slot(row)][slot(col)] (aij_matrix_func.h:278-322);
  // contributions stay in element order inside every (row, col): two stable
  // counting passes, by column and then by row
  auto &ents = w.ents;
  ents.clear();
  for (int k = 0; k < nel; k++) {
    const int32_t *d = &h.nop[10 * k + 4];
    int64_t base = (e0 + k) * 36;
    for (int i = 0; i < nd; i++)
      for (int j = 0; j < nd; j++)
        if (d[i] >= d[j]) ents.push_back({d[i], d[j], base + i * 6 + j});
  }
  w.tmp.resize(ents.size());
  for (int pass = 0; pass < 2; pass++) {
    w.count.assign(h.nmp + 1, 0);
    for (const auto &x : ents) w.count[(pass ? x.row : x.col) + 1]++;
    for (int i = 0; i < h.nmp; i++) w.count[i + 1] += w.count[i];
    for (const auto &x : ents) w.tmp[w.count[pass ? x.row : x.col]++] = x;
    ents.swap(w.tmp);
  }
  h.row_ptr.assign(h.nmp + 1, 0);
  h.col.clear();
  L.contrib.resize(ents.size());
  for (size_t q = 0; q < ents.size(); q++) {
    bool fresh = q == 0 || ents[q].row != ents[q - 1].row || ents[q].col != ents[q - 1].col;
    if (fresh) {
      h.col.push_back(ents[q].col);
      h.row_ptr[ents[q].row + 1]++;
      L.contrib_cnt.push_back(0);
    }
    L.contrib_cnt.back()++;
    L.contrib[q] = ents[q].contrib;
  }
  for (int i = 0; i < h.nmp; i++) h.row_ptr[i + 1] += h.row_ptr[i];

  // symmetric adjacency with lower-CSR positions.  Rows are filled in
  // ascending order, a row's own lower entries (ascending columns) first and
  // the entries above the diagonal as later rows reach them, so every
  // adjacency row comes out sorted by column.
  std::vector<int32_t> adj_cnt(h.nmp + 1, 0);
  for (int r = 0; r < h.nmp; r++)
    for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++) {
      adj_cnt[r + 1]++;
      if (h.col[q] != r) adj_cnt[h.col[q] + 1]++;
    }
  for (int i = 0; i < h.nmp; i++) adj_cnt[i + 1] += adj_cnt[i];
  std::vector<int32_t> adj_col(adj_cnt[h.nmp]);
  std::vector<int64_t> adj_src(adj_cnt[h.nmp]);
  {
    std::vector<int32_t> fill(adj_cnt.begin(), adj_cnt.end() - 1);
    for (int r = 0; r < h.nmp; r++)
      for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++) {
        int c = h.col[q];
        adj_col[fill[r]] = c;
        adj_src[fill[r]++] = q;
        if (c != r) {
          adj_col[fill[c]] = r;
          adj_src[fill[c]++] = q;
        }
      }
  }
  auto diag_pos = [&](int r) -> int64_t {
    for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++)
      if (h.col[q] == r) return q;
    return -1;
  };
  // interior rows: coupling to the interface and the interior operator
  L.cpl_ptr.push_back(0);
  L.aii_ptr.push_back(0);
  int32_t cpl_n = 0, aii_n = 0;
  for (int r = 0; r < h.nmp; r++) {
    if (h.isbc[r]) continue;
    L.int_local.push_back(r);
    L.int_diag_src.push_back(diag_pos(r));
    for (int q = adj_cnt[r]; q < adj_cnt[r + 1]; q++) {
      int c = adj_col[q];
      if (h.slot[c] >= 0) {
        L.cpl_col.push_back(h.slot[c]);
        L.cpl_src.push_back(adj_src[q]);
        cpl_n++;
      } else if (!h.isbc[c]) {
        L.aii_col.push_back(h.cidx[c]);
        L.aii_src.push_back(adj_src[q]);
        aii_n++;
      }
    }
    L.cpl_ptr.push_back(cpl_n);
    L.aii_ptr.push_back(aii_n);
  }
  // interface rows: q = A(G, :) x with x = (interior solution, interface values)
  L.ifr_ptr.push_back(0);
  int32_t ifr_n = 0;
  for (int k = 0; k < h.nG; k++) {
    int r = h.inbc_nfid[k];
    L.if_ln.push_back(h.inbc_ln[k]);
    L.if_local.push_back(r);
    L.if_diag_src.push_back(diag_pos(r));
    for (int q = adj_cnt[r]; q < adj_cnt[r + 1]; q++) {
      int c = adj_col[q];
      if (!h.isbc[c]) {
        L.ifr_col.push_back(h.cidx[c]);
      } else if (h.slot[c] >= 0) {
        L.ifr_col.push_back(-(h.slot[c] + 1));
      } else {
        continue;  // PEC column: the solution is zero there
      }
      L.ifr_src.push_back(adj_src[q]);
      ifr_n++;
    }
    L.ifr_ptr.push_back(ifr_n);
  }
}

// Concatenates the subdomains' lists in subdomain order (offsets first, then
// every subdomain's slice on all host threads) and builds the gather of Q.
void finish_plan(Plan &p, const std::vector<SubLists> &lists) {
  const int nsub = (int)p.subs.size();
  // concatenated in subdomain order: offsets first, then every subdomain's
  // slice written on all host threads
  p.sub_dof_off.assign(nsub + 1, 0);
  p.sub_nnz_off.assign(nsub + 1, 0);
  p.sub_int_off.assign(nsub + 1, 0);
  p.sub_if_off.assign(nsub + 1, 0);
  enum { kContrib, kNnz, kDof, kRowPtr, kInt, kIntPtr, kCpl, kAii, kIf, kIfPtr, kIfr, kLists };
  std::vector<std::array<int64_t, kLists>> off(nsub + 1);
  off[0].fill(0);
  for (int s = 0; s < nsub; s++) {
    const SubHost &h = p.subs[s];
    const SubLists &L = lists[s];
    const int64_t n[kLists] = {(int64_t)L.contrib.size(), (int64_t)h.col.size(), h.nmp, h.nmp + 1,
                               (int64_t)L.int_local.size(), (int64_t)L.cpl_ptr.size(), (int64_t)L.cpl_col.size(),
                               (int64_t)L.aii_col.size(), (int64_t)L.if_ln.size(), (int64_t)L.ifr_ptr.size(),
                               (int64_t)L.ifr_col.size()};
    for (int k = 0; k < kLists; k++) off[s + 1][k] = off[s][k] + n[k];
    p.sub_dof_off[s + 1] = p.sub_dof_off[s] + h.nmp;
    p.sub_nnz_off[s + 1] = p.sub_nnz_off[s] + (int64_t)h.col.size();
    p.sub_int_off[s + 1] = p.sub_int_off[s] + h.nI;
    p.sub_if_off[s + 1] = p.sub_if_off[s] + h.nG;
    p.max_local = std::max(p.max_local, h.nmp);
    p.max_interior = std::max(p.max_interior, h.nI);
    p.max_iface = std::max(p.max_iface, h.nG);
  }
  const auto &tot = off[nsub];
  p.contrib.resize(tot[kContrib]);
  p.contrib_ptr.resize(tot[kNnz] + 1);
  p.csr_col.resize(tot[kNnz]);
  p.csr_row_ptr.resize(tot[kRowPtr]);
  p.isbc.resize(tot[kDof]);
  p.int_local.resize(tot[kInt]);
  p.int_diag_src.resize(tot[kInt]);
  p.cpl_ptr.resize(tot[kIntPtr]);
  p.aii_ptr.resize(tot[kIntPtr]);
  p.cpl_col.resize(tot[kCpl]);
  p.cpl_src.resize(tot[kCpl]);
  p.aii_col.resize(tot[kAii]);
  p.aii_src.resize(tot[kAii]);
  p.if_ln.resize(tot[kIf]);
  p.if_local.resize(tot[kIf]);
  p.if_diag_src.resize(tot[kIf]);
  p.ifr_ptr.resize(tot[kIfPtr]);
  p.ifr_col.resize(tot[kIfr]);
  p.ifr_src.resize(tot[kIfr]);
  {
    auto copy_to = [](auto &dst, int64_t at, const auto &src) { std::copy(src.begin(), src.end(), dst.begin() + at); };
    // src positions are local to the subdomain; -1 (no diagonal) stays -1
    auto copy_src = [](HostVec<int64_t> &dst, int64_t at, const std::vector<int64_t> &src, int64_t nnz0) {
      for (size_t i = 0; i < src.size(); i++) dst[at + i] = src[i] < 0 ? src[i] : src[i] + nnz0;
    };
    std::atomic<int> next(0);
    auto worker = [&]() {
      for (int s = next++; s < nsub; s = next++) {
        const SubHost &h = p.subs[s];
        const SubLists &L = lists[s];
        const auto &o = off[s];
        const int64_t nnz0 = o[kNnz];
        copy_to(p.contrib, o[kContrib], L.contrib);
        int64_t c = o[kContrib];
        for (size_t q = 0; q < L.contrib_cnt.size(); q++) {
          p.contrib_ptr[nnz0 + q] = c;
          c += L.contrib_cnt[q];
        }
        copy_to(p.csr_col, nnz0, h.col);
        copy_to(p.csr_row_ptr, o[kRowPtr], h.row_ptr);
        copy_to(p.isbc, o[kDof], h.isbc);
        copy_to(p.int_local, o[kInt], L.int_local);
        copy_src(p.int_diag_src, o[kInt], L.int_diag_src, nnz0);
        copy_to(p.cpl_ptr, o[kIntPtr], L.cpl_ptr);
        copy_to(p.aii_ptr, o[kIntPtr], L.aii_ptr);
        copy_to(p.cpl_col, o[kCpl], L.cpl_col);
        copy_src(p.cpl_src, o[kCpl], L.cpl_src, nnz0);
        copy_to(p.aii_col, o[kAii], L.aii_col);
        copy_src(p.aii_src, o[kAii], L.aii_src, nnz0);
        copy_to(p.if_ln, o[kIf], L.if_ln);
        copy_to(p.if_local, o[kIf], L.if_local);
        copy_src(p.if_diag_src, o[kIf], L.if_diag_src, nnz0);
        copy_to(p.ifr_ptr, o[kIfPtr], L.ifr_ptr);
        copy_to(p.ifr_col, o[kIfr], L.ifr_col);
        copy_src(p.ifr_src, o[kIfr], L.ifr_src, nnz0);
      }
    };
    const int nthreads = std::max(1, std::min<int>(nsub, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
  }
  p.nnz_total = tot[kNnz];
  p.contrib_ptr[tot[kNnz]] = tot[kContrib];

  // Q[g] = sum over the subdomains holding g, in subdomain order
  // (COM_RES_SP_FUNC, hddm_solver_sp.h:41-54, called per subdomain in order)
  std::vector<int32_t> gcnt(p.total_free + 1, 0);
  for (int s = 0; s < nsub; s++)
    for (int32_t ln : p.subs[s].inbc_ln) gcnt[ln + 1]++;
  for (int g = 0; g < p.total_free; g++) gcnt[g + 1] += gcnt[g];
  p.gq_ptr = gcnt;
  p.gq_slot.resize(gcnt[p.total_free]);
  {
    std::vector<int32_t> fill(gcnt.begin(), gcnt.end() - 1);
    for (int s = 0; s < nsub; s++) {
      const SubHost &h = p.subs[s];
      for (int k = 0; k < h.nG; k++) p.gq_slot[fill[h.inbc_ln[k]]++] = p.sub_if_off[s] + k;
    }
  }
}

}  // namespace

std::string build_plan(const Model &m, Plan &p) {
  const int nsub = m.nsub;
  if (nsub <= 0 || m.nt <= 0 || m.ne <= 0 || m.nv <= 0) return "empty model";
  p = Plan();
  p.subs.resize(nsub);

  // elements of each subdomain in ascending global id (counting sort)
  std::vector<int64_t> cnt(nsub + 1, 0);
  for (int t = 0; t < m.nt; t++) {
    int s = m.sub_of_tet[t];
    if (s < 0 || s >= nsub) return "sub_of_tet out of range";
    cnt[s + 1]++;
  }
  for (int s = 0; s < nsub; s++) {
    if (cnt[s + 1] == 0) return "empty subdomain " + std::to_string(s);
    cnt[s + 1] += cnt[s];
  }
  p.sub_el_off = cnt;
  p.el_order.resize(m.nt);
  {
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int t = 0; t < m.nt; t++) p.el_order[pos[m.sub_of_tet[t]]++] = t;
  }

  // how many subdomains hold each edge; the first one is its owner
  std::vector<int32_t> ecount(m.ne, 0), eowner(m.ne, -1), mark(m.ne, -1);
  for (int s = 0; s < nsub; s++) {
    for (int64_t k = p.sub_el_off[s]; k < p.sub_el_off[s + 1]; k++) {
      int t = p.el_order[k];
      for (int i = 0; i < 6; i++) {
        int e = m.te[6 * (int64_t)t + i];
        if (e < 0 || e >= m.ne) return "tet_edges out of range";
        if (mark[e] != s) {
          mark[e] = s;
          ecount[e]++;
          if (eowner[e] < 0) eowner[e] = s;
        }
      }
    }
  }
  for (int64_t k = 0; k < 4 * (int64_t)m.nt; k++)
    if (m.tv[k] < 0 || m.tv[k] >= m.nv) return "tet_vertices out of range";
  // part-level interface DOFs in ascending global edge id
  std::vector<int32_t> iface_of_edge(m.ne, -1);
  for (int e = 0; e < m.ne; e++) {
    if (ecount[e] >= 2 && !m.pec[e]) {
      iface_of_edge[e] = (int32_t)p.iface_gid.size();
      p.iface_gid.push_back(e);
      p.iface_owner_sub.push_back(eowner[e]);
    }
  }
  p.total_free = (int32_t)p.iface_gid.size();

  // the subdomains are independent: built on all host threads
  std::vector<SubLists> lists(nsub);
  {
    const int nthreads = std::max(1, std::min<int>(nsub, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next(0);
    auto worker = [&]() {
      Scratch w;
      w.eloc.assign(m.ne, -1);
      w.vloc.assign(m.nv, -1);
      for (int s = next++; s < nsub; s = next++) build_sub(m, p, iface_of_edge, s, p.subs[s], lists[s], w);
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
  }
  for (int s = 0; s < nsub; s++)
    if (!lists[s].err.empty()) return lists[s].err;

  finish_plan(p, lists);
  return "";
}


// The correction-Jo problem of one antenna (main/fullwave/main.c:92-98):
// nodal unknowns at the vertices of the antenna's elements, with the
// integer setup the reference makes in make_PartMesh_FW:
//   - a subdomain's DOFs are the vertices of its elements whose flag is the
//     antenna's, in the subdomain's vertex order (ap order), numbered
//     0, 1, ... in that order (enf, make_PartMesh_make_ANTENNA_make_enf,
//     lib/hddm/make_PartMesh.c:973-983 with make_MESH.c:459-500);
//   - interface DOFs are the antenna vertices held by two or more subdomains
//     (make_PartMesh_FW_change_innerbc_ANTENNA with its make_nf,
//     make_PartMesh.c:1288-1340,1546-1575) that are not on a Dirichlet list
//     (the pass that excludes essential BCs, :393-421), numbered in ascending
//     global vertex id;
//   - the Dirichlet list is the sorted PEC antenna DOFs, then the interface
//     DOFs in ascending local id; a subdomain with neither holds its DOF 0 at
//     zero (make_PartMesh_make_ANTENNA_change_bc / _add_inbc,
//     make_PartMesh.c:986-1063).
// Only subdomains with antenna elements enter the problem: sub_map gives
// the original subdomain id of each.
std::string build_plan_cojo(const Model &m, int32_t antenna_flag, const std::vector<uint8_t> &pec_vertex, Plan &p,
                            std::vector<int32_t> &sub_map) {
  const int nsub_all = m.nsub;
  if (nsub_all <= 0 || m.nt <= 0 || m.nv <= 0) return "empty model";
  if (!pec_vertex.empty() && (int64_t)pec_vertex.size() != m.nv) return "pec_vertex must hold one flag per vertex";
  p = Plan();
  p.el_dofs = 4;
  sub_map.clear();
  for (int64_t k = 0; k < 4 * (int64_t)m.nt; k++)
    if (m.tv[k] < 0 || m.tv[k] >= m.nv) return "tet_vertices out of range";
  // antenna elements of each subdomain, ascending global id
  std::vector<int64_t> cnt(nsub_all + 1, 0);
  for (int t = 0; t < m.nt; t++) {
    const int s = m.sub_of_tet[t];
    if (s < 0 || s >= nsub_all) return "sub_of_tet out of range";
    if (m.flag[t] == antenna_flag) cnt[s + 1]++;
  }
  std::vector<int32_t> rs_of(nsub_all, -1);
  for (int s = 0; s < nsub_all; s++)
    if (cnt[s + 1] > 0) {
      rs_of[s] = (int32_t)sub_map.size();
      sub_map.push_back(s);
    }
  const int nsub = (int)sub_map.size();
  if (nsub == 0) return "no element carries the antenna flag";
  p.sub_el_off.assign(nsub + 1, 0);
  for (int r = 0; r < nsub; r++) p.sub_el_off[r + 1] = p.sub_el_off[r] + cnt[sub_map[r] + 1];
  p.el_order.resize(p.sub_el_off[nsub]);
  {
    std::vector<int64_t> pos(p.sub_el_off.begin(), p.sub_el_off.end() - 1);
    for (int t = 0; t < m.nt; t++)
      if (m.flag[t] == antenna_flag) p.el_order[pos[rs_of[m.sub_of_tet[t]]]++] = t;
  }
  // each subdomain's antenna vertices in its vertex order
  std::vector<std::vector<int32_t>> dofs(nsub);
  std::vector<int32_t> vcount(m.nv, 0), mark(m.nv, -1);
  for (int r = 0; r < nsub; r++) {
    std::vector<int32_t> &d = dofs[r];
    for (int64_t k = p.sub_el_off[r]; k < p.sub_el_off[r + 1]; k++)
      for (int i = 0; i < 4; i++) {
        const int v = m.tv[4 * (int64_t)p.el_order[k] + i];
        if (mark[v] != r) {
          mark[v] = r;
          d.push_back(v);
          vcount[v]++;
        }
      }
    if (!m.sub_vptr.empty()) {
      const int s = sub_map[r];
      std::vector<int32_t> ord;
      ord.reserve(d.size());
      for (int64_t q = m.sub_vptr[s]; q < m.sub_vptr[s + 1]; q++)
        if (mark[m.sub_vord[q]] == r) ord.push_back(m.sub_vord[q]);
      if (ord.size() != d.size())
        return "subdomain " + std::to_string(s) + ": the given vertex order misses an antenna vertex";
      d.swap(ord);
    } else {
      std::sort(d.begin(), d.end());
    }
  }
  std::vector<int32_t> iface_of_vertex(m.nv, -1), vowner(m.nv, -1);
  for (int r = 0; r < nsub; r++)
    for (int v : dofs[r])
      if (vowner[v] < 0) vowner[v] = r;
  for (int v = 0; v < m.nv; v++)
    if (vcount[v] >= 2 && (pec_vertex.empty() || !pec_vertex[v])) {
      iface_of_vertex[v] = (int32_t)p.iface_gid.size();
      p.iface_gid.push_back(v);
      p.iface_owner_sub.push_back(vowner[v]);
    }
  p.total_free = (int32_t)p.iface_gid.size();

  p.subs.resize(nsub);
  std::vector<SubLists> lists(nsub);
  Scratch w;
  w.vloc.assign(m.nv, -1);
  for (int r = 0; r < nsub; r++) {
    SubHost &h = p.subs[r];
    const std::vector<int32_t> &d = dofs[r];
    const int64_t e0 = p.sub_el_off[r];
    const int nel = (int)(p.sub_el_off[r + 1] - e0);
    h.els.assign(p.el_order.begin() + e0, p.el_order.begin() + p.sub_el_off[r + 1]);
    h.nmp = h.nap = (int32_t)d.size();
    h.edge_gid = d;
    for (int i = 0; i < h.nmp; i++) w.vloc[d[i]] = i;
    h.nop.assign((size_t)nel * 10, -1);
    for (int k = 0; k < nel; k++)
      for (int i = 0; i < 4; i++) {
        const int32_t loc = w.vloc[m.tv[4 * (int64_t)h.els[k] + i]];
        h.nop[10 * k + i] = loc;
        h.nop[10 * k + 4 + i] = loc;
      }
    for (int i = 0; i < h.nmp; i++) w.vloc[d[i]] = -1;
    h.isbc.assign(h.nmp, 0);
    h.cidx.assign(h.nmp, -1);
    h.slot.assign(h.nmp, -1);
    std::vector<int32_t> pecl;
    for (int i = 0; i < h.nmp; i++) {
      const int v = d[i];
      if (!pec_vertex.empty() && pec_vertex[v]) {
        pecl.push_back(i);
        h.isbc[i] = 1;
      }
      if (iface_of_vertex[v] >= 0) {
        h.slot[i] = (int32_t)h.inbc_nfid.size();
        h.inbc_nfid.push_back(i);
        h.inbc_ln.push_back(iface_of_vertex[v]);
        h.isbc[i] = 1;
      }
    }
    if (pecl.empty() && h.inbc_nfid.empty() && h.nmp > 0) {
      pecl.push_back(0);  // the pinned DOF: zero, like a PEC DOF
      h.isbc[0] = 1;
    }
    h.npec = (int32_t)pecl.size();
    h.ibc = pecl;
    h.ibc.insert(h.ibc.end(), h.inbc_nfid.begin(), h.inbc_nfid.end());
    h.nG = (int32_t)h.inbc_nfid.size();
    int nI = 0;
    for (int i = 0; i < h.nmp; i++)
      if (!h.isbc[i]) h.cidx[i] = nI++;
    h.nI = nI;
    build_lists(h, lists[r], w, e0, nel, 4);
  }
  finish_plan(p, lists);
  return "";
}


namespace {

// fn(s) for every subdomain s, on all host threads (each call writes slices
// of its own).
template <typename F>
void for_each_subdomain(int nsub, F fn) {
  const int nthreads = std::max(1, std::min<int>(nsub, (int)std::thread::hardware_concurrency()));
  std::atomic<int> next(0);
  auto worker = [&]() {
    for (int s = next++; s < nsub; s = next++) fn(s);
  };
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
}

// per-subdomain offsets of lists whose per-row pointers are stored per
// subdomain (rows + 1 entries each, concatenated)
std::vector<int64_t> offsets_from_rel(const HostVec<int32_t> &rel_ptr, const std::vector<int64_t> &count_off,
                                      int nsub) {
  std::vector<int64_t> off(nsub + 1, 0);
  for (int s = 0; s < nsub; s++) off[s + 1] = off[s] + rel_ptr[count_off[s + 1] + s];
  return off;
}

}  // namespace

void global_rows(const Plan &p, GlobalRows &g) {
  const int nsub = (int)p.subs.size();
  g.cpl_off = offsets_from_rel(p.cpl_ptr, p.sub_int_off, nsub);
  g.ifr_off = offsets_from_rel(p.ifr_ptr, p.sub_if_off, nsub);
  g.aii_off = offsets_from_rel(p.aii_ptr, p.sub_int_off, nsub);
  const int64_t nI_all = p.sub_int_off[nsub], nG_all = p.sub_if_off[nsub];
  g.cpl_rowptr.resize(nI_all + 1);
  g.aii_rowptr.resize(nI_all + 1);
  g.ifr_rowptr.resize(nG_all + 1);
  g.cpl_gcol.resize(p.cpl_col.size());
  g.ifr_gcol.resize(p.ifr_col.size());
  g.aii_gcol.resize(p.aii_col.size());
  for_each_subdomain(nsub, [&](int s) {
    const int64_t io = p.sub_int_off[s], go = p.sub_if_off[s];
    const int nI = (int)(p.sub_int_off[s + 1] - io), nG = (int)(p.sub_if_off[s + 1] - go);
    for (int cI = 0; cI < nI; cI++) {
      g.cpl_rowptr[io + cI] = g.cpl_off[s] + p.cpl_ptr[io + s + cI];
      g.aii_rowptr[io + cI] = g.aii_off[s] + p.aii_ptr[io + s + cI];
    }
    for (int k = 0; k < nG; k++) g.ifr_rowptr[go + k] = g.ifr_off[s] + p.ifr_ptr[go + s + k];
    for (int64_t q = g.cpl_off[s]; q < g.cpl_off[s + 1]; q++) g.cpl_gcol[q] = p.if_ln[go + p.cpl_col[q]];
    for (int64_t q = g.ifr_off[s]; q < g.ifr_off[s + 1]; q++) {
      const int col = p.ifr_col[q];
      g.ifr_gcol[q] = col >= 0 ? (int32_t)(io + col) : -p.if_ln[go + (-col - 1)] - 1;
    }
    for (int64_t q = g.aii_off[s]; q < g.aii_off[s + 1]; q++) g.aii_gcol[q] = (int32_t)(io + p.aii_col[q]);
  });
  // every subdomain's rows end where the next one's begin
  g.cpl_rowptr[nI_all] = g.cpl_off[nsub];
  g.aii_rowptr[nI_all] = g.aii_off[nsub];
  g.ifr_rowptr[nG_all] = g.ifr_off[nsub];
}

void envelope_layout(const Plan &p, const int32_t *idx1, EnvelopeLayout &e) {
  const int nsub = (int)p.subs.size();
  const int64_t nI_tot = p.sub_int_off[nsub];
  e.env_lo.assign(nI_tot, 0);
  e.env_ptr.assign(nI_tot, 0);
  e.dst.resize(p.nnz_total);
  // per subdomain: its interior envelope length and the reference's skyline length
  std::vector<int64_t> len(nsub), ref(nsub), start(nsub);
  for_each_subdomain(nsub, [&](int s) {
    const SubHost &h = p.subs[s];
    const int32_t *i1 = idx1 + p.sub_dof_off[s];
    int64_t idx2 = 0;
    for (int i = 1; i < h.nmp; i++) idx2 += i - i1[i];
    ref[s] = idx2 + h.nmp;
    int64_t n = 0;
    for (int r = 0; r < h.nmp; r++) {
      const int cI = h.cidx[r];
      if (cI >= 0) n += cI - h.cidx[i1[r]] + 1;
    }
    len[s] = n;
  });
  int64_t pos = 0, nref = 0;
  for (int s = 0; s < nsub; s++) {
    pos = (pos + 1) & ~(int64_t)1;  // every subdomain's envelope starts 16-byte aligned in FP32 too
    start[s] = pos;
    pos += len[s];
    nref += ref[s];
  }
  e.nlen = pos;
  e.nlen_ref = nref;
  for_each_subdomain(nsub, [&](int s) {
    const SubHost &h = p.subs[s];
    const int32_t *i1 = idx1 + p.sub_dof_off[s];
    const int64_t io = p.sub_int_off[s], z0 = p.sub_nnz_off[s];
    int64_t at = start[s];
    for (int r = 0; r < h.nmp; r++) {
      const int cI = h.cidx[r];
      if (cI < 0) continue;
      const int lo = h.cidx[i1[r]];
      e.env_lo[io + cI] = lo;
      e.env_ptr[io + cI] = at;
      at += cI - lo + 1;
    }
    for (int r = 0; r < h.nmp; r++) {
      const int cI = h.cidx[r];
      const int lo = cI >= 0 ? e.env_lo[io + cI] : 0;
      for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++) {
        const int cj = h.cidx[h.col[q]];
        e.dst[z0 + q] = (cI < 0 || cj < 0 || cj < lo) ? -1 : e.env_ptr[io + cI] + (cj - lo);
      }
    }
  });
}

}  // namespace fw
