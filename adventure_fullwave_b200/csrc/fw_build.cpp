// Host-side integer setup of the HDDM hot path: subdomain-local numbering,
// Dirichlet lists, interface maps and the index lists the device gathers use.
//
// For one part this is what the reference's make_PartMesh_FW
// (lib/hddm/make_PartMesh.c:1201-1241) leaves in every DomMesh:
//   - local vertex ids ("ap") are ranks of the subdomain's vertex nodes and
//     local edge DOF ids are ranks of its mid-edge nodes, both in subdomain
//     node order (make_MESH_make_ap / make_MESH_change_ap,
//     lib/fem/make_MESH.c:237-272,539-552); subdomain node order is
//     ascending global node id with vertices before mid-edge nodes;
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
#include <numeric>

#include "fw_internal.h"

namespace fw {

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

  std::vector<int32_t> eloc(m.ne, -1), vloc(m.nv, -1);
  p.sub_dof_off.assign(nsub + 1, 0);
  p.sub_nnz_off.assign(nsub + 1, 0);
  p.sub_int_off.assign(nsub + 1, 0);
  p.sub_if_off.assign(nsub + 1, 0);

  for (int s = 0; s < nsub; s++) {
    SubHost &h = p.subs[s];
    const int64_t e0 = p.sub_el_off[s], e1 = p.sub_el_off[s + 1];
    const int nel = (int)(e1 - e0);
    h.els.assign(p.el_order.begin() + e0, p.el_order.begin() + e1);
    std::vector<int32_t> ve, vv;
    ve.reserve(nel * 2);
    vv.reserve(nel);
    for (int k = 0; k < nel; k++) {
      int t = h.els[k];
      for (int i = 0; i < 6; i++) ve.push_back(m.te[6 * (int64_t)t + i]);
      for (int i = 0; i < 4; i++) vv.push_back(m.tv[4 * (int64_t)t + i]);
    }
    std::sort(ve.begin(), ve.end());
    ve.erase(std::unique(ve.begin(), ve.end()), ve.end());
    std::sort(vv.begin(), vv.end());
    vv.erase(std::unique(vv.begin(), vv.end()), vv.end());
    h.nmp = (int32_t)ve.size();
    h.nap = (int32_t)vv.size();
    h.edge_gid = ve;
    for (int i = 0; i < h.nmp; i++) eloc[ve[i]] = i;
    for (int i = 0; i < h.nap; i++) vloc[vv[i]] = i;
    h.nop.resize((size_t)nel * 10);
    for (int k = 0; k < nel; k++) {
      int t = h.els[k];
      for (int i = 0; i < 4; i++) h.nop[10 * k + i] = vloc[m.tv[4 * (int64_t)t + i]];
      for (int i = 0; i < 6; i++) h.nop[10 * k + 4 + i] = eloc[m.te[6 * (int64_t)t + kFileSlot[i]]];
    }
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

    // structural lower rows: entry (row = larger DOF, col = smaller DOF) of
    // every element, value M[slot(row)][slot(col)] (aij_matrix_func.h:278-322)
    struct Ent {
      int32_t row, col;
      int64_t contrib;
    };
    std::vector<Ent> ents;
    ents.reserve((size_t)nel * 21);
    for (int k = 0; k < nel; k++) {
      const int32_t *d = &h.nop[10 * k + 4];
      int64_t base = (e0 + k) * 36;
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++)
          if (d[i] >= d[j]) ents.push_back({d[i], d[j], base + i * 6 + j});
    }
    // stable: keeps element order inside every (row, col)
    std::stable_sort(ents.begin(), ents.end(), [](const Ent &a, const Ent &b) {
      return a.row != b.row ? a.row < b.row : a.col < b.col;
    });
    h.row_ptr.assign(h.nmp + 1, 0);
    h.col.clear();
    const int64_t nnz0 = (int64_t)p.csr_col.size();
    for (size_t q = 0; q < ents.size(); q++) {
      bool fresh = q == 0 || ents[q].row != ents[q - 1].row || ents[q].col != ents[q - 1].col;
      if (fresh) {
        h.col.push_back(ents[q].col);
        h.row_ptr[ents[q].row + 1]++;
        p.contrib_ptr.push_back((int64_t)p.contrib.size());
      }
      p.contrib.push_back(ents[q].contrib);
    }
    for (int i = 0; i < h.nmp; i++) h.row_ptr[i + 1] += h.row_ptr[i];
    const int64_t nnz = (int64_t)h.col.size();
    p.csr_row_ptr.insert(p.csr_row_ptr.end(), h.row_ptr.begin(), h.row_ptr.end());
    p.csr_col.insert(p.csr_col.end(), h.col.begin(), h.col.end());
    p.isbc.insert(p.isbc.end(), h.isbc.begin(), h.isbc.end());

    // symmetric adjacency with lower-CSR positions
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
          adj_src[fill[r]++] = nnz0 + q;
          if (c != r) {
            adj_col[fill[c]] = r;
            adj_src[fill[c]++] = nnz0 + q;
          }
        }
      // rows of the adjacency sorted by column
      for (int r = 0; r < h.nmp; r++) {
        std::vector<std::pair<int32_t, int64_t>> tmp;
        for (int q = adj_cnt[r]; q < adj_cnt[r + 1]; q++) tmp.push_back({adj_col[q], adj_src[q]});
        std::sort(tmp.begin(), tmp.end());
        for (int q = adj_cnt[r], u = 0; q < adj_cnt[r + 1]; q++, u++) {
          adj_col[q] = tmp[u].first;
          adj_src[q] = tmp[u].second;
        }
      }
    }
    auto diag_pos = [&](int r) -> int64_t {
      for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++)
        if (h.col[q] == r) return nnz0 + q;
      return -1;
    };
    // interior rows: coupling to the interface and the interior operator
    p.cpl_ptr.push_back(0);
    p.aii_ptr.push_back(0);
    int32_t cpl_n = 0, aii_n = 0;
    for (int r = 0; r < h.nmp; r++) {
      if (h.isbc[r]) continue;
      p.int_local.push_back(r);
      p.int_diag_src.push_back(diag_pos(r));
      for (int q = adj_cnt[r]; q < adj_cnt[r + 1]; q++) {
        int c = adj_col[q];
        if (h.slot[c] >= 0) {
          p.cpl_col.push_back(h.slot[c]);
          p.cpl_src.push_back(adj_src[q]);
          cpl_n++;
        } else if (!h.isbc[c]) {
          p.aii_col.push_back(h.cidx[c]);
          p.aii_src.push_back(adj_src[q]);
          aii_n++;
        }
      }
      p.cpl_ptr.push_back(cpl_n);
      p.aii_ptr.push_back(aii_n);
    }
    // interface rows: q = A(G, :) x with x = (interior solution, interface values)
    p.ifr_ptr.push_back(0);
    int32_t ifr_n = 0;
    for (int k = 0; k < h.nG; k++) {
      int r = h.inbc_nfid[k];
      p.if_ln.push_back(h.inbc_ln[k]);
      p.if_local.push_back(r);
      p.if_diag_src.push_back(diag_pos(r));
      for (int q = adj_cnt[r]; q < adj_cnt[r + 1]; q++) {
        int c = adj_col[q];
        if (!h.isbc[c]) {
          p.ifr_col.push_back(h.cidx[c]);
        } else if (h.slot[c] >= 0) {
          p.ifr_col.push_back(-(h.slot[c] + 1));
        } else {
          continue;  // PEC column: the solution is zero there
        }
        p.ifr_src.push_back(adj_src[q]);
        ifr_n++;
      }
      p.ifr_ptr.push_back(ifr_n);
    }

    p.sub_dof_off[s + 1] = p.sub_dof_off[s] + h.nmp;
    p.sub_nnz_off[s + 1] = p.sub_nnz_off[s] + nnz;
    p.sub_int_off[s + 1] = p.sub_int_off[s] + h.nI;
    p.sub_if_off[s + 1] = p.sub_if_off[s] + h.nG;
    p.max_local = std::max(p.max_local, h.nmp);
    p.max_interior = std::max(p.max_interior, h.nI);
    p.max_iface = std::max(p.max_iface, h.nG);
    for (int i = 0; i < h.nmp; i++) eloc[ve[i]] = -1;
    for (int i = 0; i < h.nap; i++) vloc[vv[i]] = -1;
  }
  p.nnz_total = (int64_t)p.csr_col.size();
  p.contrib_ptr.push_back((int64_t)p.contrib.size());

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
  return "";
}

}  // namespace fw
