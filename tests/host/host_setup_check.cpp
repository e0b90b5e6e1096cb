// CPU check of the host setup's threaded builders (adventure_fullwave_b200/
// csrc/fw_build.cpp): fw::global_rows and fw::envelope_layout against plain
// serial restatements of the same maps, on a model given as raw arrays.
// Usage: host_setup_check <dir> <n_subdomains>; <dir> holds crd.bin (f64),
// tv.bin, te.bin, flag.bin, sub.bin (i32) and pec.bin (u8).  Prints the sizes
// and exits 0 when every array is identical.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "fw_internal.h"

template <typename T>
static std::vector<T> rd(const std::string &f) {
  std::ifstream in(f, std::ios::binary | std::ios::ate);
  const size_t n = in.tellg();
  in.seekg(0);
  std::vector<T> v(n / sizeof(T));
  in.read((char *)v.data(), n);
  return v;
}

template <typename A, typename B>
static bool same(const char *what, const A &a, const B &b) {
  const bool ok = a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(a[0])) == 0);
  if (!ok) std::printf("differs: %s\n", what);
  return ok;
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const std::string d = argv[1];
  fw::Model m;
  m.crd = rd<double>(d + "/crd.bin");
  m.tv = rd<int32_t>(d + "/tv.bin");
  m.te = rd<int32_t>(d + "/te.bin");
  m.flag = rd<int32_t>(d + "/flag.bin");
  m.pec = rd<uint8_t>(d + "/pec.bin");
  m.sub_of_tet = rd<int32_t>(d + "/sub.bin");
  m.nv = (int32_t)(m.crd.size() / 3);
  m.nt = (int32_t)(m.tv.size() / 4);
  m.ne = (int32_t)m.pec.size();
  m.nsub = std::stoi(argv[2]);
  fw::Plan p;
  const std::string err = fw::build_plan(m, p);
  if (!err.empty()) {
    std::printf("plan: %s\n", err.c_str());
    return 1;
  }
  const int nsub = m.nsub;
  // serial restatement: per-subdomain list offsets, then each subdomain's rows
  auto offs = [&](const fw::HostVec<int32_t> &rel, const std::vector<int64_t> &cnt) {
    std::vector<int64_t> o(nsub + 1, 0);
    for (int s = 0; s < nsub; s++) o[s + 1] = o[s] + rel[cnt[s + 1] + s];
    return o;
  };
  const auto cpl_off = offs(p.cpl_ptr, p.sub_int_off), ifr_off = offs(p.ifr_ptr, p.sub_if_off),
             aii_off = offs(p.aii_ptr, p.sub_int_off);
  const int64_t nI_all = p.sub_int_off[nsub], nG_all = p.sub_if_off[nsub];
  std::vector<int64_t> crp(nI_all + 1, 0), irp(nG_all + 1, 0), arp(nI_all + 1, 0);
  std::vector<int32_t> cg(p.cpl_col.size()), ig(p.ifr_col.size()), ag(p.aii_col.size());
  for (int s = 0; s < nsub; s++) {
    const int64_t io = p.sub_int_off[s], go = p.sub_if_off[s];
    const int nI = (int)(p.sub_int_off[s + 1] - io), nG = (int)(p.sub_if_off[s + 1] - go);
    for (int c = 0; c <= nI; c++) {
      crp[io + c] = cpl_off[s] + p.cpl_ptr[io + s + c];
      arp[io + c] = aii_off[s] + p.aii_ptr[io + s + c];
    }
    for (int k = 0; k <= nG; k++) irp[go + k] = ifr_off[s] + p.ifr_ptr[go + s + k];
    for (int64_t q = cpl_off[s]; q < cpl_off[s + 1]; q++) cg[q] = p.if_ln[go + p.cpl_col[q]];
    for (int64_t q = ifr_off[s]; q < ifr_off[s + 1]; q++) {
      const int col = p.ifr_col[q];
      ig[q] = col >= 0 ? (int32_t)(io + col) : -p.if_ln[go + (-col - 1)] - 1;
    }
    for (int64_t q = aii_off[s]; q < aii_off[s + 1]; q++) ag[q] = (int32_t)(io + p.aii_col[q]);
  }
  fw::GlobalRows g;
  fw::global_rows(p, g);
  bool ok = same("cpl_off", g.cpl_off, cpl_off) && same("ifr_off", g.ifr_off, ifr_off) &&
            same("aii_off", g.aii_off, aii_off) && same("cpl_rowptr", g.cpl_rowptr, crp) &&
            same("ifr_rowptr", g.ifr_rowptr, irp) && same("aii_rowptr", g.aii_rowptr, arp) &&
            same("cpl_gcol", g.cpl_gcol, cg) && same("ifr_gcol", g.ifr_gcol, ig) && same("aii_gcol", g.aii_gcol, ag);
  // a profile to lay out: the first non-Dirichlet column of every row
  std::vector<int32_t> idx1(p.sub_dof_off[nsub]);
  for (int s = 0; s < nsub; s++) {
    const fw::SubHost &h = p.subs[s];
    for (int r = 0; r < h.nmp; r++) {
      int first = r;
      if (!h.isbc[r])
        for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++)
          if (!h.isbc[h.col[q]]) {
            first = h.col[q];
            break;
          }
      idx1[p.sub_dof_off[s] + r] = first;
    }
  }
  // serial restatement of the envelope layout
  std::vector<int32_t> lo_s(nI_all, 0);
  std::vector<int64_t> ptr_s(nI_all, 0), dst_s(p.nnz_total, -1);
  int64_t pos = 0, nref = 0;
  for (int s = 0; s < nsub; s++) {
    const fw::SubHost &h = p.subs[s];
    const int32_t *i1 = idx1.data() + p.sub_dof_off[s];
    pos = (pos + 1) & ~(int64_t)1;
    int64_t idx2 = 0;
    for (int i = 1; i < h.nmp; i++) idx2 += i - i1[i];
    nref += idx2 + h.nmp;
    const int64_t io = p.sub_int_off[s], z0 = p.sub_nnz_off[s];
    for (int r = 0; r < h.nmp; r++) {
      const int c = h.cidx[r];
      if (c < 0) continue;
      lo_s[io + c] = h.cidx[i1[r]];
      ptr_s[io + c] = pos;
      pos += c - lo_s[io + c] + 1;
    }
    for (int r = 0; r < h.nmp; r++) {
      const int c = h.cidx[r];
      if (c < 0) continue;
      for (int q = h.row_ptr[r]; q < h.row_ptr[r + 1]; q++) {
        const int cj = h.cidx[h.col[q]];
        if (cj >= 0 && cj >= lo_s[io + c]) dst_s[z0 + q] = ptr_s[io + c] + (cj - lo_s[io + c]);
      }
    }
  }
  fw::EnvelopeLayout e;
  fw::envelope_layout(p, idx1.data(), e);
  ok = ok && same("env_lo", e.env_lo, lo_s) && same("env_ptr", e.env_ptr, ptr_s) && same("dst", e.dst, dst_s);
  if (e.nlen != pos || e.nlen_ref != nref) {
    std::printf("differs: lengths\n");
    ok = false;
  }
  std::printf("subdomains %d interior rows %lld lower entries %lld envelope %lld: %s\n", nsub, (long long)nI_all,
              (long long)p.nnz_total, (long long)pos, ok ? "identical" : "DIFFERENT");
  return ok ? 0 : 1;
}
