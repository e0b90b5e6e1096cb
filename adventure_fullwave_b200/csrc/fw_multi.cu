// Batched right-hand sides: up to kMaxRhs sources solved together on one set
// of subdomain factors (the reference solves one source per HDDM run,
// hddm_solver.h:25-183; several sources are several runs of the same loop).
//
// Every vector is stored right-hand-side minor, [row][kMaxRhs], so that the
// 16 values of one DOF are one 256-byte (FP64) line.  The subdomain phase of
// an iteration is three launches, as in the single-source staged path:
//   multi_rhs_kernel     f_I - A_IG v for every (interior row, source),
//   multi_sweep_kernel   the envelope sweeps, 16/kRW warps per subdomain
//                        with kRW sources each: lane groups take the kRW
//                        sources and split every row's dot product; the
//                        factor entries come from the TMA-staged row blocks
//                        as shared-memory broadcasts, so one staged block
//                        serves kRW sources and one row's dependent chain is
//                        shared by all of them,
//   multi_iface_kernel   q = A_G.[x; v] (- f_G) for every (slot, source).
// The COCG kernels keep one set of scalars and a stopping status per source
// (ITERATION_S, hddm_solver_s.h:260-400, per source); a finished source
// keeps its vectors while the others go on.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "fw_device.cuh"
#include "fw_kernels.cuh"

namespace fw {

namespace {

using namespace dev;

constexpr int kR = kMaxRhs;
constexpr int kMT = 256;  // reduction blocks: 16 DOFs x 16 sources
enum { kMPqRe = 0, kMPqIm, kMMax, kMRzRe, kMRzIm, kML2, kMFields };

__device__ __forceinline__ bool multi_stopped(const MultiProblem &m, int mode) {
  return mode == kModeIter && m.ms->all_status != 0;
}

// ---- grid-wide products, one thread per (row, source) -----------------------

__global__ void multi_rhs_kernel(MultiProblem m, int mode, double2 *__restrict__ out) {
  if (multi_stopped(m, mode)) return;
  const DevProblem &p = m.p;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (int)(t % kR);
  const int64_t i = t / kR;
  if (i >= p.n_interior) return;
  const int64_t row = p.row0 + i;
  double2 acc = cz();
  if (mode != kModeFirst) {
    const int64_t q1 = p.cpl_rowptr[row + 1];
    for (int64_t q = p.cpl_rowptr[row]; q < q1; q++)
      acc = cadd(acc, cmul(p.cpl_val[q], m.P[(int64_t)p.cpl_gcol[q] * kR + r]));
  }
  out[row * kR + r] = csub(mode != kModeIter ? m.fI[row * kR + r] : cz(), acc);
}

__global__ void multi_iface_kernel(MultiProblem m, int mode) {
  if (multi_stopped(m, mode)) return;
  const DevProblem &p = m.p;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (int)(t % kR);
  const int64_t i = t / kR;
  if (i >= p.n_slots) return;
  const int64_t slot = p.slot0 + i;
  const bool with_bc = mode != kModeFirst;
  double2 acc = cz();
  const int64_t q1 = p.ifr_rowptr[slot + 1];
  for (int64_t q = p.ifr_rowptr[slot]; q < q1; q++) {
    const int64_t g = p.ifr_gcol[q];
    const double2 x = g >= 0 ? m.Y[g * kR + r] : (with_bc ? m.P[(-g - 1) * kR + r] : cz());
    acc = cadd(acc, cmul(p.ifr_val[q], x));
  }
  if (mode != kModeIter) acc = csub(acc, m.fG[slot * kR + r]);
  m.qloc[slot * kR + r] = acc;
  if (mode == kModeLast) m.V[slot * kR + r] = with_bc ? m.P[(int64_t)p.if_ln[slot] * kR + r] : cz();
}

__global__ void multi_residual_kernel(MultiProblem m, int mode) {
  if (multi_stopped(m, mode)) return;
  const DevProblem &p = m.p;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (int)(t % kR);
  const int64_t i = t / kR;
  if (i >= p.n_interior) return;
  const int64_t row = p.row0 + i;
  double2 acc = cz();
  const int64_t q1 = p.aii_rowptr[row + 1];
  for (int64_t q = p.aii_rowptr[row]; q < q1; q++)
    acc = cadd(acc, cmul(p.aii_val[q], m.Y[(int64_t)p.aii_gcol[q] * kR + r]));
  m.Rres[row * kR + r] = csub(m.B[row * kR + r], acc);
}

// ---- the sweeps --------------------------------------------------------------

struct MultiLayout {
  size_t y, buf0, buf1, meta, rect, bar, blk, total;
};

__host__ __device__ inline MultiLayout multi_layout(int max_interior, int max_blocks, int cap, bool fp32, int rw) {
  const size_t es = fp32 ? 8 : 16;
  MultiLayout l;
  size_t o = 0;
  l.y = o;
  o += a16((size_t)max_interior * rw * es);
  l.buf0 = o;
  o += a16((size_t)cap * es);
  l.buf1 = o;
  o += a16((size_t)cap * es);
  l.meta = o;
  o += 32 * 8;
  l.rect = o;
  o += a16((size_t)32 * rw * es);
  l.bar = o;
  o += 16;
  l.blk = o;
  o += a16(((size_t)max_blocks + 1) * 8);
  l.total = o;
  return l;
}

// Sources per sweep warp: 16 / kRW warps share a subdomain, each with kRW of
// the 16 sources; lane = (group h, source r), kQ = 32 / kRW groups.  Per
// staged block of rows r0 .. r0+nb-1:
//   forward  - the entries left of the block for all its rows at once: group
//              h takes rows h, h+kQ, ..., one accumulator per (row, source),
//              the row's entries in order; no row waits for another.  Then
//              the triangle row by row, y_i = b_i - (left_i + sum over the
//              block's columns), the groups splitting the block's columns
//              (shuffles add them), z_i = y_i / d_i;
//   backward - the triangle row by row from the last: x_t final, then
//              y_c -= L_tc x_t for the block's columns of row t; then the
//              columns left of the block for all its rows: column c belongs to
//              group c % kQ, which applies the rows from the last to the
//              first in place, so no row waits for another.
// Each (c, r) has one writer.  y holds the warp's kRW sources, [row][kRW].
template <typename T, int kRW>
__global__ void __launch_bounds__(32) multi_sweep_kernel(MultiProblem m, int mode, const double2 *rhs,
                                                        double2 *xout, T *zstash, int accumulate, MultiLayout lay,
                                                        int first) {
  constexpr int kQ = 32 / kRW;
  constexpr int kWarps = kR / kRW;
  if (multi_stopped(m, mode)) return;
  const DevProblem &p = m.p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x;
  const int r = lane & (kRW - 1);
  const int h = lane / kRW;
  const int part = blockIdx.x % kWarps;  // which kRW sources
  const int s = p.sub_order[first + blockIdx.x / kWarps];
  const int64_t io = p.int_off[s];
  const int nI = (int)(p.int_off[s + 1] - io);
  const int b0 = p.blk_off[s];
  const int nblk = p.blk_off[s + 1] - b0 - 1;
  if (nI == 0 || nblk <= 0) return;
  T *__restrict__ y = (T *)(smem_raw + lay.y);
  int2 *meta = (int2 *)(smem_raw + lay.meta);
  T *rect = (T *)(smem_raw + lay.rect);
  int2 *blk = (int2 *)(smem_raw + lay.blk);
  Stage<T> st;
  st.buf0 = (T *)(smem_raw + lay.buf0);
  st.buf1 = (T *)(smem_raw + lay.buf1);
  st.bar = (uint64_t *)(smem_raw + lay.bar);
  st.blk = blk;
  stage_init(st, &m.ms->err, 0);
  const int64_t base = p.env_ptr[io];
  st.L = (sizeof(T) == 8 ? (const T *)(const void *)p.L32 : (const T *)(const void *)p.L64) + base;
  for (int b = lane; b <= nblk; b += 32) blk[b] = p.blk_tab[b0 + b];
  if (lane == 0) {
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_mbar_init();
  }
  // global vectors are [row][16]; this warp's sources are kRW*part ..
  const int64_t g0 = io * kR + part * kRW;
  for (int e = lane; e < nI * kRW; e += 32) y[e] = from_d2<T>(rhs[g0 + (int64_t)(e / kRW) * kR + (e % kRW)]);
  __syncwarp();
  const int32_t *lo_g = p.env_lo + io;
  const int64_t *ptr_g = p.env_ptr + io;
  T *z = zstash + g0;

  // forward
  bool ok = true;
  int nlo, npr;
  stage_issue(st, 0, lane);
  stage_row_meta(lo_g, ptr_g, base, blk[0].x, blk[1].x, lane, nlo, npr);
  for (int b = 0; b < nblk; b++) {
    const int r0 = blk[b].x, nb = blk[b + 1].x - r0;
    meta[lane] = make_int2(nlo, npr);
    if (b + 1 < nblk) {
      stage_issue(st, b + 1, lane);
      stage_row_meta(lo_g, ptr_g, base, blk[b + 1].x, blk[b + 2].x, lane, nlo, npr);
    }
    if (!__all_sync(0xffffffffu, stage_wait(st, b))) {
      ok = false;
      break;
    }
    __syncwarp();
    const T *S = ((b & 1) ? st.buf1 : st.buf0) - stage_a0(st, b);
    // entries left of the block, every row of the block at once
    for (int t = h; t < nb; t += kQ) {
      const int2 mt = meta[t];
      const int len = max(0, r0 - mt.x);
      const T *__restrict__ row = S + mt.y;
      const T *__restrict__ yk = y + (int64_t)mt.x * kRW + r;
      T a0 = czero<T>(), a1 = czero<T>();
      int k = 0;
      for (; k + 1 < len; k += 2) {
        a0 = cmac(a0, row[k], yk[k * kRW]);
        a1 = cmac(a1, row[k + 1], yk[(k + 1) * kRW]);
      }
      if (k < len) a0 = cmac(a0, row[k], yk[k * kRW]);
      rect[t * kRW + r] = cadd(a0, a1);
    }
    __syncwarp();
    // the triangle, row by row over the block's columns
    for (int t = 0; t < nb; t++) {
      const int2 mt = meta[t];
      const int i = r0 + t;
      const int len = i - mt.x;
      const int k0 = max(0, r0 - mt.x);
      const T *__restrict__ row = S + mt.y;
      const T *__restrict__ yk = y + (int64_t)mt.x * kRW + r;
      T a0 = czero<T>(), a1 = czero<T>();
      int k = k0 + h;
      for (; k + kQ < len; k += 2 * kQ) {
        a0 = cmac(a0, row[k], yk[k * kRW]);
        a1 = cmac(a1, row[k + kQ], yk[(k + kQ) * kRW]);
      }
      if (k < len) a0 = cmac(a0, row[k], yk[k * kRW]);
      T acc = cadd(a0, a1);
#pragma unroll
      for (int o = kRW; o < 32; o <<= 1) acc = cadd(acc, shfl_xor(acc, o));
      const T val = csub(y[i * kRW + r], cadd(rect[t * kRW + r], acc));
      const T dinv = row[len];
      __syncwarp();
      if (h == 0) {
        y[i * kRW + r] = val;
        z[(int64_t)i * kR + r] = cmul(val, dinv);
      }
      __syncwarp();
    }
  }
  for (int e = lane; e < nI * kRW; e += 32) y[e] = z[(int64_t)(e / kRW) * kR + (e % kRW)];
  __syncwarp();

  // backward
  stage_row_meta(lo_g, ptr_g, base, blk[nblk - 1].x, blk[nblk].x, lane, nlo, npr);
  for (int b = nblk - 1; b >= 0 && ok; b--) {
    const int r0 = blk[b].x, nb = blk[b + 1].x - r0;
    meta[lane] = make_int2(nlo, npr);
    if (b >= 1) {
      if (b - 1 < nblk - 2) stage_issue(st, b - 1, lane);
      stage_row_meta(lo_g, ptr_g, base, blk[b - 1].x, blk[b].x, lane, nlo, npr);
    }
    if (!__all_sync(0xffffffffu, stage_wait(st, b))) {
      ok = false;
      break;
    }
    __syncwarp();
    const T *S = ((b & 1) ? st.buf1 : st.buf0) - stage_a0(st, b);
    // the triangle from the last row: the block's columns of each row
    for (int t = nb - 1; t >= 0; t--) {
      const int2 mt = meta[t];
      const int i = r0 + t;
      const int len = i - mt.x;
      const T xi = y[i * kRW + r];
      const T *__restrict__ row = S + mt.y;
      T *__restrict__ yc = y + (int64_t)mt.x * kRW + r;
      for (int k = max(0, r0 - mt.x) + h; k < len; k += kQ) yc[k * kRW] = cmsub(yc[k * kRW], row[k], xi);
      __syncwarp();
    }
    // the columns left of the block: column c belongs to group c % kQ, which
    // applies the block's rows from the last to the first
    for (int t = nb - 1; t >= 0; t--) {
      const int2 mt = meta[t];
      const int len = max(0, r0 - mt.x);
      const T xi = y[(r0 + t) * kRW + r];
      const T *__restrict__ row = S + mt.y;
      T *__restrict__ yc = y + (int64_t)mt.x * kRW + r;
      int k = (h - mt.x % kQ + kQ) % kQ;  // the first column of this group
      for (; k < len; k += kQ) yc[k * kRW] = cmsub(yc[k * kRW], row[k], xi);
    }
    __syncwarp();
  }
  // every copy issued into this CTA's shared memory has landed before it exits
  stage_drain(st);
  if (!ok) return;
  for (int e = lane; e < nI * kRW; e += 32) {
    const int64_t ge = g0 + (int64_t)(e / kRW) * kR + (e % kRW);
    double2 x = make_double2((double)y[e].x, (double)y[e].y);
    if (accumulate) x = cadd(xout[ge], x);
    xout[ge] = x;
  }
}

// ---- COCG, one set of scalars per source ------------------------------------

// per-source block reduction: thread (gi, r) = (threadIdx.x >> 4, & 15)
__device__ __forceinline__ double block_sum_r(double v, double *sh, bool is_max) {
  const int r = threadIdx.x & (kR - 1), gi = threadIdx.x >> 4;
  __syncthreads();
  sh[gi * (kR + 1) + r] = v;
  __syncthreads();
  double a = 0.0;
  if (gi == 0) {
    for (int j = 0; j < kMT / kR; j++) {
      const double x = sh[j * (kR + 1) + r];
      a = is_max ? fmax(a, x) : a + x;
    }
  }
  return a;  // valid in threads gi == 0
}

__device__ __forceinline__ void write_part(const MultiProblem &m, int f, double v) {
  if ((threadIdx.x >> 4) == 0)
    m.part[((int64_t)f * m.p.n_part_blocks + blockIdx.x) * kR + (threadIdx.x & (kR - 1))] = v;
}

// the last CTA: field f of source r over all blocks, blocks split over the 16
// thread groups and combined in group order (fixed order)
__device__ double reduce_part_r(const MultiProblem &m, int f, bool is_max, double *sh) {
  const int r = threadIdx.x & (kR - 1), gi = threadIdx.x >> 4;
  const int nb = m.p.n_part_blocks;
  double a = 0.0;
  for (int j = gi; j < nb; j += kMT / kR) {
    const double x = __ldcg(m.part + ((int64_t)f * nb + j) * kR + r);
    a = is_max ? fmax(a, x) : a + x;
  }
  const double t = block_sum_r(a, sh, is_max);
  __syncthreads();
  if (gi == 0) sh[kMT + r] = t;
  __syncthreads();
  const double v = sh[kMT + r];
  __syncthreads();
  return v;
}

__device__ __forceinline__ double2 gather_slots_r(const DevProblem &p, const double2 *v, int g, int r) {
  double2 q = cz();
  for (int t = p.gq_ptr[g]; t < p.gq_ptr[g + 1]; t++) q = cadd(q, v[p.gq_slot[t] * kR + r]);
  return q;
}

__global__ void multi_set_status_kernel(MultiScalars *ms, double eps, int32_t max_loop) {
  for (int r = 0; r < kR; r++) {
    ms->s[r].eps = eps;
    ms->s[r].max_loop = max_loop;
    ms->s[r].status = 0;
    ms->s[r].converged = 0;
    ms->s[r].nonfinite = 0;
  }
  ms->all_status = 0;
  for (int i = 0; i < 4; i++) ms->ticket[i] = 0;
}

// first step of every source (hddm_solver_s.h:158-256): Q, PC, r = q, z, p, max|r|, (r, z)
__global__ void multi_first_kernel(MultiProblem m, const double2 *__restrict__ pcloc) {
  __shared__ double sh[kMT + kR + 32];
  const DevProblem &p = m.p;
  const int r = threadIdx.x & (kR - 1), gi = threadIdx.x >> 4;
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  for (int g = blockIdx.x * (kMT / kR) + gi; g < p.nfree; g += gridDim.x * (kMT / kR)) {
    const double2 q = gather_slots_r(p, m.qloc, g, r);
    double2 pc = cz();
    for (int t = p.gq_ptr[g]; t < p.gq_ptr[g + 1]; t++) pc = cadd(pc, pcloc[p.gq_slot[t]]);
    pc = ciszero(pc) ? make_double2(1.0, 0.0) : cdiv_ref(make_double2(1.0, 0.0), pc);
    if (r == 0) m.PC[g] = pc;
    const int64_t e = (int64_t)g * kR + r;
    m.Q[e] = q;
    m.R[e] = q;
    const double2 z = cmul(q, pc);
    m.Z[e] = z;
    m.P[e] = z;
    m.U[e] = cz();
    mx = fmax(mx, cabs_ref(q));
    const double2 rz = cmul(q, z);
    rzr += rz.x;
    rzi += rz.y;
    l2 += q.x * q.x + q.y * q.y;
  }
  write_part(m, kMMax, block_sum_r(mx, sh, true));
  write_part(m, kMRzRe, block_sum_r(rzr, sh, false));
  write_part(m, kMRzIm, block_sum_r(rzi, sh, false));
  write_part(m, kML2, block_sum_r(l2, sh, false));
  if (!last_cta(&m.ms->ticket[0])) return;
  const double vmx = reduce_part_r(m, kMMax, true, sh);
  const double vrr = reduce_part_r(m, kMRzRe, false, sh);
  const double vri = reduce_part_r(m, kMRzIm, false, sh);
  const double vl2 = reduce_part_r(m, kML2, false, sh);
  if (gi == 0) {
    CocgScalars &c = m.ms->s[r];
    c.norm0 = vmx;
    c.l2_0 = sqrt(vl2);
    c.r0inv = vmx > 0.0 ? 1.0 / vmx : 0.0;
    c.rz = make_double2(vrr, vri);
    c.resi = 1.0;
    c.resi_l2 = 1.0;
    c.loop = 1;
    const bool bad = !isfinite(vmx) || !isfinite(vl2) || !isfinite(vrr) || !isfinite(vri);
    c.status = (bad || vmx < kNearlyZero) ? 1 : 0;
    c.converged = (!bad && vmx < kNearlyZero) ? 1 : 0;
    c.nonfinite = bad ? 1 : 0;
  }
  if (threadIdx.x == 0) m.ms->ticket[0] = 0;
}

// Q and (p, q); last CTA: -alpha per iterating source
__global__ void multi_pq_kernel(MultiProblem m) {
  if (m.ms->all_status != 0) return;
  __shared__ double sh[kMT + kR + 32];
  const DevProblem &p = m.p;
  const int r = threadIdx.x & (kR - 1), gi = threadIdx.x >> 4;
  double re = 0.0, im = 0.0;
  for (int g = blockIdx.x * (kMT / kR) + gi; g < p.nfree; g += gridDim.x * (kMT / kR)) {
    const int64_t e = (int64_t)g * kR + r;
    const double2 q = gather_slots_r(p, m.qloc, g, r);
    m.Q[e] = q;
    const double2 t = cmul(m.P[e], q);
    re += t.x;
    im += t.y;
  }
  write_part(m, kMPqRe, block_sum_r(re, sh, false));
  write_part(m, kMPqIm, block_sum_r(im, sh, false));
  if (!last_cta(&m.ms->ticket[1])) return;
  const double pr = reduce_part_r(m, kMPqRe, false, sh);
  const double pi = reduce_part_r(m, kMPqIm, false, sh);
  if (gi == 0) {
    CocgScalars &c = m.ms->s[r];
    if (c.status == 0) {
      const double2 pq = make_double2(pr, pi);
      c.malpha = (cabs_ref(c.rz) < kNearlyZero && cabs_ref(pq) < kNearlyZero) ? cz() : csub(cz(), cdiv_ref(c.rz, pq));
    }
  }
  if (threadIdx.x == 0) m.ms->ticket[1] = 0;
}

// u += -alpha p, r += -alpha q, z, max|r|, (r, z); last CTA: resi, beta, stopping
__global__ void multi_update_kernel(MultiProblem m) {
  if (m.ms->all_status != 0) return;
  __shared__ double sh[kMT + kR + 32];
  const DevProblem &p = m.p;
  const int r = threadIdx.x & (kR - 1), gi = threadIdx.x >> 4;
  const bool live = m.ms->s[r].status == 0;
  const double2 ma = m.ms->s[r].malpha;
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  if (live) {
    for (int g = blockIdx.x * (kMT / kR) + gi; g < p.nfree; g += gridDim.x * (kMT / kR)) {
      const int64_t e = (int64_t)g * kR + r;
      m.U[e] = cadd(m.U[e], cmul(ma, m.P[e]));
      const double2 rv = cadd(m.R[e], cmul(ma, m.Q[e]));
      m.R[e] = rv;
      mx = fmax(mx, cabs_ref(rv));
      const double2 z = cmul(rv, m.PC[g]);
      m.Z[e] = z;
      const double2 rz = cmul(rv, z);
      rzr += rz.x;
      rzi += rz.y;
      l2 += rv.x * rv.x + rv.y * rv.y;
    }
  }
  write_part(m, kMMax, block_sum_r(mx, sh, true));
  write_part(m, kMRzRe, block_sum_r(rzr, sh, false));
  write_part(m, kMRzIm, block_sum_r(rzi, sh, false));
  write_part(m, kML2, block_sum_r(l2, sh, false));
  if (!last_cta(&m.ms->ticket[2])) return;
  const double vmx = reduce_part_r(m, kMMax, true, sh);
  const double vrr = reduce_part_r(m, kMRzRe, false, sh);
  const double vri = reduce_part_r(m, kMRzIm, false, sh);
  const double vl2 = reduce_part_r(m, kML2, false, sh);
  if (gi == 0) {
    CocgScalars &c = m.ms->s[r];
    if (c.status == 0) {
      const double resi = vmx * c.r0inv;
      c.resi = resi;
      c.resi_l2 = c.l2_0 > 0.0 ? sqrt(vl2) / c.l2_0 : 0.0;
      const double2 rz = make_double2(vrr, vri);
      c.beta = (cabs_ref(rz) < kNearlyZero && cabs_ref(c.rz) < kNearlyZero) ? cz() : cdiv_ref(rz, c.rz);
      c.rz = rz;
      if (!isfinite(vl2) || !isfinite(vrr) || !isfinite(vri)) {
        c.status = 1;
        c.nonfinite = 1;
      } else if (resi < c.eps) {
        c.status = 1;
        c.converged = 1;
      } else if (c.loop >= c.max_loop) {
        c.status = 1;
      }
      c.loop += 1;
    }
  }
  if (threadIdx.x == 0) m.ms->ticket[2] = 0;
}

// p = z + beta p, or p = u for a source that just stopped; last CTA marks
// stopped sources finished and the batch finished when all are
__global__ void multi_pupdate_kernel(MultiProblem m) {
  if (m.ms->all_status != 0) return;
  const DevProblem &p = m.p;
  const int r = threadIdx.x & (kR - 1), gi = threadIdx.x >> 4;
  const int st = m.ms->s[r].status;
  const double2 be = m.ms->s[r].beta;
  if (st != 2) {
    for (int g = blockIdx.x * (kMT / kR) + gi; g < p.nfree; g += gridDim.x * (kMT / kR)) {
      const int64_t e = (int64_t)g * kR + r;
      m.P[e] = st == 1 ? m.U[e] : cadd(m.Z[e], cmul(be, m.P[e]));
    }
  }
  if (!last_cta(&m.ms->ticket[3])) return;
  if (threadIdx.x == 0) {
    int all = 2;
    for (int k = 0; k < kR; k++) {
      if (m.ms->s[k].status == 1) m.ms->s[k].status = 2;
      if (m.ms->s[k].status != 2) all = 0;
    }
    m.ms->all_status = all;
    m.ms->ticket[3] = 0;
  }
}

__global__ void multi_edge_solution_kernel(int64_t ne, int k, const int64_t *__restrict__ src,
                                           const double2 *__restrict__ Y, const double2 *__restrict__ V,
                                           double2 *__restrict__ x) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int64_t s = src[e];
  x[e] = s >= 0 ? Y[s * kR + k] : (s < -1 ? V[(-s - 2) * kR + k] : make_double2(0.0, 0.0));
}

unsigned grid_for(int64_t n, int threads) { return n > 0 ? (unsigned)((n + threads - 1) / threads) : 1u; }

}  // namespace

// sources per sweep warp: FP64 8 (its vectors are twice as large), FP32 16
constexpr int kRwFp64 = 8, kRwFp32 = 16;

size_t multi_smem_bytes(int max_interior, int max_blocks, int cap, bool fp32) {
  return multi_layout(max_interior, max_blocks, cap, fp32, fp32 ? kRwFp32 : kRwFp64).total;
}

int configure_multi(size_t smem, bool fp32) {
  return fp32 ? raise_smem_limit((const void *)multi_sweep_kernel<float2, kRwFp32>, kSlotMulti32, smem)
              : raise_smem_limit((const void *)multi_sweep_kernel<double2, kRwFp64>, kSlotMulti64, smem);
}

// The sweep, one launch per size bucket, each with the shared memory of its
// largest subdomain (a single bucket of every subdomain when none are set).
template <typename T, int kRW>
static void launch_multi_sweep(const MultiProblem &m, int mode, bool fp32, const double2 *rhs, double2 *xout,
                               T *zstash, int accumulate, cudaStream_t stream) {
  const DevProblem &p = m.p;
  const int nb = m.n_buckets > 0 ? m.n_buckets : 1;
  for (int k = 0; k < nb; k++) {
    const int first = m.n_buckets > 0 ? m.bucket_first[k] : 0;
    const int count = m.n_buckets > 0 ? m.bucket_count[k] : p.nsub;
    const int mi = m.n_buckets > 0 ? m.bucket_max_interior[k] : p.max_interior;
    const int mb = m.n_buckets > 0 ? m.bucket_max_blocks[k] : p.max_blocks;
    if (count <= 0) continue;
    const MultiLayout lay = multi_layout(mi, mb, p.stage_cap, fp32, kRW);
    multi_sweep_kernel<T, kRW><<<(unsigned)count * (kR / kRW), 32, lay.total, stream>>>(m, mode, rhs, xout, zstash,
                                                                                       accumulate, lay, first);
  }
}

void launch_multi_subsolve(const MultiProblem &m, int mode, bool fp32, cudaStream_t stream) {
  const DevProblem &p = m.p;
  const unsigned gi = grid_for(p.n_interior * kR, 256), gs = grid_for(p.n_slots * kR, 256);
  double2 *rhs = fp32 ? m.B : m.Y;
  multi_rhs_kernel<<<gi, 256, 0, stream>>>(m, mode, rhs);
  if (fp32) {
    float2 *zs = (float2 *)m.Zs;
    launch_multi_sweep<float2, kRwFp32>(m, mode, true, m.B, m.Y, zs, 0, stream);
    for (int k = 0; k < p.ir_steps; k++) {
      multi_residual_kernel<<<gi, 256, 0, stream>>>(m, mode);
      launch_multi_sweep<float2, kRwFp32>(m, mode, true, m.Rres, m.Y, zs, 1, stream);
    }
  } else {
    launch_multi_sweep<double2, kRwFp64>(m, mode, false, m.Y, m.Y, (double2 *)m.Zs, 0, stream);
  }
  multi_iface_kernel<<<gs, 256, 0, stream>>>(m, mode);
}

int multi_iteration_launches(bool fp32, int ir_steps, int n_buckets) {
  const int nb = n_buckets > 0 ? n_buckets : 1;
  return 2 + nb * (fp32 ? 1 + ir_steps : 1) + (fp32 ? ir_steps : 0) + 3;
}

void launch_multi_set_status(MultiScalars *ms, double eps, int32_t max_loop, cudaStream_t stream) {
  multi_set_status_kernel<<<1, 1, 0, stream>>>(ms, eps, max_loop);
}

void launch_multi_first(const MultiProblem &m, const double2 *pcloc, cudaStream_t stream) {
  multi_first_kernel<<<m.p.n_part_blocks, kMT, 0, stream>>>(m, pcloc);
}

void launch_multi_iteration(const MultiProblem &m, bool fp32, cudaStream_t stream) {
  launch_multi_subsolve(m, kModeIter, fp32, stream);
  multi_pq_kernel<<<m.p.n_part_blocks, kMT, 0, stream>>>(m);
  multi_update_kernel<<<m.p.n_part_blocks, kMT, 0, stream>>>(m);
  multi_pupdate_kernel<<<m.p.n_part_blocks, kMT, 0, stream>>>(m);
}

void launch_multi_edge_solution(const MultiProblem &m, int k, int64_t ne, const int64_t *edge_src, double2 *x,
                                cudaStream_t stream) {
  if (ne <= 0) return;
  multi_edge_solution_kernel<<<grid_for(ne, 256), 256, 0, stream>>>(ne, k, edge_src, m.Y, m.V, x);
}

}  // namespace fw
