// Device kernels of the HDDM hot path: value gather into the assembled
// lower rows, skyline profile, envelope scatter, batched LDL^T factor, the
// per-iteration subdomain solves and the interface COCG.
//
// Layout.  Subdomains are concatenated.  Each subdomain's non-Dirichlet
// ("interior") DOFs keep the reference's order and form a compressed
// envelope: interior row c stores columns env_lo[c]..c contiguously from
// env_ptr[c], the diagonal last.  The reference's envelope
// (advlas_skyline.c:12-25) also spans Dirichlet columns, whose factor entries
// are exactly zero (their rows are identity after SetBC,
// aij_matrix_func.h:83-104), so leaving them out changes no result and
// removes those bytes from every substitution pass.
//
// One warp works on one subdomain; warps take subdomains largest first.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "fw_device.cuh"
#include "fw_kernels.cuh"

namespace fw {

namespace {

using namespace dev;

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;

// 1/b by Smith's algorithm (R. L. Smith, CACM 5(8), 1962): the pivot
// reciprocal of the skyline factor, which the reference takes with C99
// complex division.
__device__ __forceinline__ double2 crecip_smith(double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x;
    const double den = b.x + b.y * r;
    return make_double2(1.0 / den, -r / den);
  }
  const double r = b.x / b.y;
  const double den = b.x * r + b.y;
  return make_double2(r / den, -1.0 / den);
}

// An interface iteration's refinement step is skipped once the COCG residual
// is below ir_relax: the accuracy an inexact Krylov product needs falls as the
// residual falls.  The first and last solves always refine.
__device__ __forceinline__ bool refine_skipped(const DevProblem &p, int mode) {
  return mode == kModeIter && p.ir_relax > 0.0 && p.sc->resi <= p.ir_relax;
}

__device__ __forceinline__ int warp_id_global() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }

// ----------------------------------------------------------------------------
// assembly

// aval[q] = sum of the element-matrix contributions of lower entry q in
// element order (aij_matrix_func.h:289-322 adds them in element order into a
// zero-initialised slot; zero contributions leave the sum unchanged).
__global__ void gather_values_kernel(int64_t nnz, const int64_t *__restrict__ cptr, const int64_t *__restrict__ contrib,
                                     const double2 *__restrict__ elmat, double2 *__restrict__ aval) {
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnz) return;
  double re = 0.0, im = 0.0;
  for (int64_t t = cptr[q]; t < cptr[q + 1]; t++) {
    const double2 v = elmat[contrib[t]];
    re = re + v.x;
    im = im + v.y;
  }
  aval[q] = make_double2(re, im);
}

// Skyline profile after Dirichlet elimination and DeleteZero: the first
// column of each sorted row (advlas_copy_nzindex_to_skyindex,
// advlas_skyline.c:12-25); Dirichlet rows keep only their unit diagonal
// (aij_matrix_func.h:98-103) and Dirichlet columns are zeroed and deleted
// (:107-135).
__global__ void profile_kernel(int32_t nsub, const int64_t *__restrict__ dof_off, const int64_t *__restrict__ nnz_off,
                               const int32_t *__restrict__ row_ptr_rel, const int32_t *__restrict__ col,
                               const double2 *__restrict__ aval, const uint8_t *__restrict__ isbc,
                               int32_t *__restrict__ idx1) {
  const int s = warp_id_global();
  if (s >= nsub) return;
  const int lane = threadIdx.x & 31;
  const int64_t d0 = dof_off[s];
  const int n = (int)(dof_off[s + 1] - d0);
  const int32_t *rp = row_ptr_rel + d0 + s;  // n+1 entries per subdomain
  const int64_t z0 = nnz_off[s];
  for (int r = lane; r < n; r += 32) {
    int first = r;
    if (!isbc[d0 + r]) {
      for (int q = rp[r]; q < rp[r + 1]; q++) {
        const int c = col[z0 + q];
        if (isbc[d0 + c]) continue;
        if (ciszero(aval[z0 + q])) continue;
        first = c;
        break;
      }
    }
    idx1[d0 + r] = first;
  }
}

__global__ void scatter_envelope_kernel(int64_t nnz, const int64_t *__restrict__ dst, const double2 *__restrict__ aval,
                                        double2 *__restrict__ L) {
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnz) return;
  const int64_t d = dst[q];
  if (d >= 0) L[d] = aval[q];
}

__global__ void gather_ops_kernel(int64_t n, const int64_t *__restrict__ src, const double2 *__restrict__ aval,
                                  double2 *__restrict__ dst) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  dst[t] = aval[src[t]];
}

// DIAG_MAKE (lib/hddm/hddm_pc.h:52-86) at the interface DOFs: the diagonal
// of the unmodified matrix, 1 where it is absent or zero.
__global__ void diag_pc_kernel(int64_t n, const int64_t *__restrict__ diag_src, const double2 *__restrict__ aval,
                               double2 *__restrict__ pcloc) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double2 v = make_double2(1.0, 0.0);
  const int64_t q = diag_src[t];
  if (q >= 0 && !ciszero(aval[q])) v = aval[q];
  pcloc[t] = v;
}

__global__ void to_fp32_kernel(int64_t n, const double2 *__restrict__ src, float2 *__restrict__ dst) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double2 v = src[t];
  dst[t] = make_float2((float)v.x, (float)v.y);
}

// ----------------------------------------------------------------------------
// LDL^T factor (advlas_skyline_ldl_decomposite, advlas_skyline.c:79-128),
// row-Crout without pivoting, in place: off-diagonals become L (unit lower),
// the diagonal becomes 1/d.  One warp per subdomain; the dot products of each
// (i, j) step are split across the lanes.
__global__ void factor_kernel(int32_t nsub, const int32_t *__restrict__ sub_order, const int64_t *__restrict__ int_off,
                              const int32_t *__restrict__ env_lo, const int64_t *__restrict__ env_ptr,
                              double2 *L, int32_t *status) {
  const int w = warp_id_global();
  if (w >= nsub) return;
  const int s = sub_order[w];
  const int lane = threadIdx.x & 31;
  const int64_t o = int_off[s];
  const int nI = (int)(int_off[s + 1] - o);
  const int32_t *lo = env_lo + o;
  const int64_t *ptr = env_ptr + o;
  bool bad = false;
  for (int i = 0; i < nI; i++) {
    const int lo_i = lo[i];
    double2 *Gi = L + ptr[i] - lo_i;  // Gi[k]: entry (i, k)
    for (int j = lo_i; j < i; j++) {
      const int lo_j = lo[j];
      const double2 *Lj = L + ptr[j] - lo_j;
      const int k0 = lo_i > lo_j ? lo_i : lo_j;
      double2 acc = cz();
      for (int k = k0 + lane; k < j; k += 32) acc = cadd(acc, cmul(Gi[k], Lj[k]));
      acc = warp_sum(acc);
      if (lane == 0) Gi[j] = csub(Gi[j], acc);
      __syncwarp();
    }
    double2 acc = cz();
    for (int k = lo_i + lane; k < i; k += 32) {
      const double2 g = Gi[k];
      const double2 dk = L[ptr[k] + (k - lo[k])];
      acc = cadd(acc, cmul(cmul(g, g), dk));
      Gi[k] = cmul(g, dk);
    }
    acc = warp_sum(acc);
    if (lane == 0) {
      const double2 d = csub(Gi[i], acc);
      const double2 r = crecip_smith(d);
      if (!(isfinite(r.x) && isfinite(r.y)) || ciszero(d)) bad = true;
      Gi[i] = r;
    }
    __syncwarp();
  }
  if (lane == 0 && bad) atomicMax(status, 1);
}

// ----------------------------------------------------------------------------
// Envelope substitutions (advlas_skyline_ldl_solve, advlas_skyline.c:134-167):
// forward row dot products with unit L, scaling by the stored 1/d, backward
// column updates with L^T.  In place on y.
template <typename T>
__device__ __forceinline__ void env_solve(int nI, const int32_t *__restrict__ lo, const int64_t *__restrict__ ptr,
                                          const T *__restrict__ L, T *y, int lane) {
  for (int i = 1; i < nI; i++) {
    const int lo_i = lo[i];
    const T *row = L + ptr[i] - lo_i;
    T acc = czero<T>();
    for (int k = lo_i + lane; k < i; k += 32) acc = cadd(acc, cmul(row[k], y[k]));
    acc = warp_sum(acc);
    if (lane == 0) y[i] = csub(y[i], acc);
    __syncwarp();
  }
  for (int i = lane; i < nI; i += 32) y[i] = cmul(y[i], L[ptr[i] + (i - lo[i])]);
  __syncwarp();
  for (int i = nI - 1; i >= 1; i--) {
    const int lo_i = lo[i];
    const T *row = L + ptr[i] - lo_i;
    const T xi = y[i];
    for (int k = lo_i + lane; k < i; k += 32) y[k] = csub(y[k], cmul(row[k], xi));
    __syncwarp();
  }
}

// One subdomain solve of the HDDM loop per warp:
//   first (solve_dom_1st_d, hddm_solver.h:461-555):  v = 0, b = f
//   iteration (solve_dom_d, :559-622):                v = P, b = 0
//   last (solve_dom_last_d, :626-693):                v = P, b = f
// Dirichlet elimination gives the interior right-hand side f_I - A_IG v
// (aij_matrix_func.h:60-136, the PEC values are zero); after the solve,
// q = A_G. x (- f_G when b = f) is the subdomain's contribution to Q at its
// interface DOFs (MxV_TMP_AIJ, aij_matrix_func.h:624-658, restricted to the
// interface rows that COM_RES_SP_FUNC reads, hddm_solver_sp.h:41-54).
template <bool kFp32>
__global__ void __launch_bounds__(kThreads) subsolve_kernel(DevProblem p, int mode) {
  if (p.sc->status != 0 && mode == kModeIter) return;
  const int w = warp_id_global();
  if (w >= p.nsub) return;
  const int s = p.sub_order[w];
  const int lane = threadIdx.x & 31;
  const int64_t io = p.int_off[s], go = p.if_off[s];
  const int nI = (int)(p.int_off[s + 1] - io);
  const int nG = (int)(p.if_off[s + 1] - go);
  const bool with_bc = mode != kModeFirst;
  const bool with_f = mode != kModeIter;
  double2 *y = p.Y + io;
  double2 *v = p.V + go;
  for (int k = lane; k < nG; k += 32) v[k] = with_bc ? p.P[p.if_ln[go + k]] : cz();
  __syncwarp();
  const int32_t *cptr = p.cpl_ptr + io + s;
  const int64_t cbase = p.cpl_off[s];
  double2 *b = kFp32 ? p.B + io : y;
  for (int c = lane; c < nI; c += 32) {
    double2 acc = with_f ? p.fI[io + c] : cz();
    for (int q = cptr[c]; q < cptr[c + 1]; q++) acc = csub(acc, cmul(p.cpl_val[cbase + q], v[p.cpl_col[cbase + q]]));
    b[c] = acc;
  }
  __syncwarp();
  const int32_t *lo = p.env_lo + io;
  const int64_t *ptr = p.env_ptr + io;
  if (!kFp32) {
    env_solve<double2>(nI, lo, ptr, p.L64, y, lane);
  } else {
    // FP32 factor with FP64 iterative refinement: x0 = solve32(b);
    // repeat r = b - A_II x (FP64), x += solve32(r).
    float2 *y32 = p.Y32 + io;
    for (int c = lane; c < nI; c += 32) y32[c] = make_float2((float)b[c].x, (float)b[c].y);
    __syncwarp();
    env_solve<float2>(nI, lo, ptr, p.L32, y32, lane);
    for (int c = lane; c < nI; c += 32) y[c] = make_double2((double)y32[c].x, (double)y32[c].y);
    __syncwarp();
    const int32_t *aptr = p.aii_ptr + io + s;
    const int64_t abase = p.aii_off[s];
    double bnorm = 0.0;
    if (p.ir_tol > 0.0) {
      for (int c = lane; c < nI; c += 32) bnorm = fmax(bnorm, fabs(b[c].x) + fabs(b[c].y));
      for (int o2 = 16; o2 > 0; o2 >>= 1) bnorm = fmax(bnorm, __shfl_xor_sync(0xffffffffu, bnorm, o2));
    }
    const int ir_steps = refine_skipped(p, mode) ? 0 : p.ir_steps;
    for (int step = 0; step < ir_steps; step++) {
      double rnorm = 0.0;
      for (int c = lane; c < nI; c += 32) {
        double2 r = b[c];
        for (int q = aptr[c]; q < aptr[c + 1]; q++) r = csub(r, cmul(p.aii_val[abase + q], y[p.aii_col[abase + q]]));
        y32[c] = make_float2((float)r.x, (float)r.y);
        rnorm = fmax(rnorm, fabs(r.x) + fabs(r.y));
      }
      if (p.ir_tol > 0.0) {
        for (int o2 = 16; o2 > 0; o2 >>= 1) rnorm = fmax(rnorm, __shfl_xor_sync(0xffffffffu, rnorm, o2));
        if (rnorm <= p.ir_tol * bnorm) break;
      }
      __syncwarp();
      env_solve<float2>(nI, lo, ptr, p.L32, y32, lane);
      for (int c = lane; c < nI; c += 32)
        y[c] = cadd(y[c], make_double2((double)y32[c].x, (double)y32[c].y));
      __syncwarp();
    }
  }
  __syncwarp();
  const int32_t *rptr = p.ifr_ptr + go + s;
  const int64_t rbase = p.ifr_off[s];
  for (int k = lane; k < nG; k += 32) {
    double2 acc = cz();
    for (int q = rptr[k]; q < rptr[k + 1]; q++) {
      const int c = p.ifr_col[rbase + q];
      const double2 xv = c >= 0 ? y[c] : v[-c - 1];
      acc = cadd(acc, cmul(p.ifr_val[rbase + q], xv));
    }
    if (with_f) acc = csub(acc, p.fG[go + k]);
    p.qloc[go + k] = acc;
  }
}

// ----------------------------------------------------------------------------
// Block-row envelope substitutions, one CTA per subdomain.
//
// Rows are taken in blocks of 32.  Forward: the rectangle left of the block
// (columns < r0) is a set of independent dot products, spread over all warps;
// the 32x32 triangle inside the block is then resolved by one warp with
// shuffles from a padded shared-memory tile (row stride 33 keeps both the
// column-wise forward reads and the row-wise backward reads free of bank
// conflicts).  Backward: the block's triangle first, then the transposed
// rectangle update of the columns left of the block, spread over all threads.
// The interior vector, the interface values and the row metadata of the
// subdomain stay in shared memory; the factor streams from global memory.
constexpr int kRB = 32;       // rows per block
constexpr int kTriStride = 33;
constexpr int kCtaThreads = 256;

struct CtaMeta {
  const int32_t *lo;   // shared: first stored column of each interior row
  const int32_t *pr;   // shared: row start (column lo) relative to the subdomain base
  const int32_t *bmin; // shared: smallest lo of each row block
  int nI;
};

// rows of a block handled by one warp (rows w, w+nw, ...); kRowsPerWarp
// independent accumulators keep several loads in flight per lane
constexpr int kRowsPerWarp = kRB / (kCtaThreads / 32);

template <typename T>
__device__ void cta_forward(const CtaMeta &m, const T *__restrict__ L, T *y, T *tri, T *rect) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  for (int r0 = 0; r0 < m.nI; r0 += kRB) {
    const int nb = min(kRB, m.nI - r0);
    int lo_u[kRowsPerWarp], len_u[kRowsPerWarp];
    const T *row_u[kRowsPerWarp];
    int maxlen = 0;
#pragma unroll
    for (int u = 0; u < kRowsPerWarp; u++) {
      const int t = warp + u * nw;
      const int i = r0 + t;
      if (t < nb) {
        lo_u[u] = m.lo[i];
        row_u[u] = L + m.pr[i] - lo_u[u];
        len_u[u] = max(0, r0 - lo_u[u]);
      } else {
        lo_u[u] = 0;
        row_u[u] = L;
        len_u[u] = 0;
      }
      maxlen = max(maxlen, len_u[u]);
    }
    T acc[kRowsPerWarp];
#pragma unroll
    for (int u = 0; u < kRowsPerWarp; u++) acc[u] = czero<T>();
    for (int k = lane; k < maxlen; k += 32) {
#pragma unroll
      for (int u = 0; u < kRowsPerWarp; u++) {
        if (k < len_u[u]) {
          const int col = lo_u[u] + k;
          acc[u] = cadd(acc[u], cmul(row_u[u][col], y[col]));
        }
      }
    }
    // stage the block's triangle: tri[t][j] = L[r0+t][r0+j]
#pragma unroll
    for (int u = 0; u < kRowsPerWarp; u++) {
      const int t = warp + u * nw;
      if (t < nb) {
        const int col = r0 + lane;
        tri[t * kTriStride + lane] = (col < r0 + t && col >= lo_u[u]) ? row_u[u][col] : czero<T>();
      }
    }
#pragma unroll
    for (int u = 0; u < kRowsPerWarp; u++) {
      const T a = warp_sum(acc[u]);
      const int t = warp + u * nw;
      if (lane == 0 && t < nb) rect[t] = a;
    }
    __syncthreads();
    if (warp == 0) {
      T val = lane < nb ? csub(y[r0 + lane], rect[lane]) : czero<T>();
      for (int j = 0; j < nb - 1; j++) {
        const T yj = shfl_idx(val, j);
        if (lane > j) val = csub(val, cmul(tri[lane * kTriStride + j], yj));
      }
      if (lane < nb) y[r0 + lane] = val;
    }
    __syncthreads();
  }
}

template <typename T>
__device__ void cta_diag(const CtaMeta &m, const T *__restrict__ L, T *y) {
  for (int i = threadIdx.x; i < m.nI; i += blockDim.x) y[i] = cmul(y[i], L[m.pr[i] + (i - m.lo[i])]);
  __syncthreads();
}

template <typename T>
__device__ void cta_backward(const CtaMeta &m, const T *__restrict__ L, T *y, T *tri) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  const int nblk = (m.nI + kRB - 1) / kRB;
  for (int blk = nblk - 1; blk >= 0; blk--) {
    const int r0 = blk * kRB;
    const int nb = min(kRB, m.nI - r0);
#pragma unroll
    for (int u = 0; u < kRowsPerWarp; u++) {
      const int t = warp + u * nw;
      if (t < nb) {
        const int i = r0 + t;
        const int lo_i = m.lo[i];
        const T *row = L + m.pr[i] - lo_i;
        const int col = r0 + lane;
        tri[t * kTriStride + lane] = (col < i && col >= lo_i) ? row[col] : czero<T>();
      }
    }
    __syncthreads();
    if (warp == 0) {
      T val = lane < nb ? y[r0 + lane] : czero<T>();
      for (int i = nb - 1; i >= 1; i--) {
        const T xi = shfl_idx(val, i);
        if (lane < i) val = csub(val, cmul(tri[i * kTriStride + lane], xi));
      }
      if (lane < nb) y[r0 + lane] = val;
    }
    __syncthreads();
    // columns left of the block: y_k -= sum_i L_ik x_i, loads issued
    // unconditionally (clamped index, zero weight outside the row)
    const int kmin = m.bmin[blk];
    for (int k = kmin + tid; k < r0; k += blockDim.x) {
      T acc = czero<T>();
#pragma unroll 8
      for (int t = 0; t < nb; t++) {
        const int i = r0 + t;
        const int d = k - m.lo[i];
        const T lv = L[m.pr[i] + max(d, 0)];
        if (d >= 0) acc = cadd(acc, cmul(lv, y[i]));
      }
      y[k] = csub(y[k], acc);
    }
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ void cta_solve(const CtaMeta &m, const T *__restrict__ L, T *y, T *tri, T *rect) {
  cta_forward<T>(m, L, y, tri, rect);
  cta_diag<T>(m, L, y);
  cta_backward<T>(m, L, y, tri);
}

// Shared-memory bytes of one subdomain CTA.
__host__ __device__ inline size_t cta_smem_bytes(int nI, int nG, bool fp32) {
  const int nblk = (nI + kRB - 1) / kRB;
  size_t b = 0;
  b += (size_t)nI * 8 + (size_t)nblk * 4;        // lo, pr, bmin
  b = (b + 15) & ~(size_t)15;
  b += (size_t)nG * 16;                           // v
  if (fp32) {
    b += (size_t)nI * 32;                         // x, b (FP64)
    b += (size_t)nI * 8;                          // y (FP32)
    b += (size_t)kRB * kTriStride * 8 + kRB * 8;  // tri, rect
  } else {
    b += (size_t)nI * 16;                         // y
    b += (size_t)kRB * kTriStride * 16 + kRB * 16;
  }
  return b + 64;
}

template <bool kFp32>
__global__ void __launch_bounds__(kCtaThreads) subsolve_cta_kernel(DevProblem p, int mode) {
  using LT = typename std::conditional<kFp32, float2, double2>::type;
  if (mode == kModeIter && p.sc->status != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = p.sub_order[blockIdx.x];
  const int64_t io = p.int_off[s], go = p.if_off[s];
  const int nI = (int)(p.int_off[s + 1] - io);
  const int nG = (int)(p.if_off[s + 1] - go);
  const int nblk = (nI + kRB - 1) / kRB;
  const int tid = threadIdx.x;
  // shared layout
  int32_t *lo = (int32_t *)smem_raw;
  int32_t *pr = lo + nI;
  int32_t *bmin = pr + nI;
  size_t off = ((size_t)nI * 8 + (size_t)nblk * 4 + 15) & ~(size_t)15;
  double2 *v = (double2 *)(smem_raw + off);
  off += (size_t)nG * 16;
  double2 *xd = nullptr, *bd = nullptr;
  if (kFp32) {
    xd = (double2 *)(smem_raw + off);
    off += (size_t)nI * 16;
    bd = (double2 *)(smem_raw + off);
    off += (size_t)nI * 16;
  }
  LT *y = (LT *)(smem_raw + off);
  off += (size_t)nI * sizeof(LT);
  LT *tri = (LT *)(smem_raw + off);
  off += (size_t)kRB * kTriStride * sizeof(LT);
  LT *rect = (LT *)(smem_raw + off);

  const int64_t base = nI > 0 ? p.env_ptr[io] : 0;
  for (int i = tid; i < nI; i += blockDim.x) {
    lo[i] = p.env_lo[io + i];
    pr[i] = (int32_t)(p.env_ptr[io + i] - base);
  }
  const bool with_bc = mode != kModeFirst;
  const bool with_f = mode != kModeIter;
  for (int k = tid; k < nG; k += blockDim.x) v[k] = with_bc ? p.P[p.if_ln[go + k]] : cz();
  __syncthreads();
  for (int b = tid; b < nblk; b += blockDim.x) {
    int mn = b * kRB;
    const int e = min(nI, (b + 1) * kRB);
    for (int i = b * kRB; i < e; i++) mn = min(mn, lo[i]);
    bmin[b] = mn;
  }
  // Dirichlet elimination: interior right-hand side f_I - A_IG v
  const int32_t *cptr = p.cpl_ptr + io + s;
  const int64_t cbase = p.cpl_off[s];
  for (int c = tid; c < nI; c += blockDim.x) {
    double2 acc = with_f ? p.fI[io + c] : cz();
    for (int q = cptr[c]; q < cptr[c + 1]; q++) acc = csub(acc, cmul(p.cpl_val[cbase + q], v[p.cpl_col[cbase + q]]));
    if (kFp32) bd[c] = acc;
    y[c] = from_d2<LT>(acc);
  }
  __syncthreads();
  CtaMeta m{lo, pr, bmin, nI};
  if (!kFp32) {
    cta_solve<LT>(m, (const LT *)p.L64 + base, y, tri, rect);
  } else {
    const LT *L = (const LT *)p.L32 + base;
    cta_solve<LT>(m, L, y, tri, rect);
    for (int c = tid; c < nI; c += blockDim.x) xd[c] = make_double2((double)y[c].x, (double)y[c].y);
    __syncthreads();
    const int32_t *aptr = p.aii_ptr + io + s;
    const int64_t abase = p.aii_off[s];
    __shared__ double red[kCtaThreads / 32];
    __shared__ int stop;
    const int ir_steps = refine_skipped(p, mode) ? 0 : p.ir_steps;
    for (int step = 0; step < ir_steps; step++) {
      // FP64 residual of the subdomain system, rounded into the FP32 work vector
      double rn = 0.0;
      for (int c = tid; c < nI; c += blockDim.x) {
        double2 r = bd[c];
        for (int q = aptr[c]; q < aptr[c + 1]; q++) r = csub(r, cmul(p.aii_val[abase + q], xd[p.aii_col[abase + q]]));
        y[c] = from_d2<LT>(r);
        rn = fmax(rn, fabs(r.x) + fabs(r.y));
      }
      if (p.ir_tol > 0.0) {
        double bn = 0.0;
        for (int c = tid; c < nI; c += blockDim.x) bn = fmax(bn, fabs(bd[c].x) + fabs(bd[c].y));
        for (int o2 = 16; o2 > 0; o2 >>= 1) {
          rn = fmax(rn, __shfl_xor_sync(0xffffffffu, rn, o2));
          bn = fmax(bn, __shfl_xor_sync(0xffffffffu, bn, o2));
        }
        if ((tid & 31) == 0) red[tid >> 5] = rn <= p.ir_tol * bn ? 1.0 : 0.0;
        __syncthreads();
        if (tid == 0) {
          int all = 1;
          for (int w = 0; w < (int)(blockDim.x >> 5); w++) all &= red[w] > 0.5;
          stop = all;
        }
        __syncthreads();
        if (stop) break;
      }
      __syncthreads();
      cta_solve<LT>(m, L, y, tri, rect);
      for (int c = tid; c < nI; c += blockDim.x)
        xd[c] = cadd(xd[c], make_double2((double)y[c].x, (double)y[c].y));
      __syncthreads();
    }
  }
  // q = A_G. x (- f_G)
  const int32_t *rptr = p.ifr_ptr + go + s;
  const int64_t rbase = p.ifr_off[s];
  double2 *yout = p.Y + io;
  for (int k = tid; k < nG; k += blockDim.x) {
    double2 acc = cz();
    for (int q = rptr[k]; q < rptr[k + 1]; q++) {
      const int c = p.ifr_col[rbase + q];
      double2 xv;
      if (c >= 0) {
        if (kFp32)
          xv = xd[c];
        else
          xv = make_double2((double)y[c].x, (double)y[c].y);
      } else {
        xv = v[-c - 1];
      }
      acc = cadd(acc, cmul(p.ifr_val[rbase + q], xv));
    }
    if (with_f) acc = csub(acc, p.fG[go + k]);
    p.qloc[go + k] = acc;
  }
  if (mode == kModeLast) {
    for (int c = tid; c < nI; c += blockDim.x)
      yout[c] = kFp32 ? xd[c] : make_double2((double)y[c].x, (double)y[c].y);
    for (int k = tid; k < nG; k += blockDim.x) p.V[go + k] = v[k];
  }
}

// ----------------------------------------------------------------------------
// Staged subdomain solve: one warp per subdomain, row blocks brought into
// shared memory by TMA bulk copies.
//
// The iteration's subdomain work is split in three launches:
//   rhs_kernel           f_I - A_IG v for every interior row of every
//                        subdomain (SetBC, aij_matrix_func.h:60-136),
//   subsolve_staged_kernel  the envelope substitutions, one warp per subdomain,
//   iface_product_kernel q = A_G.[x; v] (- f_G) for every interface slot.
// The two products are grid-wide sparse products: every row of every
// subdomain in parallel, a few lanes per row, coalesced.  The substitution
// warp therefore only streams its factor.
//
// A subdomain's rows are cut on the host into blocks of at most 32 rows whose
// stored entries fit one staging buffer (blk_tab).  The block's entries are
// contiguous in the envelope, so one cp.async.bulk copies the whole block
// into shared memory, completing on an mbarrier; the copy of block b+1 is in
// flight while block b is computed (two buffers per warp).  The backward sweep
// starts on the two blocks the forward sweep left in the buffers.
//   forward  - entries left of the block: eight lanes per row (conflict-free
//              shared loads of the entry and of y[col]), four rows per step;
//              then the triangle, one lane per row, one broadcast shuffle per
//              row; the pivot scaling z = y/d is written to the z stash for
//              the backward sweep.
//   backward - the triangle with lanes over columns, then the transposed
//              update of the columns left of the block (lanes over columns,
//              the block's rows from the last in the inner loop, in place).
// Several subdomains share an SM and hide each other's dependent chains.
// With FWGPU_SOLVE_BLOCKINV the factor has a second layout in which each
// block's triangle is stored as N = (I + L_bb)^-1 - I, and the triangles are
// products with N (four independent sums per lane) instead of substitutions.
// The arithmetic is the reference's row-oriented envelope substitution
// (advlas_skyline.c:134-167) with the forward sums regrouped; the grouping
// depends on the rows' entries and the block boundaries only, so one, two or
// four warps per subdomain give the same bits.  The copies of the forward sweep
// keep their lines in L2 (evict_last) for the backward sweep, whose copies
// are the lines' last use (evict_first).  Every mbarrier wait is bounded: on
// a timeout the CTA raises the error word, issues no further copy, waits for
// the copies in flight and returns (the host reports the solve as failed).
constexpr int kSB = 32;        // rows per block at most, one per lane

struct StageLayout {
  size_t y, buf0, buf1, xb, rb, meta, gmin, bar, blk, total;
};

// Shared-memory slice of one subdomain warp of the staged solve.
__host__ __device__ inline StageLayout stage_layout(int max_interior, int max_blocks, int cap, bool fp32) {
  const size_t es = fp32 ? 8 : 16;
  StageLayout l;
  size_t o = 0;
  l.y = o;
  o += a16((size_t)max_interior * es);
  l.buf0 = o;
  o += a16((size_t)cap * es);
  l.buf1 = o;
  o += a16((size_t)cap * es);
  l.xb = o;
  o += a16(kSB * es);
  l.rb = o;
  o += a16(2 * kSB * es);
  l.meta = o;
  o += kSB * 8;
  l.gmin = o;
  o += 16;
  l.bar = o;
  o += 32;
  l.blk = o;
  o += a16(((size_t)max_blocks + 1) * 8);
  l.total = o;
  return l;
}

// Forward sweep over the row blocks.  Per block of nb <= 32 rows starting at
// row r0:
//   - the entries left of the block: eight lanes per row, four rows per
//     warp step (row groups of four shared out over the warps); lane j of a
//     row sums the row's entries j, j+8, j+16, ... in order into one
//     accumulator, and three shuffles add the eight lanes.  The sum of a row
//     therefore depends on its entries alone, not on the staging capacity or
//     the number of warps;
//   - the block's triangle: lane t holds row r0 + t, one broadcast shuffle per
//     row, the operands of 4 steps loaded ahead;
//   - the pivot scaling z = y/d goes to the z stash for the backward sweep.
// Returns false when a staged copy did not arrive (error word raised); the
// caller drains the copies in flight and stops.
template <typename T, bool kInv>
__device__ bool staged_forward(Stage<T> &st, int nblk, const int32_t *lo_g, const int64_t *ptr_g, int64_t base,
                               T *y, int2 *meta, T *zstash, T *rectb, int tid, int nw) {
  const int lane = tid & 31, w = tid >> 5;
  const int q = lane >> 3, j = lane & 7;
  int nlo, npr;
  stage_issue(st, 0, tid);
  stage_row_meta(lo_g, ptr_g, base, st.blk[0].x, st.blk[1].x, lane, nlo, npr);
  for (int b = 0; b < nblk; b++) {
    const int r0 = st.blk[b].x, nb = st.blk[b + 1].x - r0;
    const int my_lo = nlo, my_pr = npr;
    if (w == 0) meta[lane] = make_int2(nlo, npr);
    if (b + 1 < nblk) {
      stage_issue(st, b + 1, tid);
      stage_row_meta(lo_g, ptr_g, base, st.blk[b + 1].x, st.blk[b + 2].x, lane, nlo, npr);
    }
    const bool late = !stage_wait(st, b);
    if (__syncthreads_or(late)) return false;
    const T *S = ((b & 1) ? st.buf1 : st.buf0) - stage_a0(st, b);  // S[e]: entry e of the envelope
    for (int g = w; 4 * g < nb; g += nw) {
      const int t = 4 * g + q;
      const int2 mt = t < nb ? meta[t] : make_int2(r0, 0);
      const int len = t < nb ? max(0, r0 - mt.x) : 0;
      int longest = max(len, __shfl_xor_sync(0xffffffffu, len, 8));
      longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, 16));
      const T *row = S + mt.y;  // the row's entries from its first column
      const T *yr = y + mt.x;
      T acc = czero<T>();
      for (int k = j; k < longest; k += 16) {
        const bool i0 = k < len, i1 = k + 8 < len;
        const T a0 = i0 ? row[k] : czero<T>(), b0 = i0 ? yr[k] : czero<T>();
        const T a1 = i1 ? row[k + 8] : czero<T>(), b1 = i1 ? yr[k + 8] : czero<T>();
        acc = cmac(acc, a0, b0);
        acc = cmac(acc, a1, b1);
      }
      acc = cadd(acc, shfl_xor(acc, 4));
      acc = cadd(acc, shfl_xor(acc, 2));
      acc = cadd(acc, shfl_xor(acc, 1));
      if (j == 0 && t < nb) rectb[t] = acc;
    }
    __syncthreads();
    if (kInv && w == 0) {
      // y_b = (I + N) v with v = y_b - (the sums left of the block): lane t
      // sums N_tj v_j over j in four chunks of 8 columns, one accumulator
      // per chunk, in ascending j; no chain from row to row
      const int2 ml = meta[nb - 1];
      const T *N = S + ml.y + max(0, r0 - ml.x);  // after the block's left parts
      const T *Nr = N + ((lane * (lane - 1)) >> 1);
      T *vb = rectb + kSB;
      const T v = lane < nb ? csub(y[r0 + lane], rectb[lane]) : czero<T>();
      vb[lane] = v;
      __syncwarp();
      T acc[4] = {czero<T>(), czero<T>(), czero<T>(), czero<T>()};
#pragma unroll
      for (int jj = 0; jj < 8; jj++) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int j = 8 * c + jj;  // straight-line code: the loads go ahead of the sums
          const T a = (j < lane && lane < nb) ? Nr[j] : czero<T>();
          acc[c] = cmac(acc[c], a, vb[j]);
        }
      }
      const T val = cadd(v, cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3])));
      if (lane < nb) {
        y[r0 + lane] = val;
        zstash[r0 + lane] = cmul(val, N[((nb * (nb - 1)) >> 1) + lane]);  // the pivots' 1/d after N
      }
    } else if (w == 0) {
      const T rect = rectb[lane];
      T val = lane < nb ? csub(y[r0 + lane], rect) : czero<T>();
      const T *mine = S + my_pr - my_lo;  // mine[col]: this lane's row at column col
      for (int j0 = 0; j0 < nb - 1; j0 += 4) {
        T op[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int jj = j0 + u;
          op[u] = (lane > jj && r0 + jj >= my_lo) ? mine[r0 + jj] : czero<T>();
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const T yj = shfl_idx(val, min(j0 + u, 31));
          val = cmsub(val, op[u], yj);
        }
      }
      if (lane < nb) {
        y[r0 + lane] = val;
        zstash[r0 + lane] = cmul(val, mine[r0 + lane]);  // 1/d on the diagonal
      }
    }
    __syncthreads();
  }
  return true;
}

// Backward sweep, blocks from the last.  Per block: the triangle with lanes
// over the block's columns (warp 0), then the columns left of the block in
// 32-column chunks shared out over the warps: the lane of column c applies
// y_c -= L_tc x_t for the block's rows t from the last to the first, in
// place, as the reference does (advlas_skyline.c:157-165); a group of eight
// rows none of which reaches the chunk is skipped.
template <typename T, bool kInv>
__device__ bool staged_backward(Stage<T> &st, int nblk, const int32_t *lo_g, const int64_t *ptr_g, int64_t base,
                                T *y, T *xb, int2 *meta, int *gmin, int tid, int nw) {
  const int lane = tid & 31, w = tid >> 5;
  int nlo, npr;
  stage_row_meta(lo_g, ptr_g, base, st.blk[nblk - 1].x, st.blk[nblk].x, lane, nlo, npr);
  for (int b = nblk - 1; b >= 0; b--) {
    const int r0 = st.blk[b].x, nb = st.blk[b + 1].x - r0;
    const int my_lo = nlo;
    if (w == 0) {
      meta[lane] = make_int2(nlo, npr);
      int m = lane < nb ? nlo : INT_MAX;
      m = min(m, __shfl_xor_sync(0xffffffffu, m, 1));
      m = min(m, __shfl_xor_sync(0xffffffffu, m, 2));
      m = min(m, __shfl_xor_sync(0xffffffffu, m, 4));
      if ((lane & 7) == 0) gmin[lane >> 3] = m;
    }
    // the forward sweep left blocks nblk-1 and nblk-2 in the buffers
    if (b >= 1) {
      if (b - 1 < nblk - 2) stage_issue(st, b - 1, tid);
      stage_row_meta(lo_g, ptr_g, base, st.blk[b - 1].x, st.blk[b].x, lane, nlo, npr);
    }
    const bool late = !stage_wait(st, b);
    if (__syncthreads_or(late)) return false;
    const T *S = ((b & 1) ? st.buf1 : st.buf0) - stage_a0(st, b);
    if (kInv && w == 0) {
      // x_b = (I + N)^T w with w = y_b: lane j sums N_tj w_t over t in four
      // chunks of 8 rows, one accumulator per chunk, in ascending t
      const int2 ml = meta[nb - 1];
      const T *N = S + ml.y + max(0, r0 - ml.x);
      const T wv = lane < nb ? y[r0 + lane] : czero<T>();
      T acc[4] = {czero<T>(), czero<T>(), czero<T>(), czero<T>()};
#pragma unroll
      for (int tt = 0; tt < 8; tt++) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int t = 8 * c + tt;
          const T a = (lane < t && t < nb) ? N[((t * (t - 1)) >> 1) + lane] : czero<T>();
          acc[c] = cmac(acc[c], a, y[r0 + min(t, nb - 1)]);
        }
      }
      const T val = cadd(wv, cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3])));
      __syncwarp();  // every lane has read y_b before it is overwritten
      if (lane < nb) {
        y[r0 + lane] = val;
        xb[lane] = val;
      }
    } else if (w == 0) {
      // triangle, lanes over the block's columns; operands of 4 steps loaded ahead
      T val = lane < nb ? y[r0 + lane] : czero<T>();
      const int col = r0 + lane;
      for (int i0 = nb - 1; i0 >= 1; i0 -= 4) {
        T op[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int i = i0 - u;
          const int2 mt = meta[max(i, 0)];
          op[u] = (i >= 1 && lane < i && col >= mt.x) ? S[mt.y + col - mt.x] : czero<T>();
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const T xi = shfl_idx(val, max(i0 - u, 0));
          val = cmsub(val, op[u], xi);
        }
      }
      if (lane < nb) {
        y[r0 + lane] = val;
        xb[lane] = val;
      }
    }
    int bmin = lane < nb ? my_lo : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bmin = min(bmin, __shfl_xor_sync(0xffffffffu, bmin, o));
    __syncthreads();
    for (int cb = bmin + 32 * w; cb < r0; cb += 32 * nw) {
      const int c = cb + lane;
      const bool act = c < r0;
      T yc = act ? y[c] : czero<T>();
      for (int t0 = (nb - 1) & ~7; t0 >= 0; t0 -= 8) {
        if (gmin[t0 >> 3] >= cb + 32) continue;  // no row of the group reaches this chunk
        T v[8], xv[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int t = t0 + 7 - u;
          const int2 mt = meta[t];
          const int d = c - mt.x;
          v[u] = (t < nb && act && d >= 0) ? S[mt.y + d] : czero<T>();
          xv[u] = t < nb ? xb[t] : czero<T>();  // xb past the block may hold anything
        }
#pragma unroll
        for (int u = 0; u < 8; u++) yc = cmsub(yc, v[u], xv[u]);
      }
      if (act) y[c] = yc;
    }
    __syncthreads();
  }
  return true;
}

template <typename T, bool kInv>
__global__ void __launch_bounds__(128) subsolve_staged_kernel(DevProblem p, int mode, const double2 *rhs, double2 *xout,
                                                             T *zstash, int accumulate, StageLayout lay) {
  if (mode == kModeIter && p.sc->status != 0) return;
  if (accumulate && refine_skipped(p, mode)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4][2];
  const int tid = threadIdx.x, nt = blockDim.x, nw = nt >> 5;
  const int s = p.sub_order[blockIdx.x];
  const int64_t io = p.int_off[s];
  const int nI = (int)(p.int_off[s + 1] - io);
  const int32_t *blk_off = kInv ? p.inv_blk_off : p.blk_off;
  const int b0 = blk_off[s];
  const int nblk = blk_off[s + 1] - b0 - 1;
  if (nI == 0 || nblk <= 0) return;
  T *y = (T *)(smem_raw + lay.y);
  T *xb = (T *)(smem_raw + lay.xb);
  T *rectb = (T *)(smem_raw + lay.rb);
  int2 *meta = (int2 *)(smem_raw + lay.meta);
  int *gmin = (int *)(smem_raw + lay.gmin);
  int2 *blk = (int2 *)(smem_raw + lay.blk);
  Stage<T> st;
  st.buf0 = (T *)(smem_raw + lay.buf0);
  st.buf1 = (T *)(smem_raw + lay.buf1);
  st.bar = (uint64_t *)(smem_raw + lay.bar);
  st.blk = blk;
  stage_init(st, &p.sc->copy_timeout, p.stall_test);
  const int64_t *ptr_all = kInv ? p.inv_ptr : p.env_ptr;
  const int64_t base = ptr_all[io];
  if (kInv)
    st.L = (sizeof(T) == 8 ? (const T *)(const void *)p.Linv32 : (const T *)(const void *)p.Linv64) + base;
  else
    st.L = (sizeof(T) == 8 ? (const T *)(const void *)p.L32 : (const T *)(const void *)p.L64) + base;
  const int2 *blk_tab = kInv ? p.inv_blk_tab : p.blk_tab;
  for (int b = tid; b <= nblk; b += nt) blk[b] = blk_tab[b0 + b];
  if (tid == 0) {
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    mbar_init(&st.bar[2], 1);
    fence_mbar_init();
  }
  // right-hand side; a refinement step is skipped when its residual is already small
  double rn = 0.0, bn = 0.0;
  for (int c = tid; c < nI; c += nt) {
    const double2 r = rhs[io + c];
    y[c] = from_d2<T>(r);
    if (accumulate) {
      const double2 bv = p.B[io + c];
      rn = fmax(rn, fabs(r.x) + fabs(r.y));
      bn = fmax(bn, fabs(bv.x) + fabs(bv.y));
    }
  }
  __syncthreads();
  if (accumulate && p.ir_tol > 0.0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      rn = fmax(rn, __shfl_xor_sync(0xffffffffu, rn, o));
      bn = fmax(bn, __shfl_xor_sync(0xffffffffu, bn, o));
    }
    if ((tid & 31) == 0) {
      red[tid >> 5][0] = rn;
      red[tid >> 5][1] = bn;
    }
    __syncthreads();
    for (int k = 0; k < nw; k++) {
      rn = fmax(rn, red[k][0]);
      bn = fmax(bn, red[k][1]);
    }
    if (rn <= p.ir_tol * bn) return;  // the same decision in every thread
  }
  const int32_t *lo_g = p.env_lo + io;
  const int64_t *ptr_g = ptr_all + io;
  T *z = zstash + io;
  // L2: the forward sweep's blocks are read again by the backward sweep, the
  // backward sweep's reads are the last use
  st.hint = 1;
  st.policy = l2_evict_last();
  bool ok = staged_forward<T, kInv>(st, nblk, lo_g, ptr_g, base, y, meta, z, rectb, tid, nw);
  if (ok) {
    for (int c = tid; c < nI; c += nt) y[c] = z[c];
    __syncthreads();
    st.policy = l2_evict_first();
    ok = staged_backward<T, kInv>(st, nblk, lo_g, ptr_g, base, y, xb, meta, gmin, tid, nw);
  }
  // every copy issued into this CTA's shared memory has landed before it exits
  stage_drain(st);
  if (!ok) return;
  for (int c = tid; c < nI; c += nt) {
    double2 x = make_double2((double)y[c].x, (double)y[c].y);
    if (accumulate) x = cadd(xout[io + c], x);
    xout[io + c] = x;
  }
}

// The block-inverse layout of one subdomain's factor, one warp per
// subdomain, block by block.  For the block of rows r0..r0+nb-1:
//   - each row's entries left of the block (columns lo..r0-1), copied;
//   - N = (I + L_bb)^-1 - I, strictly lower, row-major (row i at i(i-1)/2),
//     where L_bb is the block's own part of the unit lower factor; row by
//     row, lane j: N_ij = -(L_ij + sum_{k=j+1}^{i-1} L_ik N_kj), k ascending,
//     in FP64 (then rounded for the FP32 layout);
//   - the rows' pivots 1/d (the envelope's diagonal).
// The sweeps then apply the block's triangle as a product with N instead of
// a row-by-row substitution.
template <typename T>
__global__ void __launch_bounds__(32) inv_relayout_kernel(DevProblem p, const double2 *__restrict__ L64, T *out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *M = (double2 *)smem_raw;  // [32][33]: L_bb
  double2 *Nd = M + 32 * 33;         // [32][33]: N
  const int s = p.sub_order[blockIdx.x], lane = threadIdx.x;  // the subdomains this context solves
  const int64_t io = p.int_off[s];
  const int b0 = p.inv_blk_off[s];
  const int nblk = p.inv_blk_off[s + 1] - b0 - 1;
  for (int b = 0; b < nblk; b++) {
    const int r0 = p.inv_blk_tab[b0 + b].x, nb = p.inv_blk_tab[b0 + b + 1].x - r0;
    int lo = r0;
    int64_t ep = 0, ip = 0;
    if (lane < nb) {
      lo = p.env_lo[io + r0 + lane];
      ep = p.env_ptr[io + r0 + lane];
      ip = p.inv_ptr[io + r0 + lane];
    }
    for (int t = 0; t < nb; t++) {
      const int lo_t = __shfl_sync(0xffffffffu, lo, t);
      const int64_t ep_t = __shfl_sync(0xffffffffu, ep, t), ip_t = __shfl_sync(0xffffffffu, ip, t);
      for (int k = lane; k < r0 - lo_t; k += 32) out[ip_t + k] = from_d2<T>(L64[ep_t + k]);
      const int col = r0 + lane;
      M[t * 33 + lane] = (lane < t && col >= lo_t) ? L64[ep_t + (col - lo_t)] : make_double2(0.0, 0.0);
    }
    __syncwarp();
    for (int i = 1; i < nb; i++) {
      if (lane < i) {
        double2 acc = M[i * 33 + lane];
        for (int k = lane + 1; k < i; k++) acc = cmac(acc, M[i * 33 + k], Nd[k * 33 + lane]);
        Nd[i * 33 + lane] = make_double2(-acc.x, -acc.y);  // lane j reads only its own column of N
      }
    }
    const int lo_l = __shfl_sync(0xffffffffu, lo, nb - 1);
    const int64_t ip_l = __shfl_sync(0xffffffffu, ip, nb - 1);
    const int64_t tri0 = ip_l + max(0, r0 - lo_l);
    for (int i = 1; i < nb; i++)
      if (lane < i) out[tri0 + ((i * (i - 1)) >> 1) + lane] = from_d2<T>(Nd[i * 33 + lane]);
    if (lane < nb) out[tri0 + ((nb * (nb - 1)) >> 1) + lane] = from_d2<T>(L64[ep + (r0 + lane - lo)]);
    __syncwarp();  // M and N are rewritten for the next block
  }
}

// ---- grid-wide products of the staged path, kL lanes per row ------------

template <int kL>
__device__ __forceinline__ double2 group_sum(double2 v) {
#pragma unroll
  for (int o = kL / 2; o > 0; o >>= 1) v = cadd(v, shfl_xor(v, o));
  return v;
}

// rhs[g] = f_I[g] (first and last solves) - A_IG v (all but the first)
template <int kL>
__global__ void rhs_kernel(DevProblem p, int mode, double2 *__restrict__ out) {
  if (mode == kModeIter && p.sc->status != 0) return;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t / kL < p.n_interior;
  const int64_t row = p.row0 + t / kL;
  const int sub = (int)(t % kL);
  double2 acc = cz();
  if (in && mode != kModeFirst) {
    const int64_t q1 = p.cpl_rowptr[row + 1];
    for (int64_t q = p.cpl_rowptr[row] + sub; q < q1; q += kL) acc = cadd(acc, cmul(p.cpl_val[q], p.P[p.cpl_gcol[q]]));
  }
  acc = group_sum<kL>(acc);
  if (in && sub == 0) out[row] = csub(mode != kModeIter ? p.fI[row] : cz(), acc);
}

// q[slot] = A_G. [x; v] (- f_G): x from Y, v = P at the slot's interface DOF.
// The first 4 entries of each lane are loaded together (column indices, then
// values and gathered operands), the rest of a long row in a loop.
template <int kL>
__global__ void iface_product_kernel(DevProblem p, int mode) {
  if (mode == kModeIter && p.sc->status != 0) return;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t / kL < p.n_slots;
  const int64_t row = p.slot0 + t / kL;
  const int sub = (int)(t % kL);
  const bool with_bc = mode != kModeFirst;
  double2 acc = cz();
  if (in) {
    const int64_t q0 = p.ifr_rowptr[row] + sub, q1 = p.ifr_rowptr[row + 1];
    constexpr int kU = 4;
    int32_t g[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) g[u] = q0 + u * kL < q1 ? p.ifr_gcol[q0 + u * kL] : 0;
    double2 a[kU], xv[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const bool in = q0 + u * kL < q1;
      a[u] = in ? p.ifr_val[q0 + u * kL] : cz();
      xv[u] = !in ? cz() : g[u] >= 0 ? p.Y[g[u]] : (with_bc ? p.P[-g[u] - 1] : cz());
    }
#pragma unroll
    for (int u = 0; u < kU; u++) acc = cadd(acc, cmul(a[u], xv[u]));
    for (int64_t q = q0 + kU * kL; q < q1; q += kL) {
      const int32_t gq = p.ifr_gcol[q];
      const double2 x = gq >= 0 ? p.Y[gq] : (with_bc ? p.P[-gq - 1] : cz());
      acc = cadd(acc, cmul(p.ifr_val[q], x));
    }
  }
  acc = group_sum<kL>(acc);
  if (in && sub == 0) {
    if (mode != kModeIter) acc = csub(acc, p.fG[row]);
    p.qloc[row] = acc;
    if (mode == kModeLast) p.V[row] = with_bc ? p.P[p.if_ln[row]] : cz();
  }
}

// refinement residual r = b - A_II x of every subdomain, FP64
template <int kL>
__global__ void ir_residual_kernel(DevProblem p, int mode) {
  if (mode == kModeIter && p.sc->status != 0) return;
  if (refine_skipped(p, mode)) return;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t / kL < p.n_interior;
  const int64_t row = p.row0 + t / kL;
  const int sub = (int)(t % kL);
  double2 acc = cz();
  if (in) {
    const int64_t q1 = p.aii_rowptr[row + 1];
    for (int64_t q = p.aii_rowptr[row] + sub; q < q1; q += kL) acc = cadd(acc, cmul(p.aii_val[q], p.Y[p.aii_gcol[q]]));
  }
  acc = group_sum<kL>(acc);
  if (in && sub == 0) p.Rres[row] = csub(p.B[row], acc);
}

// ----------------------------------------------------------------------------
// interface COCG (ITERATION_S_1ST / ITERATION_S, hddm_solver_s.h:158-400)

constexpr int kRedThreads = 256;
enum { kFPqRe = 0, kFPqIm, kFMax, kFRzRe, kFRzIm, kFL2, kNFields };

__device__ __forceinline__ double2 gather_slots(const DevProblem &p, const double2 *v, int g) {
  double2 q = cz();
  for (int t = p.gq_ptr[g]; t < p.gq_ptr[g + 1]; t++) {
    const int64_t sl = p.gq_slot[t];
    if (sl >= p.slot0 && sl < p.slot0 + p.n_slots) q = cadd(q, v[sl]);
  }
  return q;
}
__device__ __forceinline__ double2 gather_q(const DevProblem &p, int g) { return gather_slots(p, p.qloc, g); }

// A shard's partial interface sums, written to the exchange buffer that the
// caller sums over ranks: Q (and on the first step the diagonal PC sums)
// over this shard's subdomains (COM_RES_SP / DIAG_GATHER_S over one part's
// subdomains, hddm_solver_sp.h:8-25, hddm_pc.h:110-124).

// first step: Q and PC gathered over subdomains (hddm_solver_s.h:174-181),
// PC reciprocal (hddm_pc.h:128-135), r = Q, z = r pc, p = z, max|r|, (r, z)
__global__ void cocg_first_kernel(DevProblem p, const double2 *__restrict__ pcloc) {
  __shared__ double sh[40];
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.nfree; g += gridDim.x * blockDim.x) {
    const double2 q = gather_q(p, g);
    double2 pc = gather_slots(p, pcloc, g);
    pc = ciszero(pc) ? make_double2(1.0, 0.0) : cdiv_ref(make_double2(1.0, 0.0), pc);
    p.PC[g] = pc;
    p.Q[g] = q;
    p.R[g] = q;
    const double2 z = cmul(q, pc);
    p.Z[g] = z;
    p.P[g] = z;
    p.U[g] = cz();
    mx = fmax(mx, cabs_ref(q));
    const double2 rz = cmul(q, z);
    rzr += rz.x;
    rzi += rz.y;
    l2 += q.x * q.x + q.y * q.y;
  }
  const int nb = p.n_part_blocks;
  double r;
  r = block_max(mx, sh);
  if (threadIdx.x == 0) p.part[kFMax * nb + blockIdx.x] = r;
  r = block_sum(rzr, sh);
  if (threadIdx.x == 0) p.part[kFRzRe * nb + blockIdx.x] = r;
  r = block_sum(rzi, sh);
  if (threadIdx.x == 0) p.part[kFRzIm * nb + blockIdx.x] = r;
  r = block_sum(l2, sh);
  if (threadIdx.x == 0) p.part[kFL2 * nb + blockIdx.x] = r;
}

__global__ void cocg_first_scalars_kernel(DevProblem p) {
  __shared__ double sh[40];
  const int nb = p.n_part_blocks;
  const double mx = reduce_partials(p.part, nb, kFMax, true, sh);
  const double rzr = reduce_partials(p.part, nb, kFRzRe, false, sh);
  const double rzi = reduce_partials(p.part, nb, kFRzIm, false, sh);
  const double l2 = reduce_partials(p.part, nb, kFL2, false, sh);
  if (threadIdx.x == 0) {
    CocgScalars *sc = p.sc;
    // fmax drops NaN, so a non-finite residual shows in the sums only
    const bool bad = !isfinite(mx) || !isfinite(l2) || !isfinite(rzr) || !isfinite(rzi);
    sc->norm0 = mx;
    sc->l2_0 = sqrt(l2);
    sc->status = (bad || mx < kNearlyZero) ? 1 : 0;
    sc->r0inv = 1.0 / mx;
    sc->rz = make_double2(rzr, rzi);
    sc->resi = 1.0;
    sc->resi_l2 = 1.0;
    sc->loop = 1;
    sc->converged = (!bad && mx < kNearlyZero) ? 1 : 0;
    sc->nonfinite = bad ? 1 : 0;
  }
}

// Q gathered over subdomains (hddm_solver_s.h:273 with COM_RES_SP), (p, q),
// and in the last CTA -alpha = -(r, z) / (p, q)  (hddm_solver_s.h:282-295)
__global__ void cocg_gather_pq_kernel(DevProblem p) {
  if (p.sc->status != 0) return;
  __shared__ double sh[40];
  double re = 0.0, im = 0.0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.nfree; g += gridDim.x * blockDim.x) {
    const double2 q = gather_q(p, g);
    p.Q[g] = q;
    const double2 t = cmul(p.P[g], q);
    re += t.x;
    im += t.y;
  }
  const int nb = p.n_part_blocks;
  double r = block_sum(re, sh);
  if (threadIdx.x == 0) p.part[kFPqRe * nb + blockIdx.x] = r;
  r = block_sum(im, sh);
  if (threadIdx.x == 0) p.part[kFPqIm * nb + blockIdx.x] = r;
  if (!last_cta(&p.sc->ticket[0])) return;
  const double pr = reduce_partials(p.part, nb, kFPqRe, false, sh);
  const double pi = reduce_partials(p.part, nb, kFPqIm, false, sh);
  if (threadIdx.x == 0) {
    CocgScalars *sc = p.sc;
    const double2 pq = make_double2(pr, pi);
    if (cabs_ref(sc->rz) < kNearlyZero && cabs_ref(pq) < kNearlyZero) {
      sc->malpha = cz();
    } else {
      sc->malpha = csub(cz(), cdiv_ref(sc->rz, pq));
    }
    sc->ticket[0] = 0;
  }
}

// u += -alpha p, r += -alpha q, max|r|, z = r pc, (r, z)  (hddm_solver_s.h:297-344)
__global__ void cocg_update_kernel(DevProblem p) {
  if (p.sc->status != 0) return;
  __shared__ double sh[40];
  const double2 ma = p.sc->malpha;
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.nfree; g += gridDim.x * blockDim.x) {
    p.U[g] = cadd(p.U[g], cmul(ma, p.P[g]));
    const double2 r = cadd(p.R[g], cmul(ma, p.Q[g]));
    p.R[g] = r;
    mx = fmax(mx, cabs_ref(r));
    const double2 z = cmul(r, p.PC[g]);
    p.Z[g] = z;
    const double2 rz = cmul(r, z);
    rzr += rz.x;
    rzi += rz.y;
    l2 += r.x * r.x + r.y * r.y;
  }
  const int nb = p.n_part_blocks;
  double r;
  r = block_max(mx, sh);
  if (threadIdx.x == 0) p.part[kFMax * nb + blockIdx.x] = r;
  r = block_sum(rzr, sh);
  if (threadIdx.x == 0) p.part[kFRzRe * nb + blockIdx.x] = r;
  r = block_sum(rzi, sh);
  if (threadIdx.x == 0) p.part[kFRzIm * nb + blockIdx.x] = r;
  r = block_sum(l2, sh);
  if (threadIdx.x == 0) p.part[kFL2 * nb + blockIdx.x] = r;
  // last CTA: resi, beta = (r', z') / (r, z), convergence and loop count
  // (hddm_solver_s.h:318-379, hddm_solver.h:125-143)
  if (!last_cta(&p.sc->ticket[1])) return;
  const double rmx = reduce_partials(p.part, nb, kFMax, true, sh);
  const double rzr_t = reduce_partials(p.part, nb, kFRzRe, false, sh);
  const double rzi_t = reduce_partials(p.part, nb, kFRzIm, false, sh);
  const double l2_t = reduce_partials(p.part, nb, kFL2, false, sh);
  if (threadIdx.x == 0) {
    CocgScalars *sc = p.sc;
    const double resi = rmx * sc->r0inv;
    sc->resi = resi;
    sc->resi_l2 = sqrt(l2_t) / sc->l2_0;
    if (sc->loop - 1 < p.hist_cap) p.hist[sc->loop - 1] = resi;
    const double2 rz = make_double2(rzr_t, rzi_t);
    if (cabs_ref(rz) < kNearlyZero && cabs_ref(sc->rz) < kNearlyZero) {
      sc->beta = cz();
    } else {
      sc->beta = cdiv_ref(rz, sc->rz);
    }
    sc->rz = rz;
    if (!isfinite(l2_t) || !isfinite(rzr_t) || !isfinite(rzi_t)) {
      // the reference would run on to hddm_max_loop; stop and report it
      sc->status = 1;
      sc->nonfinite = 1;
    } else if (resi < sc->eps) {
      sc->status = 1;
      sc->converged = 1;
    } else if (sc->loop >= sc->max_loop) {
      sc->status = 1;
    }
    sc->loop += 1;
    sc->ticket[1] = 0;
  }
}

// p = z + beta p, or p = u after the last iteration (hddm_solver_s.h:356-376)
// After the last iteration's p = u the last CTA marks the loop finished
// (status 2), so that the iterations left in a graph launch do nothing.
__global__ void cocg_pupdate_kernel(DevProblem p) {
  const int st = p.sc->status;
  if (st == 2) return;
  const double2 be = p.sc->beta;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.nfree; g += gridDim.x * blockDim.x) {
    p.P[g] = st == 1 ? p.U[g] : cadd(p.Z[g], cmul(be, p.P[g]));
  }
  if (st == 1 && last_cta(&p.sc->ticket[2]) && threadIdx.x == 0) {
    p.sc->status = 2;
    p.sc->ticket[2] = 0;
  }
}

// ---- sharded solve, exchange packed to the shared interface DOFs -----------
// Every shard runs the COCG on the interface DOFs its subdomains hold (the
// same recurrence as the kernels above, on the same summed values, so the
// shards holding a DOF keep the same bits for it); the dot products and the
// max-norm run over the DOFs it owns, and the shards add them up (the
// reference's p-mode: hddm_solver_ph.h:112-131,158-175,199,228-329).  Only
// the DOFs held by two or more shards cross between the ranks, packed.

__device__ __forceinline__ double2 dist_q(const DevProblem &p, int i, int g) {
  const int pos = p.dist_pos[i];
  return pos >= 0 ? p.dist_pack[pos] : gather_slots(p, p.qloc, g);
}

// this shard's partial Q (and PC diagonal) of its shared DOFs; the host
// zeroed the packed buffer, so the DOFs it does not hold add nothing
__global__ void dist_pack_kernel(DevProblem p, const double2 *__restrict__ pcloc, int with_pc, int status_check) {
  if (status_check && p.sc->status != 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.dist_n; i += gridDim.x * blockDim.x) {
    const int pos = p.dist_pos[i];
    if (pos < 0) continue;
    const int g = p.dist_dof[i];
    p.dist_pack[pos] = gather_slots(p, p.qloc, g);
    if (with_pc) p.dist_pack[p.n_shared + pos] = gather_slots(p, pcloc, g);
  }
}

// the first step on the held DOFs (cocg_first_kernel); the last CTA writes the
// local sums of the owned DOFs: (r, z) and |r|^2 to scal[0..2], max|r| to scal[4]
__global__ void dist_first_kernel(DevProblem p, const double2 *__restrict__ pcloc) {
  __shared__ double sh[40];
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.dist_n; i += gridDim.x * blockDim.x) {
    const int g = p.dist_dof[i], pos = p.dist_pos[i];
    const double2 q = dist_q(p, i, g);
    double2 pc = pos >= 0 ? p.dist_pack[p.n_shared + pos] : gather_slots(p, pcloc, g);
    pc = ciszero(pc) ? make_double2(1.0, 0.0) : cdiv_ref(make_double2(1.0, 0.0), pc);
    p.PC[g] = pc;
    p.Q[g] = q;
    p.R[g] = q;
    const double2 z = cmul(q, pc);
    p.Z[g] = z;
    p.P[g] = z;
    p.U[g] = cz();
    if (p.dist_own[i]) {
      mx = fmax(mx, cabs_ref(q));
      const double2 rz = cmul(q, z);
      rzr += rz.x;
      rzi += rz.y;
      l2 += q.x * q.x + q.y * q.y;
    }
  }
  const int nb = p.n_part_blocks;
  double r;
  r = block_max(mx, sh);
  if (threadIdx.x == 0) p.part[kFMax * nb + blockIdx.x] = r;
  r = block_sum(rzr, sh);
  if (threadIdx.x == 0) p.part[kFRzRe * nb + blockIdx.x] = r;
  r = block_sum(rzi, sh);
  if (threadIdx.x == 0) p.part[kFRzIm * nb + blockIdx.x] = r;
  r = block_sum(l2, sh);
  if (threadIdx.x == 0) p.part[kFL2 * nb + blockIdx.x] = r;
  if (!last_cta(&p.sc->ticket[0])) return;
  const double vmx = reduce_partials(p.part, nb, kFMax, true, sh);
  const double vrr = reduce_partials(p.part, nb, kFRzRe, false, sh);
  const double vri = reduce_partials(p.part, nb, kFRzIm, false, sh);
  const double vl2 = reduce_partials(p.part, nb, kFL2, false, sh);
  if (threadIdx.x == 0) {
    p.dist_scal[0] = vrr;
    p.dist_scal[1] = vri;
    p.dist_scal[2] = vl2;
    p.dist_scal[4] = vmx;
    p.sc->ticket[0] = 0;
  }
}

// the first step's scalars from the summed values (cocg_first_scalars_kernel)
__global__ void dist_first_finish_kernel(DevProblem p) {
  CocgScalars *sc = p.sc;
  const double mx = p.dist_scal[4], rzr = p.dist_scal[0], rzi = p.dist_scal[1], l2 = p.dist_scal[2];
  const bool bad = !isfinite(mx) || !isfinite(l2) || !isfinite(rzr) || !isfinite(rzi);
  sc->norm0 = mx;
  sc->l2_0 = sqrt(l2);
  sc->status = (bad || mx < kNearlyZero) ? 1 : 0;
  sc->r0inv = 1.0 / mx;
  sc->rz = make_double2(rzr, rzi);
  sc->resi = 1.0;
  sc->resi_l2 = 1.0;
  sc->loop = 1;
  sc->converged = (!bad && mx < kNearlyZero) ? 1 : 0;
  sc->nonfinite = bad ? 1 : 0;
}

// Q on the held DOFs and the local (p, q) of the owned ones -> scal[0..1]
__global__ void dist_pq_kernel(DevProblem p) {
  if (p.sc->status != 0) return;
  __shared__ double sh[40];
  double re = 0.0, im = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.dist_n; i += gridDim.x * blockDim.x) {
    const int g = p.dist_dof[i];
    const double2 q = dist_q(p, i, g);
    p.Q[g] = q;
    if (p.dist_own[i]) {
      const double2 t = cmul(p.P[g], q);
      re += t.x;
      im += t.y;
    }
  }
  const int nb = p.n_part_blocks;
  double r = block_sum(re, sh);
  if (threadIdx.x == 0) p.part[kFPqRe * nb + blockIdx.x] = r;
  r = block_sum(im, sh);
  if (threadIdx.x == 0) p.part[kFPqIm * nb + blockIdx.x] = r;
  if (!last_cta(&p.sc->ticket[0])) return;
  const double pr = reduce_partials(p.part, nb, kFPqRe, false, sh);
  const double pi = reduce_partials(p.part, nb, kFPqIm, false, sh);
  if (threadIdx.x == 0) {
    p.dist_scal[0] = pr;
    p.dist_scal[1] = pi;
    p.sc->ticket[0] = 0;
  }
}

// -alpha from the summed (p, q) (every thread the same), u += -alpha p,
// r += -alpha q, z on the held DOFs; the local sums of the owned ones
__global__ void dist_update_kernel(DevProblem p) {
  if (p.sc->status != 0) return;
  __shared__ double sh[40];
  const double2 pq = make_double2(p.dist_scal[0], p.dist_scal[1]);
  const double2 rz0 = p.sc->rz;
  const double2 ma =
      (cabs_ref(rz0) < kNearlyZero && cabs_ref(pq) < kNearlyZero) ? cz() : csub(cz(), cdiv_ref(rz0, pq));
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.dist_n; i += gridDim.x * blockDim.x) {
    const int g = p.dist_dof[i];
    p.U[g] = cadd(p.U[g], cmul(ma, p.P[g]));
    const double2 r = cadd(p.R[g], cmul(ma, p.Q[g]));
    p.R[g] = r;
    const double2 z = cmul(r, p.PC[g]);
    p.Z[g] = z;
    if (p.dist_own[i]) {
      mx = fmax(mx, cabs_ref(r));
      const double2 rz = cmul(r, z);
      rzr += rz.x;
      rzi += rz.y;
      l2 += r.x * r.x + r.y * r.y;
    }
  }
  const int nb = p.n_part_blocks;
  double r;
  r = block_max(mx, sh);
  if (threadIdx.x == 0) p.part[kFMax * nb + blockIdx.x] = r;
  r = block_sum(rzr, sh);
  if (threadIdx.x == 0) p.part[kFRzRe * nb + blockIdx.x] = r;
  r = block_sum(rzi, sh);
  if (threadIdx.x == 0) p.part[kFRzIm * nb + blockIdx.x] = r;
  r = block_sum(l2, sh);
  if (threadIdx.x == 0) p.part[kFL2 * nb + blockIdx.x] = r;
  if (!last_cta(&p.sc->ticket[1])) return;
  const double vmx = reduce_partials(p.part, nb, kFMax, true, sh);
  const double vrr = reduce_partials(p.part, nb, kFRzRe, false, sh);
  const double vri = reduce_partials(p.part, nb, kFRzIm, false, sh);
  const double vl2 = reduce_partials(p.part, nb, kFL2, false, sh);
  if (threadIdx.x == 0) {
    p.sc->malpha = ma;
    p.dist_scal[0] = vrr;
    p.dist_scal[1] = vri;
    p.dist_scal[2] = vl2;
    p.dist_scal[4] = vmx;
    p.sc->ticket[1] = 0;
  }
}

// resi, beta, the stopping test (the last CTA of cocg_update_kernel) from
// the summed values
__global__ void dist_finish_kernel(DevProblem p) {
  CocgScalars *sc = p.sc;
  if (sc->status != 0) return;
  const double rzr_t = p.dist_scal[0], rzi_t = p.dist_scal[1], l2_t = p.dist_scal[2], rmx = p.dist_scal[4];
  const double resi = rmx * sc->r0inv;
  sc->resi = resi;
  sc->resi_l2 = sqrt(l2_t) / sc->l2_0;
  if (sc->loop - 1 < p.hist_cap) p.hist[sc->loop - 1] = resi;
  const double2 rz = make_double2(rzr_t, rzi_t);
  if (cabs_ref(rz) < kNearlyZero && cabs_ref(sc->rz) < kNearlyZero) {
    sc->beta = cz();
  } else {
    sc->beta = cdiv_ref(rz, sc->rz);
  }
  sc->rz = rz;
  if (!isfinite(l2_t) || !isfinite(rzr_t) || !isfinite(rzi_t)) {
    sc->status = 1;
    sc->nonfinite = 1;
  } else if (resi < sc->eps) {
    sc->status = 1;
    sc->converged = 1;
  } else if (sc->loop >= sc->max_loop) {
    sc->status = 1;
  }
  sc->loop += 1;
}

// p = z + beta p, or p = u after the last iteration, on the held DOFs
__global__ void dist_pupdate_kernel(DevProblem p) {
  const int st = p.sc->status;
  if (st == 2) return;
  const double2 be = p.sc->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.dist_n; i += gridDim.x * blockDim.x) {
    const int g = p.dist_dof[i];
    p.P[g] = st == 1 ? p.U[g] : cadd(p.Z[g], cmul(be, p.P[g]));
  }
  if (st == 1 && last_cta(&p.sc->ticket[2]) && threadIdx.x == 0) {
    p.sc->status = 2;
    p.sc->ticket[2] = 0;
  }
}

// Edge value from the first subdomain holding the edge; a shard gives the
// edges whose first holder it owns and zero for the others.
__global__ void edge_solution_kernel(int64_t ne, const int64_t *__restrict__ src, const double2 *__restrict__ Y,
                                     const double2 *__restrict__ V, double2 *__restrict__ x, int64_t row0,
                                     int64_t nrow, int64_t slot0, int64_t nslot) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int64_t s = src[e];
  double2 v = make_double2(0.0, 0.0);
  if (s >= 0 && s >= row0 && s < row0 + nrow) v = Y[s];
  if (s < -1 && -s - 2 >= slot0 && -s - 2 < slot0 + nslot) v = V[-s - 2];
  x[e] = v;
}

__global__ void set_status_kernel(CocgScalars *sc, double eps, int32_t max_loop) {
  for (int i = 0; i < 4; i++) sc->ticket[i] = 0;
  sc->eps = eps;
  sc->max_loop = max_loop;
  sc->status = 0;
  sc->converged = 0;
  sc->nonfinite = 0;
}

// iteration state for kernel timing: never converges, no loop limit
__global__ void profile_reset_kernel(CocgScalars *sc) {
  for (int i = 0; i < 4; i++) sc->ticket[i] = 0;
  sc->status = 0;
  sc->eps = -1.0;
  sc->max_loop = 0x7fffffff;
  sc->loop = 1;
}

unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }
// at least one block: the kernels skip rows past the end
unsigned blocks_min1(int64_t n, int threads) { return n > 0 ? blocks_for(n, threads) : 1u; }

}  // namespace

void launch_gather_values(int64_t nnz, const int64_t *contrib_ptr, const int64_t *contrib, const double2 *elmat,
                          double2 *aval, cudaStream_t stream) {
  if (nnz <= 0) return;
  gather_values_kernel<<<blocks_for(nnz, 256), 256, 0, stream>>>(nnz, contrib_ptr, contrib, elmat, aval);
}

void launch_profile(int32_t nsub, const int64_t *dof_off, const int64_t *nnz_off, const int32_t *row_ptr_rel,
                    const int32_t *col, const double2 *aval, const uint8_t *isbc, int32_t *idx1,
                    cudaStream_t stream) {
  profile_kernel<<<blocks_for((int64_t)nsub * 32, kThreads), kThreads, 0, stream>>>(nsub, dof_off, nnz_off,
                                                                                      row_ptr_rel, col, aval, isbc,
                                                                                      idx1);
}

void launch_scatter_envelope(int64_t nnz, const int64_t *dst, const double2 *aval, double2 *L, cudaStream_t stream) {
  if (nnz <= 0) return;
  scatter_envelope_kernel<<<blocks_for(nnz, 256), 256, 0, stream>>>(nnz, dst, aval, L);
}

void launch_gather_ops(int64_t n, const int64_t *src, const double2 *aval, double2 *dst, cudaStream_t stream) {
  if (n <= 0) return;
  gather_ops_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, src, aval, dst);
}

void launch_diag_pc(int64_t n, const int64_t *diag_src, const double2 *aval, double2 *pcloc, cudaStream_t stream) {
  if (n <= 0) return;
  diag_pc_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, diag_src, aval, pcloc);
}

void launch_factor(const DevProblem &p, const int64_t *int_off, const int32_t *env_lo, const int64_t *env_ptr,
                   double2 *L, int32_t *status, cudaStream_t stream) {
  factor_kernel<<<blocks_for((int64_t)p.nsub * 32, kThreads), kThreads, 0, stream>>>(p.nsub, p.sub_order, int_off,
                                                                                       env_lo, env_ptr, L, status);
}

void launch_to_fp32(int64_t n, const double2 *src, float2 *dst, cudaStream_t stream) {
  if (n <= 0) return;
  to_fp32_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, src, dst);
}

size_t subsolve_smem_bytes(int max_interior, int max_iface, bool fp32) {
  return cta_smem_bytes(max_interior, max_iface, fp32);
}

template <bool kInv>
void launch_staged(const DevProblem &p, int mode, bool fp32, cudaStream_t stream) {
  const StageLayout lay = kInv ? stage_layout(p.max_interior, p.inv_max_blocks, p.inv_cap, fp32)
                               : stage_layout(p.max_interior, p.max_blocks, p.stage_cap, fp32);
  double2 *rhs = fp32 ? p.B : p.Y;
  // one thread per row for both products: their rows are short (a few to a
  // few tens of entries) and the loads of several entries in flight per
  // thread beat lanes sharing a row (timed with 1, 2, 4 and 8 lanes)
  rhs_kernel<1><<<blocks_min1(p.n_interior, 256), 256, 0, stream>>>(p, mode, rhs);
  if (fp32) {
    subsolve_staged_kernel<float2, kInv><<<p.nsub, 32 * p.stage_warps, lay.total, stream>>>(p, mode, p.B, p.Y, p.Y32,
                                                                                           0, lay);
    for (int k = 0; k < p.ir_steps; k++) {
      ir_residual_kernel<4><<<blocks_min1(p.n_interior * 4, 256), 256, 0, stream>>>(p, mode);
      subsolve_staged_kernel<float2, kInv><<<p.nsub, 32 * p.stage_warps, lay.total, stream>>>(p, mode, p.Rres, p.Y,
                                                                                             p.Y32, 1, lay);
    }
  } else {
    subsolve_staged_kernel<double2, kInv><<<p.nsub, 32 * p.stage_warps, lay.total, stream>>>(p, mode, p.Y, p.Y, p.Y,
                                                                                            0, lay);
  }
  iface_product_kernel<1><<<blocks_min1(p.n_slots, 256), 256, 0, stream>>>(p, mode);
}

void launch_subsolve(const DevProblem &p, int mode, bool fp32, cudaStream_t stream) {
  if (p.solve_variant == kSolveWarp) {
    launch_staged<false>(p, mode, fp32, stream);
    return;
  }
  if (p.solve_variant == kSolveInv) {
    launch_staged<true>(p, mode, fp32, stream);
    return;
  }
  if (p.solve_variant == kSolveCta && p.cta_smem > 0) {
    if (fp32)
      subsolve_cta_kernel<true><<<p.nsub, kCtaThreads, p.cta_smem, stream>>>(p, mode);
    else
      subsolve_cta_kernel<false><<<p.nsub, kCtaThreads, p.cta_smem, stream>>>(p, mode);
    return;
  }
  // subdomains too large for one CTA's shared memory: one warp each, vectors in global memory
  const unsigned nb = blocks_for((int64_t)p.nsub * 32, kThreads);
  if (fp32)
    subsolve_kernel<true><<<nb, kThreads, 0, stream>>>(p, mode);
  else
    subsolve_kernel<false><<<nb, kThreads, 0, stream>>>(p, mode);
}

size_t subsolve_staged_smem_bytes(int max_interior, int max_blocks, int cap, bool fp32) {
  return stage_layout(max_interior, max_blocks, cap, fp32).total;
}

// The dynamic shared-memory limit of a kernel is process-wide (per device):
// it is only ever raised, so that a context configured later with smaller
// subdomains cannot break the launches of an earlier one.
// Each kernel has a slot of its own (SmemSlot): two kernels sharing one would
// see the other's limit as theirs and launch above their own.  A failed
// attribute call is cleared from the runtime's last error, so that a later
// check of a launch does not report it.
int raise_smem_limit(const void *func, int slot, size_t smem) {
  constexpr int kDevs = 64;
  static std::mutex mu;
  static size_t current[kDevs][kSmemSlots] = {};
  if (smem > 227 * 1024) return -1;
  if (slot < 0 || slot >= kSmemSlots) return -2;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) return -2;
  std::lock_guard<std::mutex> lock(mu);
  if (smem <= current[dev][slot]) return 0;
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    (void)cudaGetLastError();
    return -2;
  }
  current[dev][slot] = smem;
  return 0;
}

int configure_subsolve_staged(size_t smem, bool fp32) {
  return fp32 ? raise_smem_limit((const void *)subsolve_staged_kernel<float2, false>, kSlotStaged32, smem)
              : raise_smem_limit((const void *)subsolve_staged_kernel<double2, false>, kSlotStaged64, smem);
}

int configure_subsolve_inv(size_t smem, bool fp32) {
  return fp32 ? raise_smem_limit((const void *)subsolve_staged_kernel<float2, true>, kSlotInv32, smem)
              : raise_smem_limit((const void *)subsolve_staged_kernel<double2, true>, kSlotInv64, smem);
}

void launch_inv_relayout(const DevProblem &p, const double2 *L64, bool fp32, cudaStream_t stream) {
  if (p.nsub <= 0) return;
  constexpr size_t smem = 2 * 32 * 33 * sizeof(double2);
  if (fp32)
    inv_relayout_kernel<float2><<<p.nsub, 32, smem, stream>>>(p, L64, (float2 *)(void *)p.Linv32);
  else
    inv_relayout_kernel<double2><<<p.nsub, 32, smem, stream>>>(p, L64, (double2 *)(void *)p.Linv64);
}

int subsolve_launches(const DevProblem &p, bool fp32) {
  if (p.solve_variant == kSolveWarp || p.solve_variant == kSolveInv) return 3 + (fp32 ? 2 * p.ir_steps : 0);
  return 1;
}

int configure_subsolve(size_t smem, bool fp32) {
  return fp32 ? raise_smem_limit((const void *)subsolve_cta_kernel<true>, kSlotCta32, smem)
              : raise_smem_limit((const void *)subsolve_cta_kernel<false>, kSlotCta64, smem);
}

void launch_cocg_first(const DevProblem &p, const double2 *pcloc, cudaStream_t stream) {
  cocg_first_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p, pcloc);
  cocg_first_scalars_kernel<<<1, kRedThreads, 0, stream>>>(p);
}

void launch_cocg_update(const DevProblem &p, cudaStream_t stream) {
  cocg_gather_pq_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
  cocg_update_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
  cocg_pupdate_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
}

void launch_cocg_iteration(const DevProblem &p, cudaStream_t stream) {
  launch_subsolve(p, kModeIter, p.L32 != nullptr, stream);
  launch_cocg_update(p, stream);
}

void launch_edge_solution(const DevProblem &p, int64_t ne, const int64_t *edge_src, const double2 *Y,
                          const double2 *V, double2 *x, cudaStream_t stream) {
  if (ne <= 0) return;
  edge_solution_kernel<<<blocks_for(ne, 256), 256, 0, stream>>>(ne, edge_src, Y, V, x, p.row0, p.n_interior, p.slot0,
                                                                 p.n_slots);
}


void launch_profile_reset(CocgScalars *sc, cudaStream_t stream) { profile_reset_kernel<<<1, 1, 0, stream>>>(sc); }

void launch_dist_pack(const DevProblem &p, const double2 *pcloc, bool with_pc, bool status_check, cudaStream_t stream) {
  dist_pack_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p, pcloc, with_pc ? 1 : 0, status_check ? 1 : 0);
}
void launch_dist_first(const DevProblem &p, const double2 *pcloc, cudaStream_t stream) {
  dist_first_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p, pcloc);
}
void launch_dist_first_finish(const DevProblem &p, cudaStream_t stream) {
  dist_first_finish_kernel<<<1, 1, 0, stream>>>(p);
}
void launch_dist_pq(const DevProblem &p, cudaStream_t stream) {
  dist_pq_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
}
void launch_dist_update(const DevProblem &p, cudaStream_t stream) {
  dist_update_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
}
void launch_dist_finish(const DevProblem &p, cudaStream_t stream) {
  dist_finish_kernel<<<1, 1, 0, stream>>>(p);
  dist_pupdate_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
}

void launch_set_status(CocgScalars *sc, double eps, int32_t max_loop, cudaStream_t stream) {
  set_status_kernel<<<1, 1, 0, stream>>>(sc, eps, max_loop);
}

}  // namespace fw
