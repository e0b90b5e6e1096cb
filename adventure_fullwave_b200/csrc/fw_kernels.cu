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

#include <cstdint>
#include <type_traits>

#include "fw_kernels.cuh"

namespace fw {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;
constexpr double kNearlyZero = 1.0e-60;  // NEARLY_ZERO, lib/std/defs.h:105

__device__ __forceinline__ double2 cz() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cabs_ref(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }  // ComplexAbs
__device__ __forceinline__ bool ciszero(double2 a) { return a.x == 0.0 && a.y == 0.0; }           // ISZERO
// ComplexReciprocal / ComplexDivide (lib/std/complex_adv.c:39-52,133-137)
__device__ __forceinline__ double2 crecip_ref(double2 a) {
  const double d = 1.0 / (a.x * a.x + a.y * a.y);
  return make_double2(a.x * d, -(a.y * d));
}
__device__ __forceinline__ double2 cdiv_ref(double2 a, double2 b) { return cmul(a, crecip_ref(b)); }
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

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int o);
template <>
__device__ __forceinline__ double2 shfl_xor(double2 v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
template <>
__device__ __forceinline__ float2 shfl_xor(float2 v, int o) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = cadd(v, shfl_xor(v, o));
  return v;
}

template <typename T>
__device__ __forceinline__ T czero();
template <>
__device__ __forceinline__ double2 czero<double2>() {
  return make_double2(0.0, 0.0);
}
template <>
__device__ __forceinline__ float2 czero<float2>() {
  return make_float2(0.0f, 0.0f);
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
    for (int step = 0; step < p.ir_steps; step++) {
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

template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src);
template <>
__device__ __forceinline__ double2 shfl_idx(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <>
__device__ __forceinline__ float2 shfl_idx(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

template <typename T>
__device__ __forceinline__ T from_d2(double2 a);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 a) {
  return a;
}
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}

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
    for (int step = 0; step < p.ir_steps; step++) {
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
// interface COCG (ITERATION_S_1ST / ITERATION_S, hddm_solver_s.h:158-400)

constexpr int kRedThreads = 256;
enum { kFPqRe = 0, kFPqIm, kFMax, kFRzRe, kFRzIm, kFL2, kNFields };

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r += sh[i];
  return r;  // valid in thread 0
}
__device__ __forceinline__ double block_max(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r = fmax(r, sh[i]);
  return r;
}

// reduce the per-block partials of field f in a fixed order (one block)
__device__ double reduce_partials(const double *part, int nb, int f, bool is_max, double *sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    const double x = part[f * nb + i];
    v = is_max ? fmax(v, x) : v + x;
  }
  double r = is_max ? block_max(v, sh) : block_sum(v, sh);
  __syncthreads();
  if (threadIdx.x == 0) sh[32] = r;
  __syncthreads();
  r = sh[32];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double2 gather_q(const DevProblem &p, int g) {
  double2 q = cz();
  for (int t = p.gq_ptr[g]; t < p.gq_ptr[g + 1]; t++) q = cadd(q, p.qloc[p.gq_slot[t]]);
  return q;
}

// first step: Q and PC gathered over subdomains (hddm_solver_s.h:174-181),
// PC reciprocal (hddm_pc.h:128-135), r = Q, z = r pc, p = z, max|r|, (r, z)
__global__ void cocg_first_kernel(DevProblem p, const double2 *__restrict__ pcloc) {
  __shared__ double sh[40];
  double mx = 0.0, rzr = 0.0, rzi = 0.0, l2 = 0.0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.nfree; g += gridDim.x * blockDim.x) {
    const double2 q = gather_q(p, g);
    double2 pc = cz();
    for (int t = p.gq_ptr[g]; t < p.gq_ptr[g + 1]; t++) pc = cadd(pc, pcloc[p.gq_slot[t]]);
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
    sc->norm0 = mx;
    sc->l2_0 = sqrt(l2);
    sc->status = mx < kNearlyZero ? 1 : 0;
    sc->r0inv = 1.0 / mx;
    sc->rz = make_double2(rzr, rzi);
    sc->pad = 0;
    sc->resi = 1.0;
    sc->resi_l2 = 1.0;
    sc->loop = 1;
    sc->converged = mx < kNearlyZero ? 1 : 0;
  }
}

__global__ void cocg_begin_kernel(CocgScalars *sc) {
  if (sc->status == 1) sc->status = 2;
}

// Q gathered over subdomains (hddm_solver_s.h:273 with COM_RES_SP) and (p, q)
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
}

// -alpha = -(r, z) / (p, q)  (hddm_solver_s.h:282-295)
__global__ void cocg_alpha_kernel(DevProblem p) {
  if (p.sc->status != 0) return;
  __shared__ double sh[40];
  const int nb = p.n_part_blocks;
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
}

// resi, beta = (r', z') / (r, z), convergence and loop count
// (hddm_solver_s.h:318-379, hddm_solver.h:125-143)
__global__ void cocg_beta_kernel(DevProblem p) {
  if (p.sc->status != 0) return;
  __shared__ double sh[40];
  const int nb = p.n_part_blocks;
  const double mx = reduce_partials(p.part, nb, kFMax, true, sh);
  const double rzr = reduce_partials(p.part, nb, kFRzRe, false, sh);
  const double rzi = reduce_partials(p.part, nb, kFRzIm, false, sh);
  const double l2 = reduce_partials(p.part, nb, kFL2, false, sh);
  if (threadIdx.x == 0) {
    CocgScalars *sc = p.sc;
    const double resi = mx * sc->r0inv;
    sc->resi = resi;
    sc->resi_l2 = sqrt(l2) / sc->l2_0;
    if (sc->loop - 1 < p.hist_cap) p.hist[sc->loop - 1] = resi;
    const double2 rz = make_double2(rzr, rzi);
    if (cabs_ref(rz) < kNearlyZero && cabs_ref(sc->rz) < kNearlyZero) {
      sc->beta = cz();
    } else {
      sc->beta = cdiv_ref(rz, sc->rz);
    }
    sc->rz = rz;
    if (resi < sc->eps) {
      sc->status = 1;
      sc->converged = 1;
    } else if (sc->loop >= sc->max_loop) {
      sc->status = 1;
    }
    sc->loop += 1;
  }
}

// p = z + beta p, or p = u after the last iteration (hddm_solver_s.h:356-376)
__global__ void cocg_pupdate_kernel(DevProblem p) {
  const int st = p.sc->status;
  if (st == 2) return;
  const double2 be = p.sc->beta;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < p.nfree; g += gridDim.x * blockDim.x) {
    p.P[g] = st == 1 ? p.U[g] : cadd(p.Z[g], cmul(be, p.P[g]));
  }
}

__global__ void edge_solution_kernel(int64_t ne, const int64_t *__restrict__ src, const double2 *__restrict__ Y,
                                     const double2 *__restrict__ V, double2 *__restrict__ x) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int64_t s = src[e];
  x[e] = s >= 0 ? Y[s] : (s < -1 ? V[-s - 2] : make_double2(0.0, 0.0));
}

__global__ void set_status_kernel(CocgScalars *sc, double eps, int32_t max_loop) {
  sc->eps = eps;
  sc->max_loop = max_loop;
  sc->status = 0;
  sc->converged = 0;
  sc->pad = 0;
}

// iteration state for kernel timing: never converges, no loop limit
__global__ void profile_reset_kernel(CocgScalars *sc) {
  sc->status = 0;
  sc->eps = -1.0;
  sc->max_loop = 0x7fffffff;
  sc->loop = 1;
}

unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

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

void launch_subsolve(const DevProblem &p, int mode, bool fp32, cudaStream_t stream) {
  if (p.cta_smem > 0) {
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

int configure_subsolve(size_t smem) {
  if (smem > 227 * 1024) return -1;
  cudaError_t e1 = cudaFuncSetAttribute(subsolve_cta_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaError_t e2 = cudaFuncSetAttribute(subsolve_cta_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return (e1 == cudaSuccess && e2 == cudaSuccess) ? 0 : -2;
}

void launch_cocg_first(const DevProblem &p, const double2 *pcloc, cudaStream_t stream) {
  cocg_first_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p, pcloc);
  cocg_first_scalars_kernel<<<1, kRedThreads, 0, stream>>>(p);
}

void launch_cocg_iteration(const DevProblem &p, cudaStream_t stream) {
  cocg_begin_kernel<<<1, 1, 0, stream>>>(p.sc);
  launch_subsolve(p, kModeIter, p.L32 != nullptr, stream);
  cocg_gather_pq_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
  cocg_alpha_kernel<<<1, kRedThreads, 0, stream>>>(p);
  cocg_update_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
  cocg_beta_kernel<<<1, kRedThreads, 0, stream>>>(p);
  cocg_pupdate_kernel<<<p.n_part_blocks, kRedThreads, 0, stream>>>(p);
}

void launch_edge_solution(int64_t ne, const int64_t *edge_src, const double2 *Y, const double2 *V, double2 *x,
                          cudaStream_t stream) {
  if (ne <= 0) return;
  edge_solution_kernel<<<blocks_for(ne, 256), 256, 0, stream>>>(ne, edge_src, Y, V, x);
}

void launch_profile_reset(CocgScalars *sc, cudaStream_t stream) { profile_reset_kernel<<<1, 1, 0, stream>>>(sc); }

void launch_set_status(CocgScalars *sc, double eps, int32_t max_loop, cudaStream_t stream) {
  set_status_kernel<<<1, 1, 0, stream>>>(sc, eps, max_loop);
}

}  // namespace fw
