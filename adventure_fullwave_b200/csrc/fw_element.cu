// Nedelec edge-element matrices of the E-method full-wave formulation.
//
// Restates tet_MakeElement_EM_E (lib/fem/make_elem_em.c:14-400) for the
// current-source case without antenna elements: for each tetrahedron
//   Ae = (nu/omega) RR - (eps omega) SS + i sigma SS,   nu = 7.957747e+05,
// with RR = (rot u, rot v) (tetNedelec_rotrot, lib/fem/tetrahedral.c:344-358)
// and SS = (u, v) (tetNedelec_sideside, :362-422) built from the edge
// lengths (tet_SideLength :27-40), the global edge orientation
// (tetNedelec_Direction :225-263), the opposite-edge vectors
// (tetNedelec_mk :267-281, tetNedelec_XYZ :285-301, tetNedelec_km_mk
// :305-319) and the centroid (tet_Center :80-86).
//
// Every product and sum is evaluated in the reference's order and this file
// is compiled with floating-point contraction off (-fmad=false), so each
// matrix entry is bit-identical to the reference's on the same coordinates:
// the exact-zero pattern of the assembled matrix, and with it the skyline
// profile, then matches the reference's.  Squares are formed as x*x (the
// reference calls pow(x, 2)); both are exact for the dyadic grid spacings of
// the synthetic meshes.
#include <cuda_runtime.h>

#include <cstdint>

namespace fw {

__constant__ int c_tet_n[6][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}};

// 1/mu0 as the reference hard-codes it (make_elem_em.c:37, fullwave.c:674)
constexpr double nu_const_host = 7.957747e+05;
__device__ __forceinline__ double nu_const() { return nu_const_host; }

// Geometry of one tetrahedron as the reference's element routine builds it.
struct TetGeom {
  double D, drr, dss;
  double lsi[6], xi[6], yi[6], zi[6], X[6], Y[6], Z[6], xy[6], yz[6], zx[6], g[3], gxx[6];
  bool bad;
};

// 6 x the signed volume (tet_Volume6, lib/fem/tetrahedral.c:44-61), summed term
// by term in the reference's order
__device__ __forceinline__ double tet_volume6(const double *x, const double *y, const double *z) {
  double D = -x[0] * y[1] * z[2];
  D = D + x[0] * y[1] * z[3];
  D = D + x[0] * y[2] * z[1];
  D = D - x[0] * y[2] * z[3];
  D = D - x[0] * y[3] * z[1];
  D = D + x[0] * y[3] * z[2];
  D = D + x[1] * y[0] * z[2];
  D = D - x[1] * y[0] * z[3];
  D = D - x[1] * y[2] * z[0];
  D = D + x[1] * y[2] * z[3];
  D = D + x[1] * y[3] * z[0];
  D = D - x[1] * y[3] * z[2];
  D = D - x[2] * y[0] * z[1];
  D = D + x[2] * y[0] * z[3];
  D = D + x[2] * y[1] * z[0];
  D = D - x[2] * y[1] * z[3];
  D = D - x[2] * y[3] * z[0];
  D = D + x[2] * y[3] * z[1];
  D = D + x[3] * y[0] * z[1];
  D = D - x[3] * y[0] * z[2];
  D = D - x[3] * y[1] * z[0];
  D = D + x[3] * y[1] * z[2];
  D = D + x[3] * y[2] * z[0];
  D = D - x[3] * y[2] * z[1];
  return D;
}

__device__ __forceinline__ void tet_geometry(const double *x, const double *y, const double *z, TetGeom &G) {
  G.bad = false;
  const double D = tet_volume6(x, y, z);
  if (!(D > 0.0)) G.bad = true;
  G.D = D;
  for (int i = 0; i < 6; i++) {
    const int a = c_tet_n[i][0], b = c_tet_n[i][1];
    const double dx = x[a] - x[b], dy = y[a] - y[b], dz = z[a] - z[b];
    const double l = sqrt(dx * dx + dy * dy + dz * dz);
    // orientation from the first non-zero of (x_b - x_a, y_b - y_a, z_b - z_a)
    int si;
    double pp = x[b] - x[a];
    if (pp > 0.0) {
      si = 1;
    } else if (pp < 0.0) {
      si = -1;
    } else {
      pp = y[b] - y[a];
      if (pp > 0.0) {
        si = 1;
      } else if (pp < 0.0) {
        si = -1;
      } else {
        pp = z[b] - z[a];
        if (pp > 0.0) {
          si = 1;
        } else if (pp < 0.0) {
          si = -1;
        } else {
          si = 0;
          G.bad = true;
        }
      }
    }
    const int p = c_tet_n[i][2], q = c_tet_n[i][3];
    G.xi[i] = x[q] - x[p];
    G.yi[i] = y[q] - y[p];
    G.zi[i] = z[q] - z[p];
    const double d = l * (double)si;
    G.X[i] = d * G.xi[i];
    G.Y[i] = d * G.yi[i];
    G.Z[i] = d * G.zi[i];
    G.xy[i] = x[p] * y[q] - x[q] * y[p];
    G.yz[i] = y[p] * z[q] - y[q] * z[p];
    G.zx[i] = z[p] * x[q] - z[q] * x[p];
    G.lsi[i] = l * (double)si;
  }
  G.g[0] = (x[0] + x[1] + x[2] + x[3]) * 0.25;
  G.g[1] = (y[0] + y[1] + y[2] + y[3]) * 0.25;
  G.g[2] = (z[0] + z[1] + z[2] + z[3]) * 0.25;
  // second moments of the vertex coordinates (sideside, tetrahedral.c:377-398)
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int i = 0; i < 4; i++) {
    sx += x[i];
    sy += y[i];
    sz += z[i];
  }
  G.gxx[0] = sx * sx;
  G.gxx[1] = sy * sy;
  G.gxx[2] = sz * sz;
  G.gxx[3] = sx * sy;
  G.gxx[4] = sy * sz;
  G.gxx[5] = sz * sx;
  for (int i = 0; i < 4; i++) {
    G.gxx[0] += x[i] * x[i];
    G.gxx[1] += y[i] * y[i];
    G.gxx[2] += z[i] * z[i];
    G.gxx[3] += x[i] * y[i];
    G.gxx[4] += y[i] * z[i];
    G.gxx[5] += z[i] * x[i];
  }
  for (int i = 0; i < 6; i++) G.gxx[i] *= 0.05;
  G.drr = 2.0 / (3.0 * D);
  G.dss = 1.0 / (6.0 * D);
}

// (rot u_i, rot u_j) of the reference (tetNedelec_rotrot)
__device__ __forceinline__ double tet_rr(const TetGeom &G, int i, int j) {
  return G.drr * (G.X[i] * G.X[j] + G.Y[i] * G.Y[j] + G.Z[i] * G.Z[j]);
}

// (u_i, u_j) of the reference (tetNedelec_sideside)
__device__ __forceinline__ double tet_ss(const TetGeom &G, int i, int j) {
  const double *zi = G.zi, *yi = G.yi, *xi = G.xi, *yz = G.yz, *zx = G.zx, *xy = G.xy, *gxx = G.gxx, *g = G.g;
  double e = -zi[i] * (-zi[j] * gxx[1] + yi[j] * gxx[4] + yz[j] * g[1]);
  e = e + yi[i] * (-zi[j] * gxx[4] + yi[j] * gxx[2] + yz[j] * g[2]);
  e = e + yz[i] * (-zi[j] * g[1] + yi[j] * g[2] + yz[j]);
  e = e - xi[i] * (-xi[j] * gxx[2] + zi[j] * gxx[5] + zx[j] * g[2]);
  e = e + zi[i] * (-xi[j] * gxx[5] + zi[j] * gxx[0] + zx[j] * g[0]);
  e = e + zx[i] * (-xi[j] * g[2] + zi[j] * g[0] + zx[j]);
  e = e - yi[i] * (-yi[j] * gxx[0] + xi[j] * gxx[3] + xy[j] * g[0]);
  e = e + xi[i] * (-yi[j] * gxx[3] + xi[j] * gxx[1] + xy[j] * g[1]);
  e = e + xy[i] * (-yi[j] * g[0] + xi[j] * g[1] + xy[j]);
  return G.lsi[i] * G.lsi[j] * G.dss * e;
}

__device__ __forceinline__ void load_tet(int t, const int32_t *__restrict__ tet_vertices, const double *__restrict__ crd,
                                         double *x, double *y, double *z) {
  for (int i = 0; i < 4; i++) {
    const int64_t v = tet_vertices[4 * (int64_t)t + i];
    x[i] = crd[3 * v + 0];
    y[i] = crd[3 * v + 1];
    z[i] = crd[3 * v + 2];
  }
}

// One thread per element.  el_order[k] is the global element of element slot
// k; the slot's 6x6 complex matrix is written to out[k*72 .. k*72+71]
// (row-major, interleaved re/im), rows and columns in the reference's edge
// table order 01,02,03,12,13,23.  status[0] is raised to 1 when an element
// has a non-positive volume or an edge with coincident end points (the
// reference aborts with emessage 2050 there, tetrahedral.c:257-258).
__global__ void element_matrices_kernel(int64_t n_el, const int32_t *__restrict__ el_order,
                                        const int32_t *__restrict__ tet_vertices, const double *__restrict__ crd,
                                        const double *__restrict__ el_eps, const double *__restrict__ el_sigma,
                                        double omega, double *__restrict__ out, int32_t *__restrict__ status) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_el) return;
  const int t = el_order[k];
  double x[4], y[4], z[4];
  load_tet(t, tet_vertices, crd, x, y, z);
  const double eps = el_eps[t];
  const double sigma = el_sigma[t];
  TetGeom G;
  tet_geometry(x, y, z, G);
  if (G.bad) atomicMax(status, 1);
  const double nu_omega = nu_const() / omega;
  const double dd = -(eps * omega);
  double *o = out + k * 72;
  for (int i = 0; i < 6; i++) {
    for (int j = 0; j < 6; j++) {
      const double rr = tet_rr(G, i, j);
      const double ss = tet_ss(G, i, j);
      // ae.re = 0 + nu_omega*rr, then += dd*ss; ae.im = 0 + sigma*ss
      double re = 0.0;
      re += nu_omega * rr;
      re += dd * ss;
      double im = 0.0;
      im += sigma * ss;
      o[2 * (i * 6 + j) + 0] = re;
      o[2 * (i * 6 + j) + 1] = im;
    }
  }
}

// Adjoint gradient of J(x) with respect to each design element's
// permittivity eps [F/m] and conductivity sigma [S/m].  With A x = b and
// A lambda = dJ/dx (A = A^T), dJ/dp = -2 Re(lambda_e^T (dA_e/dp) x_e) and,
// from A_e = (nu/omega) RR - (eps omega) SS + i sigma SS
// (make_elem_em.c:227-265), dA_e/deps = -omega SS_e, dA_e/dsigma = i SS_e:
//   dJ/deps = 2 omega Re(s),  dJ/dsigma = 2 Im(s),  s = lambda_e^T SS_e x_e.
// SS_e is recomputed from the coordinates, not stored.
__global__ void adjoint_gradient_kernel(int32_t n_design, const int32_t *__restrict__ design_tets,
                                        const int32_t *__restrict__ tet_vertices,
                                        const int32_t *__restrict__ tet_edges, const double *__restrict__ crd,
                                        double omega, const double2 *__restrict__ x, const double2 *__restrict__ lam,
                                        double *__restrict__ g_eps, double *__restrict__ g_sigma) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_design) return;
  const int t = design_tets[k];
  double vx[4], vy[4], vz[4];
  load_tet(t, tet_vertices, crd, vx, vy, vz);
  TetGeom G;
  tet_geometry(vx, vy, vz, G);
  // element DOFs in the edge table order: file mid-node slots 0,1,2,3,5,4
  const int file_slot[6] = {0, 1, 2, 3, 5, 4};
  double2 xe[6], le[6];
  for (int i = 0; i < 6; i++) {
    const int e = tet_edges[6 * (int64_t)t + file_slot[i]];
    xe[i] = x[e];
    le[i] = lam[e];
  }
  double sr = 0.0, si = 0.0;
  for (int i = 0; i < 6; i++) {
    double ar = 0.0, ai = 0.0;
    for (int j = 0; j < 6; j++) {
      const double ss = tet_ss(G, i, j);
      ar += ss * xe[j].x;
      ai += ss * xe[j].y;
    }
    sr += le[i].x * ar - le[i].y * ai;
    si += le[i].x * ai + le[i].y * ar;
  }
  g_eps[k] = 2.0 * omega * sr;
  g_sigma[k] = 2.0 * si;
}

// Element results of the post step, HDDM_post_em_E
// (main/fullwave/fullwave.c:639-763), one thread per element: the element's
// six edge values are first scaled by nu/omega (nu = 7.957747e+05 when the
// element's flag is in the Permittivity list, else 0; fullwave.c:672-677,722)
// and the scaled values feed all three results:
//   B  = (2/D)     sum_i i xe_i (X_i, Y_i, Z_i)        (rot E times nu/omega)
//   E  = (2/D)     sum_i xe_i (Fx_i, Fy_i, Fz_i)       (tetNedelec_Fxyz at the centroid)
//   Je = (sigma/D) sum_i xe_i (Fx_i, Fy_i, Fz_i)
// Same operation order as the reference (contraction off), so the results
// are bit-identical to its own on the same edge values.  Outputs are 3
// complex per element in global element order; a null output is skipped.
// status[0] (if given) is raised to 1 for a degenerate element, where the
// reference stops (tetrahedral.c:257-258).
// One element of the post step: r[0..2] = B, r[3..5] = E, r[6..8] = Je.
// Returns true for a degenerate element.
__device__ __forceinline__ bool post_element(int64_t t, const int32_t *__restrict__ tet_vertices,
                                             const int32_t *__restrict__ tet_edges, const double *__restrict__ crd,
                                             const uint8_t *__restrict__ el_has_nu,
                                             const double *__restrict__ el_sigma, double s_nu, double s_zero,
                                             const double2 *__restrict__ xedge, double2 *r) {
  const int4 tv = __ldg(reinterpret_cast<const int4 *>(tet_vertices) + t);
  const int2 *te2 = reinterpret_cast<const int2 *>(tet_edges + 6 * t);
  const int2 e01 = __ldg(te2), e23 = __ldg(te2 + 1), e45 = __ldg(te2 + 2);
  // edge-table order 01,02,03,12,13,23 from file slots 0,1,2,3,5,4
  const int eid[6] = {e01.x, e01.y, e23.x, e23.y, e45.y, e45.x};
  double2 xe[6];
#pragma unroll
  for (int i = 0; i < 6; i++) xe[i] = __ldg(xedge + eid[i]);
  const int vid[4] = {tv.x, tv.y, tv.z, tv.w};
  double vx[4], vy[4], vz[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    vx[i] = __ldg(crd + 3 * (int64_t)vid[i]);
    vy[i] = __ldg(crd + 3 * (int64_t)vid[i] + 1);
    vz[i] = __ldg(crd + 3 * (int64_t)vid[i] + 2);
  }
  // nu/omega (fullwave.c:722), the same quotient for every element of a kind
  const double s = el_has_nu[t] ? s_nu : s_zero;
  const double sigma = el_sigma[t];
  // one pass over the six edges: the element routine's per-edge quantities
  // (tet_SideLength, tetNedelec_Direction, _mk, _XYZ, _km_mk, _Fxyz) are
  // formed and used at once, each sum still taken in edge order
  constexpr int kN[6][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}};
  const double *x = vx, *y = vy, *z = vz;
  double D = -x[0] * y[1] * z[2];
  D = D + x[0] * y[1] * z[3];
  D = D + x[0] * y[2] * z[1];
  D = D - x[0] * y[2] * z[3];
  D = D - x[0] * y[3] * z[1];
  D = D + x[0] * y[3] * z[2];
  D = D + x[1] * y[0] * z[2];
  D = D - x[1] * y[0] * z[3];
  D = D - x[1] * y[2] * z[0];
  D = D + x[1] * y[2] * z[3];
  D = D + x[1] * y[3] * z[0];
  D = D - x[1] * y[3] * z[2];
  D = D - x[2] * y[0] * z[1];
  D = D + x[2] * y[0] * z[3];
  D = D + x[2] * y[1] * z[0];
  D = D - x[2] * y[1] * z[3];
  D = D - x[2] * y[3] * z[0];
  D = D + x[2] * y[3] * z[1];
  D = D + x[3] * y[0] * z[1];
  D = D - x[3] * y[0] * z[2];
  D = D - x[3] * y[1] * z[0];
  D = D + x[3] * y[1] * z[2];
  D = D + x[3] * y[2] * z[0];
  D = D - x[3] * y[2] * z[1];
  bool bad = !(D > 0.0);
  double g[3];
  g[0] = (x[0] + x[1] + x[2] + x[3]) * 0.25;
  g[1] = (y[0] + y[1] + y[2] + y[3]) * 0.25;
  g[2] = (z[0] + z[1] + z[2] + z[3]) * 0.25;
  double2 rb[3], et[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    rb[k] = make_double2(0.0, 0.0);
    et[k] = make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int i = 0; i < 6; i++) {
    const int a = kN[i][0], b = kN[i][1], p = kN[i][2], q = kN[i][3];
    const double dx = x[a] - x[b], dy = y[a] - y[b], dz = z[a] - z[b];
    const double l = sqrt(dx * dx + dy * dy + dz * dz);
    // orientation from the first non-zero of (x_b - x_a, y_b - y_a, z_b - z_a)
    int si = 0;
    const double px = x[b] - x[a], py = y[b] - y[a], pz = z[b] - z[a];
    if (px > 0.0) si = 1;
    else if (px < 0.0) si = -1;
    else if (py > 0.0) si = 1;
    else if (py < 0.0) si = -1;
    else if (pz > 0.0) si = 1;
    else if (pz < 0.0) si = -1;
    else bad = true;
    const double xi = x[q] - x[p], yi = y[q] - y[p], zi = z[q] - z[p];
    const double d = l * (double)si;
    const double X = d * xi, Y = d * yi, Z = d * zi;
    const double xy = x[p] * y[q] - x[q] * y[p];
    const double yz = y[p] * z[q] - y[q] * z[p];
    const double zx = z[p] * x[q] - z[q] * x[p];
    const double fx = d * (yz - zi * g[1] + yi * g[2]);
    const double fy = d * (zx - xi * g[2] + zi * g[0]);
    const double fz = d * (xy - yi * g[0] + xi * g[1]);
    const double2 v = make_double2(xe[i].x * s, xe[i].y * s);
    // v * i, evaluated as the full complex product with (0, 1)
    const double ccr = v.x * 0.0 - v.y * 1.0;
    const double cci = v.y * 0.0 + v.x * 1.0;
    rb[0] = make_double2(rb[0].x + ccr * X, rb[0].y + cci * X);
    rb[1] = make_double2(rb[1].x + ccr * Y, rb[1].y + cci * Y);
    rb[2] = make_double2(rb[2].x + ccr * Z, rb[2].y + cci * Z);
    et[0] = make_double2(et[0].x + v.x * fx, et[0].y + v.y * fx);
    et[1] = make_double2(et[1].x + v.x * fy, et[1].y + v.y * fy);
    et[2] = make_double2(et[2].x + v.x * fz, et[2].y + v.y * fz);
  }
  const double dd = 2.0 / D;
  const double ds = sigma / D;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    r[k] = make_double2(rb[k].x * dd, rb[k].y * dd);
    r[3 + k] = make_double2(et[k].x * dd, et[k].y * dd);
    r[6 + k] = make_double2(et[k].x * ds, et[k].y * ds);
  }
  return bad;
}

constexpr int kPostThreads = 128;

__global__ void __launch_bounds__(kPostThreads, 4) post_em_E_kernel(int64_t nt, const int32_t *__restrict__ tet_vertices,
                                                                 const int32_t *__restrict__ tet_edges,
                                                                 const double *__restrict__ crd,
                                                                 const uint8_t *__restrict__ el_has_nu,
                                                                 const double *__restrict__ el_sigma, double s_nu,
                                                                 double s_zero, const double2 *__restrict__ xedge,
                                                                 double2 *__restrict__ B, double2 *__restrict__ E,
                                                                 double2 *__restrict__ Je,
                                                                 int32_t *__restrict__ status) {
  // results staged per block so that the stores are contiguous
  __shared__ double2 stage[3][kPostThreads * 3];
  const int64_t t0 = (int64_t)blockIdx.x * kPostThreads;
  const int64_t t = t0 + threadIdx.x;
  const int n_here = nt - t0 < kPostThreads ? (int)(nt - t0) : kPostThreads;
  if (t < nt) {
    double2 r[9];
    if (post_element(t, tet_vertices, tet_edges, crd, el_has_nu, el_sigma, s_nu, s_zero, xedge, r) && status)
      atomicMax(status, 1);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      stage[0][3 * threadIdx.x + k] = r[k];
      stage[1][3 * threadIdx.x + k] = r[3 + k];
      stage[2][3 * threadIdx.x + k] = r[6 + k];
    }
  }
  __syncthreads();
  double2 *outs[3] = {B, E, Je};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!outs[k]) continue;
    double2 *o = outs[k] + 3 * t0;
    for (int j = threadIdx.x; j < 3 * n_here; j += kPostThreads) o[j] = stage[k][j];
  }
}

void launch_post_em_E(int64_t nt, const int32_t *tet_vertices, const int32_t *tet_edges, const double *crd,
                      const uint8_t *el_has_nu, const double *el_sigma, double omega, const double2 *x, double2 *B,
                      double2 *E, double2 *Je, int32_t *status, cudaStream_t stream) {
  if (nt <= 0) return;
  const int64_t blocks = (nt + kPostThreads - 1) / kPostThreads;
  // nu/omega divided once here, in double as the reference does per element
  const double s_nu = nu_const_host / omega;
  const double s_zero = 0.0 / omega;
  post_em_E_kernel<<<(unsigned)blocks, kPostThreads, 0, stream>>>(nt, tet_vertices, tet_edges, crd, el_has_nu,
                                                                   el_sigma, s_nu, s_zero, x, B, E, Je, status);
}

// Element right-hand side of tet_MakeElement_EM_E (lib/fem/make_elem_em.c:66-330),
// one thread per element slot, 6 complex per slot in the edge-table order.
//   n_gaps > 0 (volt.dat dg > 0): DGe_j = (0, dV_k) for the last gap box k
//     (inclusive) holding vertex j; if any vertex is held,
//     be_i = (sigma omega) sum_j DGe_j gs_ij, gs = tetNedelec_gradside
//     (tetrahedral.c:645-661); otherwise be = 0.
//   n_gaps = 0 (current input): for an element of an antenna flag,
//     be = 0 + (be_JoA - 0), be_JoA = tetNedelec_JoA_Complex
//     (tetrahedral.c:794-858) of Joe_j = (-Jo, -Jor) at its vertices; other
//     elements get be = 0.
// Contraction is off for this file, so be is bit-identical to the reference's.
__global__ void __launch_bounds__(128) element_rhs_kernel(int64_t n_el, const int32_t *__restrict__ el_order,
                                                          const int32_t *__restrict__ tet_vertices,
                                                          const double *__restrict__ crd,
                                                          const double *__restrict__ el_sigma, double omega,
                                                          int32_t n_gaps, const double *__restrict__ gap,
                                                          const int32_t *__restrict__ el_antenna,
                                                          const double *__restrict__ Jo,
                                                          const double *__restrict__ Jor, int64_t n_vertices,
                                                          double2 *__restrict__ be) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_el) return;
  const int t = el_order[k];
  double2 out[6];
#pragma unroll
  for (int i = 0; i < 6; i++) out[i] = make_double2(0.0, 0.0);
  const int ant = n_gaps > 0 ? -1 : el_antenna[t];
  double x[4], y[4], z[4];
  load_tet(t, tet_vertices, crd, x, y, z);
  double2 dge[4];
  bool dvn = false;
  if (n_gaps > 0) {
#pragma unroll
    for (int j = 0; j < 4; j++) dge[j] = make_double2(0.0, 0.0);
    for (int g = 0; g < n_gaps; g++) {
      const double *bx = gap + 7 * g;
#pragma unroll
      for (int j = 0; j < 4; j++)
        if ((bx[0] <= x[j] && x[j] <= bx[1]) && (bx[2] <= y[j] && y[j] <= bx[3]) && (bx[4] <= z[j] && z[j] <= bx[5])) {
          dge[j] = make_double2(0.0, bx[6]);
          dvn = true;
        }
    }
  }
  if (dvn || ant >= 0) {
    constexpr int kM[4][4] = {{0, 1, 2, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}, {3, 1, 0, 2}};
    constexpr int kN[6][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}};
    double b[4], c[4], d[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {  // tet_simple_b, _c, _d (tetrahedral.c:121-195)
      const int ii = kM[i][1], jj = kM[i][2], kk = kM[i][3];
      b[i] = -1.0 * (y[ii] * (z[jj] - z[kk]) + y[jj] * (z[kk] - z[ii]) + y[kk] * (z[ii] - z[jj]));
      c[i] = -1.0 * (z[ii] * (x[jj] - x[kk]) + z[jj] * (x[kk] - x[ii]) + z[kk] * (x[ii] - x[jj]));
      d[i] = -1.0 * (x[ii] * (y[jj] - y[kk]) + x[jj] * (y[kk] - y[ii]) + x[kk] * (y[ii] - y[jj]));
    }
    if (dvn) {
      TetGeom G;
      tet_geometry(x, y, z, G);
      const double dd = 1.0 / (6.0 * G.D);
      const double so = el_sigma[t] * omega;
#pragma unroll
      for (int i = 0; i < 6; i++) {
        // F at the centroid (tetNedelec_Fxyz, tetrahedral.c:323-340)
        const double fx = G.lsi[i] * (G.yz[i] - G.zi[i] * G.g[1] + G.yi[i] * G.g[2]);
        const double fy = G.lsi[i] * (G.zx[i] - G.xi[i] * G.g[2] + G.zi[i] * G.g[0]);
        const double fz = G.lsi[i] * (G.xy[i] - G.yi[i] * G.g[0] + G.xi[i] * G.g[1]);
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double gs = dd * (fx * b[j] + fy * c[j] + fz * d[j]);
          acc = make_double2(acc.x + dge[j].x * gs, acc.y + dge[j].y * gs);
        }
        out[i] = make_double2(acc.x * so, acc.y * so);
      }
    } else {
      const double *jo = Jo + (int64_t)ant * 3 * n_vertices;
      const double *jr = Jor + (int64_t)ant * 3 * n_vertices;
      double2 joe[4][3];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int64_t v = tet_vertices[4 * (int64_t)t + j];
#pragma unroll
        for (int cc = 0; cc < 3; cc++) joe[j][cc] = make_double2(-jo[3 * v + cc], -jr[3 * v + cc]);
      }
      constexpr double d0[6][4] = {{2.0, 1.0, 1.0, 1.0}, {2.0, 1.0, 1.0, 1.0}, {2.0, 1.0, 1.0, 1.0},
                                   {1.0, 2.0, 1.0, 1.0}, {1.0, 2.0, 1.0, 1.0}, {1.0, 1.0, 2.0, 1.0}};
      constexpr double d1[6][4] = {{-1.0, -2.0, -1.0, -1.0}, {-1.0, -1.0, -2.0, -1.0}, {-1.0, -1.0, -1.0, -2.0},
                                   {-1.0, -1.0, -2.0, -1.0}, {-1.0, -1.0, -1.0, -2.0}, {-1.0, -1.0, -1.0, -2.0}};
#pragma unroll
      for (int i = 0; i < 6; i++) {
        const int a = kN[i][0], bb = kN[i][1];
        const double dx = x[a] - x[bb], dy = y[a] - y[bb], dz = z[a] - z[bb];
        const double l = sqrt(dx * dx + dy * dy + dz * dz);
        int si = 0;
        const double px = x[bb] - x[a], py = y[bb] - y[a], pz = z[bb] - z[a];
        if (px > 0.0) si = 1;
        else if (px < 0.0) si = -1;
        else if (py > 0.0) si = 1;
        else if (py < 0.0) si = -1;
        else if (pz > 0.0) si = 1;
        else if (pz < 0.0) si = -1;
        const double dd = (double)si * l / 120.0;
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double w = dd * (d0[i][j] * b[bb] + d1[i][j] * b[a]);
          acc = make_double2(acc.x + joe[j][0].x * w, acc.y + joe[j][0].y * w);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double w = dd * (d0[i][j] * c[bb] + d1[i][j] * c[a]);
          acc = make_double2(acc.x + joe[j][1].x * w, acc.y + joe[j][1].y * w);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double w = dd * (d0[i][j] * d[bb] + d1[i][j] * d[a]);
          acc = make_double2(acc.x + joe[j][2].x * w, acc.y + joe[j][2].y * w);
        }
        // be = be + (be_JoA - be_gs); be_gs = sum of 0 * gs = +0 (make_elem_em.c:302-314)
        out[i] = make_double2(0.0 + (acc.x - 0.0), 0.0 + (acc.y - 0.0));
      }
    }
  }
  double2 *o = be + 6 * k;
#pragma unroll
  for (int i = 0; i < 6; i++) o[i] = out[i];
}

// TMP_B of every subdomain: for each local DOF the element contributions in
// element order (SetFe, aij_matrix_func.h:327-338), then the edge source.
__global__ void rhs_gather_kernel(int64_t n_dof, const int64_t *__restrict__ ptr, const int32_t *__restrict__ src,
                                  const double2 *__restrict__ be, const double2 *__restrict__ b_edge,
                                  double2 *__restrict__ b) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_dof) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t q = ptr[r]; q < ptr[r + 1]; q++) {
    const double2 v = be[src[q]];
    acc = make_double2(acc.x + v.x, acc.y + v.y);
  }
  const double2 e = b_edge[r];
  b[r] = make_double2(acc.x + e.x, acc.y + e.y);
}

// interior and interface right-hand sides from TMP_B
__global__ void rhs_split_kernel(int64_t n, const int64_t *__restrict__ pos, const double2 *__restrict__ b,
                                 double2 *__restrict__ f) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) f[k] = b[pos[k]];
}

void launch_element_rhs(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                        const double *el_sigma, double omega, int32_t n_gaps, const double *gap,
                        const int32_t *el_antenna, const double *Jo, const double *Jor, int64_t n_vertices,
                        double2 *be, cudaStream_t stream) {
  if (n_el <= 0) return;
  element_rhs_kernel<<<(unsigned)((n_el + 127) / 128), 128, 0, stream>>>(
      n_el, el_order, tet_vertices, crd, el_sigma, omega, n_gaps, gap, el_antenna, Jo, Jor, n_vertices, be);
}

void launch_rhs_gather(int64_t n_dof, const int64_t *ptr, const int32_t *src, const double2 *be,
                       const double2 *b_edge, double2 *b, cudaStream_t stream) {
  if (n_dof <= 0) return;
  rhs_gather_kernel<<<(unsigned)((n_dof + 255) / 256), 256, 0, stream>>>(n_dof, ptr, src, be, b_edge, b);
}

void launch_rhs_split(int64_t n, const int64_t *pos, const double2 *b, double2 *f, cudaStream_t stream) {
  if (n <= 0) return;
  rhs_split_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(n, pos, b, f);
}

void launch_element_matrices(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                             const double *el_eps, const double *el_sigma, double omega, double *out,
                             int32_t *status, cudaStream_t stream) {
  if (n_el <= 0) return;
  const int threads = 128;
  const int64_t blocks = (n_el + threads - 1) / threads;
  element_matrices_kernel<<<(unsigned)blocks, threads, 0, stream>>>(n_el, el_order, tet_vertices, crd, el_eps,
                                                                     el_sigma, omega, out, status);
}

void launch_adjoint_gradient(int32_t n_design, const int32_t *design_tets, const int32_t *tet_vertices,
                             const int32_t *tet_edges, const double *crd, double omega, const double2 *x,
                             const double2 *lam, double *g_eps, double *g_sigma, cudaStream_t stream) {
  if (n_design <= 0) return;
  adjoint_gradient_kernel<<<(n_design + 127) / 128, 128, 0, stream>>>(n_design, design_tets, tet_vertices, tet_edges,
                                                                      crd, omega, x, lam, g_eps, g_sigma);
}


// ---------------------------------------------------------------------------
// The correction-Jo problem of an antenna (tet_MakeElement_correct_Jo,
// lib/fem/make_elem.c:10-66): conventional linear tetrahedra on the
// antenna's elements, element matrix (grad N_i, grad N_j)
// (tet_simple_gradgrad, lib/fem/tetrahedral.c:188-202) and element vector
// (J, grad N_i) of the vertex currents J (tet_simple_be_apgrad :206-220),
// with the determinants b, c, d of tet_simple_b/c/d (:122-184) over the
// vertex table tet_m (tetrahedral.h:14-17).  Reference operation order,
// contraction off, as for the edge elements.
__constant__ int c_tet_m[4][4] = {{0, 1, 2, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}, {3, 1, 0, 2}};

__device__ __forceinline__ void tet_simple_bcd(const double *x, const double *y, const double *z, double *b, double *c,
                                               double *d) {
  for (int i = 0; i < 4; i++) {
    const int ii = c_tet_m[i][1], jj = c_tet_m[i][2], kk = c_tet_m[i][3];
    b[i] = -1.0 * (y[ii] * (z[jj] - z[kk]) + y[jj] * (z[kk] - z[ii]) + y[kk] * (z[ii] - z[jj]));
    c[i] = -1.0 * (z[ii] * (x[jj] - x[kk]) + z[jj] * (x[kk] - x[ii]) + z[kk] * (x[ii] - x[jj]));
    d[i] = -1.0 * (x[ii] * (y[jj] - y[kk]) + x[jj] * (y[kk] - y[ii]) + x[kk] * (y[ii] - y[jj]));
  }
}

// One thread per element slot k (el_order[k] a global element): its 4x4 real
// matrix is stored in the 6x6 complex slot layout of the edge elements,
// entry (i, j) at out[k*72 + 2*(i*6+j)], imaginary parts and the unused
// rows and columns zero.  status[0] is raised for a non-positive volume.
__global__ void cojo_element_matrices_kernel(int64_t n_el, const int32_t *__restrict__ el_order,
                                             const int32_t *__restrict__ tet_vertices,
                                             const double *__restrict__ crd, double *__restrict__ out,
                                             int32_t *__restrict__ status) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_el) return;
  double x[4], y[4], z[4], b[4], c[4], d[4];
  load_tet(el_order[k], tet_vertices, crd, x, y, z);
  const double D = tet_volume6(x, y, z);
  if (!(D > 0.0)) atomicMax(status, 1);
  tet_simple_bcd(x, y, z, b, c, d);
  const double dd = 1.0 / (6.0 * D);
  double *o = out + k * 72;
  for (int q = 0; q < 72; q++) o[q] = 0.0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) o[2 * (i * 6 + j)] = (b[i] * b[j] + c[i] * c[j] + d[i] * d[j]) * dd;
}

// One thread per element slot: be_i = sum_j (b_i J_j,x + c_i J_j,y + d_i J_j,z) / 24
// with J (3 per global vertex) the pass's currents, written as 6 complex
// per slot (entries 0..3, imaginary parts and entries 4, 5 zero).
__global__ void cojo_element_rhs_kernel(int64_t n_el, const int32_t *__restrict__ el_order,
                                        const int32_t *__restrict__ tet_vertices, const double *__restrict__ crd,
                                        const double *__restrict__ J, double2 *__restrict__ be) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_el) return;
  const int t = el_order[k];
  double x[4], y[4], z[4], b[4], c[4], d[4], u[4][3];
  load_tet(t, tet_vertices, crd, x, y, z);
  tet_simple_bcd(x, y, z, b, c, d);
  for (int i = 0; i < 4; i++) {
    const int64_t v = tet_vertices[4 * (int64_t)t + i];
    for (int j = 0; j < 3; j++) u[i][j] = J[3 * v + j];
  }
  const double dd = 1.0 / 24.0;
  for (int i = 0; i < 4; i++) {
    double ag = 0.0;
    for (int j = 0; j < 4; j++) ag += (b[i] * u[j][0] + c[i] * u[j][1] + d[i] * u[j][2]) * dd;
    be[6 * k + i] = make_double2(ag, 0.0);
  }
  be[6 * k + 4] = make_double2(0.0, 0.0);
  be[6 * k + 5] = make_double2(0.0, 0.0);
}

void launch_cojo_element_matrices(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices,
                                  const double *crd, double *out, int32_t *status, cudaStream_t stream) {
  if (n_el <= 0) return;
  cojo_element_matrices_kernel<<<(unsigned)((n_el + 127) / 128), 128, 0, stream>>>(n_el, el_order, tet_vertices, crd,
                                                                                   out, status);
}

void launch_cojo_element_rhs(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                             const double *J, double2 *be, cudaStream_t stream) {
  if (n_el <= 0) return;
  cojo_element_rhs_kernel<<<(unsigned)((n_el + 127) / 128), 128, 0, stream>>>(n_el, el_order, tet_vertices, crd, J,
                                                                              be);
}

}  // namespace fw
