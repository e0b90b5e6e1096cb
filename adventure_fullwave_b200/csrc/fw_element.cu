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

// 1/mu0 as the reference hard-codes it (make_elem_em.c:37)
__device__ __forceinline__ double nu_const() { return 7.957747e+05; }

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
  for (int i = 0; i < 4; i++) {
    const int64_t v = tet_vertices[4 * (int64_t)t + i];
    x[i] = crd[3 * v + 0];
    y[i] = crd[3 * v + 1];
    z[i] = crd[3 * v + 2];
  }
  const double eps = el_eps[t];
  const double sigma = el_sigma[t];

  // 6 x volume, summed term by term in the reference's order
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
  if (!(D > 0.0)) atomicMax(status, 1);

  double l[6], lsi[6], xi[6], yi[6], zi[6], X[6], Y[6], Z[6], xy[6], yz[6], zx[6];
  int si[6];
  for (int i = 0; i < 6; i++) {
    const int a = c_tet_n[i][0], b = c_tet_n[i][1];
    const double dx = x[a] - x[b], dy = y[a] - y[b], dz = z[a] - z[b];
    l[i] = sqrt(dx * dx + dy * dy + dz * dz);
    // orientation from the first non-zero of (x_b - x_a, y_b - y_a, z_b - z_a)
    double pp = x[b] - x[a];
    if (pp > 0.0) {
      si[i] = 1;
    } else if (pp < 0.0) {
      si[i] = -1;
    } else {
      pp = y[b] - y[a];
      if (pp > 0.0) {
        si[i] = 1;
      } else if (pp < 0.0) {
        si[i] = -1;
      } else {
        pp = z[b] - z[a];
        if (pp > 0.0) {
          si[i] = 1;
        } else if (pp < 0.0) {
          si[i] = -1;
        } else {
          si[i] = 0;
          atomicMax(status, 1);
        }
      }
    }
    const int p = c_tet_n[i][2], q = c_tet_n[i][3];
    xi[i] = x[q] - x[p];
    yi[i] = y[q] - y[p];
    zi[i] = z[q] - z[p];
    const double d = l[i] * (double)si[i];
    X[i] = d * xi[i];
    Y[i] = d * yi[i];
    Z[i] = d * zi[i];
    xy[i] = x[p] * y[q] - x[q] * y[p];
    yz[i] = y[p] * z[q] - y[q] * z[p];
    zx[i] = z[p] * x[q] - z[q] * x[p];
    lsi[i] = l[i] * (double)si[i];
  }
  double g[3];
  g[0] = (x[0] + x[1] + x[2] + x[3]) * 0.25;
  g[1] = (y[0] + y[1] + y[2] + y[3]) * 0.25;
  g[2] = (z[0] + z[1] + z[2] + z[3]) * 0.25;

  // second moments of the vertex coordinates (sideside, tetrahedral.c:377-398)
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int i = 0; i < 4; i++) {
    sx += x[i];
    sy += y[i];
    sz += z[i];
  }
  double gxx[6];
  gxx[0] = sx * sx;
  gxx[1] = sy * sy;
  gxx[2] = sz * sz;
  gxx[3] = sx * sy;
  gxx[4] = sy * sz;
  gxx[5] = sz * sx;
  for (int i = 0; i < 4; i++) {
    gxx[0] += x[i] * x[i];
    gxx[1] += y[i] * y[i];
    gxx[2] += z[i] * z[i];
    gxx[3] += x[i] * y[i];
    gxx[4] += y[i] * z[i];
    gxx[5] += z[i] * x[i];
  }
  for (int i = 0; i < 6; i++) gxx[i] *= 0.05;

  const double drr = 2.0 / (3.0 * D);
  const double dss = 1.0 / (6.0 * D);
  const double nu_omega = nu_const() / omega;
  const double dd = -(eps * omega);
  double *o = out + k * 72;
  for (int i = 0; i < 6; i++) {
    for (int j = 0; j < 6; j++) {
      const double rr = drr * (X[i] * X[j] + Y[i] * Y[j] + Z[i] * Z[j]);
      double e = -zi[i] * (-zi[j] * gxx[1] + yi[j] * gxx[4] + yz[j] * g[1]);
      e = e + yi[i] * (-zi[j] * gxx[4] + yi[j] * gxx[2] + yz[j] * g[2]);
      e = e + yz[i] * (-zi[j] * g[1] + yi[j] * g[2] + yz[j]);
      e = e - xi[i] * (-xi[j] * gxx[2] + zi[j] * gxx[5] + zx[j] * g[2]);
      e = e + zi[i] * (-xi[j] * gxx[5] + zi[j] * gxx[0] + zx[j] * g[0]);
      e = e + zx[i] * (-xi[j] * g[2] + zi[j] * g[0] + zx[j]);
      e = e - yi[i] * (-yi[j] * gxx[0] + xi[j] * gxx[3] + xy[j] * g[0]);
      e = e + xi[i] * (-yi[j] * gxx[3] + xi[j] * gxx[1] + xy[j] * g[1]);
      e = e + xy[i] * (-yi[j] * g[0] + xi[j] * g[1] + xy[j]);
      const double ss = lsi[i] * lsi[j] * dss * e;
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

void launch_element_matrices(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                             const double *el_eps, const double *el_sigma, double omega, double *out,
                             int32_t *status, cudaStream_t stream) {
  if (n_el <= 0) return;
  const int threads = 128;
  const int64_t blocks = (n_el + threads - 1) / threads;
  element_matrices_kernel<<<(unsigned)blocks, threads, 0, stream>>>(n_el, el_order, tet_vertices, crd, el_eps,
                                                                     el_sigma, omega, out, status);
}

}  // namespace fw
