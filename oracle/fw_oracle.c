/*
 * CPU restatement of the reference's full-wave HDDM hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the CUDA path is checked
 * against (tests/, __graft_entry__.smoke(), bench.py's CPU baseline).  The
 * product never links or calls it.  It restates, in the reference's own
 * operation order so that results agree with the reference bit for bit:
 *
 *   orc_element_matrix   tet_MakeElement_EM_E        lib/fem/make_elem_em.c:14-400
 *                        (tetrahedral.c:27-61,80-86,225-422)
 *   assemble_sub         HDDM_make_TMP_AIJ_em_E      main/fullwave/fullwave.c:221-259
 *                        mymt_CS_AIJ_SetAe/DeleteZero lib/mymt_aij_solver/aij_matrix_func.h:260-391
 *   set_bc               __MYMT_AIJ_SETBC__          aij_matrix_func.h:60-136
 *   skyline_*            advlas_skyline.c:12-167
 *   mxv                  __MYMT_AIJ_MAIJMXV_TMP_AIJ__ aij_matrix_func.h:624-658
 *   orc_hddm             s-mode HDDM loop + COCG     lib/hddm/hddm_solver.h:59-183,461-693,
 *                        hddm_solver_s.h:7-424, hddm_solver_sp.h, hddm_pc.h:52-137
 *   orc_element_rhs      tet_MakeElement_EM_E be     lib/fem/make_elem_em.c:66-330
 *                        (tetrahedral.c:121-195,645-661,794-858)
 *   orc_post_em_E        HDDM_post_em_E              main/fullwave/fullwave.c:639-763
 *                        (tetrahedral.c:27-61,80-86,225-340)
 *
 * Inputs are the per-subdomain arrays make_PartMesh_FW leaves in DomMesh
 * (local nop after the slot-8/9 swap, local vertex coordinates, the
 * Dirichlet list with the interface DOFs last, inbc with nfid and ln_part),
 * for one part.  The current source enters as each subdomain's assembled
 * right-hand side.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cpx;

static const int TET_N[6][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}};
#define NEARLY_ZERO 1.0e-60

/* complex helpers of lib/std/complex_adv.c */
static cpx c_add(cpx a, cpx b) { return (cpx){a.re + b.re, a.im + b.im}; }
static cpx c_sub(cpx a, cpx b) { return (cpx){a.re - b.re, a.im - b.im}; }
static cpx c_mul(cpx a, cpx b) { return (cpx){a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im}; }
static cpx c_recip(cpx a) {
  double d = 1.0 / (a.re * a.re + a.im * a.im);
  return (cpx){a.re * d, -(a.im * d)};
}
static cpx c_div(cpx a, cpx b) { return c_mul(a, c_recip(b)); }
static double c_abs(cpx a) { return sqrt(a.re * a.re + a.im * a.im); }
static int c_iszero(cpx a) { return a.re == 0.0 && a.im == 0.0; }

/* ------------------------------------------------------------------------ */
/* element matrix                                                           */

int orc_element_matrix(const double *xyz, double epsilon, double sigma, double omega, double *ae) {
  const double *x = xyz, *y = xyz + 4, *z = xyz + 8;
  double l[6], si_d[6], xi[6], yi[6], zi[6], X[6], Y[6], Z[6], xy[6], yz[6], zx[6], g[3], lsi[6];
  int si[6];
  double D = -x[0] * y[1] * z[2] + x[0] * y[1] * z[3] + x[0] * y[2] * z[1] - x[0] * y[2] * z[3] -
             x[0] * y[3] * z[1] + x[0] * y[3] * z[2] + x[1] * y[0] * z[2] - x[1] * y[0] * z[3] -
             x[1] * y[2] * z[0] + x[1] * y[2] * z[3] + x[1] * y[3] * z[0] - x[1] * y[3] * z[2] -
             x[2] * y[0] * z[1] + x[2] * y[0] * z[3] + x[2] * y[1] * z[0] - x[2] * y[1] * z[3] -
             x[2] * y[3] * z[0] + x[2] * y[3] * z[1] + x[3] * y[0] * z[1] - x[3] * y[0] * z[2] -
             x[3] * y[1] * z[0] + x[3] * y[1] * z[2] + x[3] * y[2] * z[0] - x[3] * y[2] * z[1];
  int bad = !(D > 0.0);
  for (int i = 0; i < 6; i++) {
    int a = TET_N[i][0], b = TET_N[i][1];
    l[i] = sqrt(pow(x[a] - x[b], 2) + pow(y[a] - y[b], 2) + pow(z[a] - z[b], 2));
    double pp = x[b] - x[a];
    if (pp > 0.0)
      si[i] = 1;
    else if (pp < 0.0)
      si[i] = -1;
    else {
      pp = y[b] - y[a];
      if (pp > 0.0)
        si[i] = 1;
      else if (pp < 0.0)
        si[i] = -1;
      else {
        pp = z[b] - z[a];
        if (pp > 0.0)
          si[i] = 1;
        else if (pp < 0.0)
          si[i] = -1;
        else {
          si[i] = 0;
          bad = 1;
        }
      }
    }
    int p = TET_N[i][2], q = TET_N[i][3];
    xi[i] = x[q] - x[p];
    yi[i] = y[q] - y[p];
    zi[i] = z[q] - z[p];
    si_d[i] = l[i] * (double)si[i];
    X[i] = si_d[i] * xi[i];
    Y[i] = si_d[i] * yi[i];
    Z[i] = si_d[i] * zi[i];
    xy[i] = x[p] * y[q] - x[q] * y[p];
    yz[i] = y[p] * z[q] - y[q] * z[p];
    zx[i] = z[p] * x[q] - z[q] * x[p];
    lsi[i] = l[i] * (double)si[i];
  }
  g[0] = (x[0] + x[1] + x[2] + x[3]) * 0.25;
  g[1] = (y[0] + y[1] + y[2] + y[3]) * 0.25;
  g[2] = (z[0] + z[1] + z[2] + z[3]) * 0.25;
  double dx = 0.0, dy = 0.0, dz = 0.0, gxx[6];
  for (int i = 0; i < 4; i++) {
    dx += x[i];
    dy += y[i];
    dz += z[i];
  }
  gxx[0] = dx * dx;
  gxx[1] = dy * dy;
  gxx[2] = dz * dz;
  gxx[3] = dx * dy;
  gxx[4] = dy * dz;
  gxx[5] = dz * dx;
  for (int i = 0; i < 4; i++) {
    gxx[0] += x[i] * x[i];
    gxx[1] += y[i] * y[i];
    gxx[2] += z[i] * z[i];
    gxx[3] += x[i] * y[i];
    gxx[4] += y[i] * z[i];
    gxx[5] += z[i] * x[i];
  }
  for (int i = 0; i < 6; i++) gxx[i] *= 0.05;
  double drr = 2.0 / (3.0 * D), dss = 1.0 / (6.0 * D);
  double nu_omega = 7.957747e+05 / omega;
  double dd = -(epsilon * omega);
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double rr = drr * (X[i] * X[j] + Y[i] * Y[j] + Z[i] * Z[j]);
      double ss = lsi[i] * lsi[j] * dss *
                  (-zi[i] * (-zi[j] * gxx[1] + yi[j] * gxx[4] + yz[j] * g[1]) +
                   yi[i] * (-zi[j] * gxx[4] + yi[j] * gxx[2] + yz[j] * g[2]) +
                   yz[i] * (-zi[j] * g[1] + yi[j] * g[2] + yz[j])

                   - xi[i] * (-xi[j] * gxx[2] + zi[j] * gxx[5] + zx[j] * g[2]) +
                   zi[i] * (-xi[j] * gxx[5] + zi[j] * gxx[0] + zx[j] * g[0]) +
                   zx[i] * (-xi[j] * g[2] + zi[j] * g[0] + zx[j])

                   - yi[i] * (-yi[j] * gxx[0] + xi[j] * gxx[3] + xy[j] * g[0]) +
                   xi[i] * (-yi[j] * gxx[3] + xi[j] * gxx[1] + xy[j] * g[1]) +
                   xy[i] * (-yi[j] * g[0] + xi[j] * g[1] + xy[j]));
      double re = 0.0, im = 0.0;
      re += nu_omega * rr;
      re += dd * ss;
      im += sigma * ss;
      ae[2 * (i * 6 + j)] = re;
      ae[2 * (i * 6 + j) + 1] = im;
    }
  return bad ? -7 : 0;
}

/* ------------------------------------------------------------------------ */
/* TMP_AIJ: lower-triangle row lists                                        */

typedef struct {
  int nf;
  int *n, *cap;
  int **col;
  cpx **val;
  cpx *b;
} Tmp;

static void tmp_init(Tmp *t, int nf) {
  t->nf = nf;
  t->n = (int *)calloc(nf + 1, sizeof(int));
  t->cap = (int *)calloc(nf + 1, sizeof(int));
  t->col = (int **)calloc(nf + 1, sizeof(int *));
  t->val = (cpx **)calloc(nf + 1, sizeof(cpx *));
  t->b = (cpx *)calloc(nf + 1, sizeof(cpx));
}

static void tmp_free(Tmp *t) {
  for (int i = 0; i < t->nf; i++) {
    free(t->col[i]);
    free(t->val[i]);
  }
  free(t->n);
  free(t->cap);
  free(t->col);
  free(t->val);
  free(t->b);
}

static void tmp_copy(Tmp *d, const Tmp *s) {
  tmp_init(d, s->nf);
  for (int i = 0; i < s->nf; i++) {
    d->n[i] = d->cap[i] = s->n[i];
    d->col[i] = (int *)malloc(sizeof(int) * (s->n[i] + 1));
    d->val[i] = (cpx *)malloc(sizeof(cpx) * (s->n[i] + 1));
    memcpy(d->col[i], s->col[i], sizeof(int) * s->n[i]);
    memcpy(d->val[i], s->val[i], sizeof(cpx) * s->n[i]);
  }
  memcpy(d->b, s->b, sizeof(cpx) * s->nf);
}

static void row_push(Tmp *t, int r, int c, cpx v) {
  if (t->n[r] == t->cap[r]) {
    t->cap[r] = t->cap[r] ? 2 * t->cap[r] : 8;
    t->col[r] = (int *)realloc(t->col[r], sizeof(int) * t->cap[r]);
    t->val[r] = (cpx *)realloc(t->val[r], sizeof(cpx) * t->cap[r]);
  }
  t->col[r][t->n[r]] = c;
  t->val[r][t->n[r]] = v;
  t->n[r]++;
}

/* stable sort of one row by column (the reference bubble-sorts,
   lib/std/sort.c:88-108; columns are unique so any stable sort agrees) */
static void row_sort(int n, int *col, cpx *val) {
  for (int i = 1; i < n; i++) {
    int c = col[i];
    cpx v = val[i];
    int j = i - 1;
    while (j >= 0 && col[j] > c) {
      col[j + 1] = col[j];
      val[j + 1] = val[j];
      j--;
    }
    col[j + 1] = c;
    val[j + 1] = v;
  }
}

static void delete_zero(Tmp *t) {
  for (int r = 0; r < t->nf; r++) {
    int k = 0;
    for (int q = 0; q < t->n[r]; q++) {
      if (c_iszero(t->val[r][q])) continue;
      t->col[r][k] = t->col[r][q];
      t->val[r][k] = t->val[r][q];
      k++;
    }
    t->n[r] = k;
  }
}

typedef struct {
  int nel;
  const int *nop;
  const double *crd;
  const double *eps;
  const double *sigma;
  int nmp;
  int nbc;
  const int *ibc;
  int ninbc;
  const int *inbc_nfid;
  const int *inbc_ln;
  const double *b;
} Sub;

static int assemble_sub(const Sub *s, double omega, Tmp *t) {
  tmp_init(t, s->nmp);
  int rc = 0;
  for (int el = 0; el < s->nel; el++) {
    const int *ne = s->nop + 10 * el;
    double xyz[12];
    for (int i = 0; i < 4; i++) {
      xyz[i] = s->crd[3 * ne[i]];
      xyz[4 + i] = s->crd[3 * ne[i] + 1];
      xyz[8 + i] = s->crd[3 * ne[i] + 2];
    }
    double ae[72];
    if (orc_element_matrix(xyz, s->eps[el], s->sigma[el], omega, ae) != 0) rc = -7;
    const int *ind = ne + 4;
    /* SetAe: keep entries with indCol >= indRow, stored in row indCol */
    for (int c = 0; c < 6; c++)
      for (int r = 0; r < 6; r++) {
        int icol = ind[c], irow = ind[r];
        if (icol < irow) continue;
        cpx dd = {ae[2 * (c * 6 + r)], ae[2 * (c * 6 + r) + 1]};
        if (c_iszero(dd)) continue;
        int found = 0;
        for (int q = 0; q < t->n[icol]; q++)
          if (t->col[icol][q] == irow) {
            t->val[icol][q] = c_add(t->val[icol][q], dd);
            found = 1;
            break;
          }
        if (!found) row_push(t, icol, irow, dd);
      }
  }
  for (int r = 0; r < t->nf; r++) row_sort(t->n[r], t->col[r], t->val[r]);
  delete_zero(t);
  for (int r = 0; r < t->nf; r++) {
    t->b[r].re += s->b[2 * r];
    t->b[r].im += s->b[2 * r + 1];
  }
  return rc;
}

/* SetBC on a copy: identity rows, eliminated columns, right-hand side */
static void set_bc(Tmp *t, int nbc, const int *ibc_in, const cpx *vbc_in) {
  int *ibc = (int *)malloc(sizeof(int) * (nbc + 1));
  cpx *val = (cpx *)malloc(sizeof(cpx) * (nbc + 1));
  memcpy(ibc, ibc_in, sizeof(int) * nbc);
  memcpy(val, vbc_in, sizeof(cpx) * nbc);
  row_sort(nbc, ibc, val);
  for (int r = 0; r < t->nf; r++) row_sort(t->n[r], t->col[r], t->val[r]);
  for (int bc = 0; bc < nbc; bc++) {
    int icol = ibc[bc];
    for (int q = 0; q < t->n[icol]; q++) {
      int col = t->col[icol][q];
      t->b[col] = c_sub(t->b[col], c_mul(t->val[icol][q], val[bc]));
    }
    t->n[icol] = 0;
    row_push(t, icol, icol, (cpx){1.0, 0.0});
  }
  for (int col = 0; col < t->nf; col++) {
    int bc = 0;
    for (int q = 0; q < t->n[col]; q++) {
      int irow = t->col[col][q];
      if (irow == col) continue;
      for (; bc < nbc; bc++) {
        if (irow < ibc[bc]) break;
        if (ibc[bc] == irow) {
          t->b[col] = c_sub(t->b[col], c_mul(t->val[col][q], val[bc]));
          t->val[col][q] = (cpx){0.0, 0.0};
          bc++;
          break;
        }
      }
    }
  }
  for (int bc = 0; bc < nbc; bc++) t->b[ibc[bc]] = val[bc];
  delete_zero(t);
  free(ibc);
  free(val);
}

/* skyline envelope, factor and solve (advlas_skyline.c:12-167) */
typedef struct {
  int n, nlen;
  int *idx1, *idx2;
  double _Complex *mat;
} Sky;

static void skyline_from_tmp(const Tmp *t, Sky *d) {
  d->n = t->nf;
  d->idx1 = (int *)calloc(d->n + 1, sizeof(int));
  d->idx2 = (int *)calloc(d->n + 1, sizeof(int));
  for (int i = 0; i < d->n; i++) d->idx1[i] = t->n[i] > 0 ? t->col[i][0] : i;
  d->idx2[0] = 0;
  for (int i = 1; i < d->n; i++) d->idx2[i] = d->idx2[i - 1] + i - d->idx1[i];
  d->nlen = d->n > 0 ? d->idx2[d->n - 1] + d->n : 0;
  d->mat = (double _Complex *)calloc(d->nlen + 1, sizeof(double _Complex));
  for (int i = 0; i < d->n; i++)
    for (int q = 0; q < t->n[i]; q++) d->mat[d->idx2[i] + t->col[i][q]] = t->val[i][q].re + t->val[i][q].im * I;
}

static void skyline_factor(Sky *d) {
  int n = d->n;
  int *ii = d->idx1, *ij = d->idx2;
  double _Complex *S = d->mat, r;
  double _Complex *Dg = (double _Complex *)calloc(n + 1, sizeof(double _Complex));
  if (n == 0) {
    free(Dg);
    return;
  }
  Dg[0] = 1 / S[0];
  for (int i = 1; i < n; i++) Dg[i] = S[ij[i] + i];
  for (int i = 1; i < n; i++) {
    int ifst = ij[i];
    for (int j = ii[i]; j < i; j++) {
      int jfst = ij[j];
      int m = ii[i] > ii[j] ? ii[i] : ii[j];
      r = 0.0 + 0.0 * I;
      for (int k = m; k < j; k++) r += S[ifst + k] * S[jfst + k];
      S[ifst + j] -= r;
    }
    r = 0.0 + 0.0 * I;
    for (int k = ii[i]; k < i; k++) {
      r += S[ifst + k] * S[ifst + k] * Dg[k];
      S[ifst + k] *= Dg[k];
    }
    Dg[i] = 1 / (Dg[i] - r);
  }
  for (int i = 0; i < n; i++) S[ij[i] + i] = Dg[i];
  free(Dg);
}

static void skyline_solve(const Sky *d, double _Complex *v) {
  int n = d->n;
  const int *ii = d->idx1, *ij = d->idx2;
  const double _Complex *S = d->mat;
  for (int i = 1; i < n; i++) {
    double _Complex r = 0.0;
    for (int j = ii[i]; j < i; j++) r += S[ij[i] + j] * v[j];
    v[i] -= r;
  }
  for (int i = 0; i < n; i++) v[i] *= S[ij[i] + i];
  for (int i = n - 1; i >= 1; i--) {
    double _Complex r = v[i];
    for (int j = ii[i]; j < i; j++) v[j] -= S[ij[i] + j] * r;
  }
}

static void sky_free(Sky *d) {
  free(d->idx1);
  free(d->idx2);
  free(d->mat);
}

/* x = A v, symmetric from the lower rows (aij_matrix_func.h:624-658) */
static void mxv(const Tmp *t, const cpx *v, cpx *x) {
  for (int i = 0; i < t->nf; i++) x[i] = (cpx){0.0, 0.0};
  for (int col = 0; col < t->nf; col++)
    for (int q = 0; q < t->n[col]; q++) {
      int irow = t->col[col][q];
      x[col] = c_add(x[col], c_mul(t->val[col][q], v[irow]));
      if (irow != col) x[irow] = c_add(x[irow], c_mul(t->val[col][q], v[col]));
    }
}

/* one subdomain solve: SetBC on a copy (b zeroed unless keep_b), the stored
   factor, then vec = A x (- b when subtract_b) */
static void solve_dom(const Tmp *orig, const Sky *fac, const Sub *s, const cpx *vbc, int keep_b, int subtract_b,
                      cpx *x, cpx *vec) {
  Tmp t;
  tmp_copy(&t, orig);
  if (!keep_b)
    for (int i = 0; i < t.nf; i++) t.b[i] = (cpx){0.0, 0.0};
  set_bc(&t, s->nbc, s->ibc, vbc);
  double _Complex *rhs = (double _Complex *)calloc(t.nf + 1, sizeof(double _Complex));
  for (int i = 0; i < t.nf; i++) rhs[i] = t.b[i].re + t.b[i].im * I;
  tmp_free(&t);
  skyline_solve(fac, rhs);
  for (int i = 0; i < s->nmp; i++) x[i] = (cpx){creal(rhs[i]), cimag(rhs[i])};
  free(rhs);
  mxv(orig, x, vec);
  if (subtract_b)
    for (int i = 0; i < s->nmp; i++) vec[i] = c_sub(vec[i], orig->b[i]);
}

static void fill_subs(Sub *subs, int nsub, const int *nel, const int *nop, const int *nap, const double *crd,
                      const double *eps, const double *sigma, const int *nmp, const int *nbc, const int *ibc,
                      const int *ninbc, const int *inbc_nfid, const int *inbc_ln, const double *b) {
  int64_t oe = 0, ov = 0, om = 0, ob = 0, oi = 0;
  for (int s = 0; s < nsub; s++) {
    subs[s].nel = nel[s];
    subs[s].nop = nop + 10 * oe;
    subs[s].eps = eps + oe;
    subs[s].sigma = sigma + oe;
    subs[s].crd = crd + 3 * ov;
    subs[s].nmp = nmp[s];
    subs[s].b = b + 2 * om;
    subs[s].nbc = nbc[s];
    subs[s].ibc = ibc + ob;
    subs[s].ninbc = ninbc[s];
    subs[s].inbc_nfid = inbc_nfid + oi;
    subs[s].inbc_ln = inbc_ln + oi;
    oe += nel[s];
    ov += nap[s];
    om += nmp[s];
    ob += nbc[s];
    oi += ninbc[s];
  }
}

/* Assembled lower rows of one subdomain (after DeleteZero) and its
   right-hand side.  Returns nnz, or -(needed) when max_nnz is too small. */
int orc_assemble_sub(int nel, const int *nop, const double *crd, const double *eps, const double *sigma, int nmp,
                     const double *b, double omega, int max_nnz, int *row_ptr, int *col, double *val, double *b_out) {
  Sub s;
  memset(&s, 0, sizeof(s));
  s.nel = nel;
  s.nop = nop;
  s.crd = crd;
  s.eps = eps;
  s.sigma = sigma;
  s.nmp = nmp;
  s.b = b;
  Tmp t;
  assemble_sub(&s, omega, &t);
  int nnz = 0;
  for (int r = 0; r < nmp; r++) nnz += t.n[r];
  if (nnz > max_nnz) {
    tmp_free(&t);
    return -nnz;
  }
  int k = 0;
  row_ptr[0] = 0;
  for (int r = 0; r < nmp; r++) {
    for (int q = 0; q < t.n[r]; q++) {
      col[k] = t.col[r][q];
      val[2 * k] = t.val[r][q].re;
      val[2 * k + 1] = t.val[r][q].im;
      k++;
    }
    row_ptr[r + 1] = k;
  }
  for (int r = 0; r < nmp; r++) {
    b_out[2 * r] = t.b[r].re;
    b_out[2 * r + 1] = t.b[r].im;
  }
  tmp_free(&t);
  return nnz;
}

/* Skyline profile and LDL^T factor of one subdomain after Dirichlet
   elimination, in the reference's layout.  Returns nlen, or -(needed). */
int orc_factor_sub(int nel, const int *nop, const double *crd, const double *eps, const double *sigma, int nmp,
                   int nbc, const int *ibc, double omega, int max_nlen, int *idx1, int *idx2, double *mat) {
  Sub s;
  memset(&s, 0, sizeof(s));
  double *zb = (double *)calloc(2 * nmp + 2, sizeof(double));
  s.nel = nel;
  s.nop = nop;
  s.crd = crd;
  s.eps = eps;
  s.sigma = sigma;
  s.nmp = nmp;
  s.b = zb;
  s.nbc = nbc;
  s.ibc = ibc;
  Tmp t, c;
  assemble_sub(&s, omega, &t);
  tmp_copy(&c, &t);
  cpx *z = (cpx *)calloc(nbc + 1, sizeof(cpx));
  set_bc(&c, nbc, ibc, z);
  Sky d;
  skyline_from_tmp(&c, &d);
  int nlen = d.nlen;
  if (nlen <= max_nlen) {
    skyline_factor(&d);
    memcpy(idx1, d.idx1, sizeof(int) * nmp);
    memcpy(idx2, d.idx2, sizeof(int) * nmp);
    for (int k = 0; k < nlen; k++) {
      mat[2 * k] = creal(d.mat[k]);
      mat[2 * k + 1] = cimag(d.mat[k]);
    }
  }
  sky_free(&d);
  tmp_free(&c);
  tmp_free(&t);
  free(z);
  free(zb);
  return nlen <= max_nlen ? nlen : -nlen;
}

/* The full s-mode HDDM solve for one part.  Writes the per-subdomain
   solutions (dm->x_c, concatenated 2*nmp), the residual history (one value
   per iteration) and returns the number of iterations (hddm_sw.loop - 1),
   or a negative code.  *norm0 receives max|r0|. */
int orc_hddm(int nsub, const int *nel, const int *nop, const int *nap, const double *crd, const double *eps,
             const double *sigma, const int *nmp, const int *nbc, const int *ibc, const int *ninbc,
             const int *inbc_nfid, const int *inbc_ln, const double *b, int tfree, double omega, double hddm_eps,
             int hddm_max_loop, double *x_out, double *hist, double *norm0) {
  Sub *subs = (Sub *)calloc(nsub, sizeof(Sub));
  fill_subs(subs, nsub, nel, nop, nap, crd, eps, sigma, nmp, nbc, ibc, ninbc, inbc_nfid, inbc_ln, b);
  Tmp *tmp = (Tmp *)calloc(nsub, sizeof(Tmp));
  Sky *fac = (Sky *)calloc(nsub, sizeof(Sky));
  cpx *P = (cpx *)calloc(tfree + 1, sizeof(cpx)), *Q = (cpx *)calloc(tfree + 1, sizeof(cpx));
  cpx *R = (cpx *)calloc(tfree + 1, sizeof(cpx)), *Z = (cpx *)calloc(tfree + 1, sizeof(cpx));
  cpx *U = (cpx *)calloc(tfree + 1, sizeof(cpx)), *PC = (cpx *)calloc(tfree + 1, sizeof(cpx));
  int maxn = 0, maxbc = 0;
  for (int s = 0; s < nsub; s++) {
    if (nmp[s] > maxn) maxn = nmp[s];
    if (nbc[s] > maxbc) maxbc = nbc[s];
  }
  cpx *x = (cpx *)calloc(maxn + 1, sizeof(cpx)), *vec = (cpx *)calloc(maxn + 1, sizeof(cpx));
  cpx *vbc = (cpx *)calloc(maxbc + 1, sizeof(cpx));
  int rc = 0;
  /* first step: assemble, factor, solve with zero interface values */
  for (int s = 0; s < nsub; s++) {
    const Sub *sb = &subs[s];
    if (assemble_sub(sb, omega, &tmp[s]) != 0) rc = -7;
    Tmp c;
    tmp_copy(&c, &tmp[s]);
    for (int k = 0; k < sb->nbc; k++) vbc[k] = (cpx){0.0, 0.0};
    set_bc(&c, sb->nbc, sb->ibc, vbc);
    skyline_from_tmp(&c, &fac[s]);
    skyline_factor(&fac[s]);
    tmp_free(&c);
    solve_dom(&tmp[s], &fac[s], sb, vbc, 1, 1, x, vec);
    for (int i = 0; i < sb->ninbc; i++) Q[sb->inbc_ln[i]] = c_add(Q[sb->inbc_ln[i]], vec[sb->inbc_nfid[i]]);
    /* DIAG_MAKE on the unmodified matrix */
    for (int i = 0; i < sb->ninbc; i++) {
      int r = sb->inbc_nfid[i];
      cpx pc = {0.0, 0.0};
      for (int q = 0; q < tmp[s].n[r]; q++)
        if (tmp[s].col[r][q] == r) {
          pc = !c_iszero(tmp[s].val[r][q]) ? tmp[s].val[r][q] : (cpx){1.0, 0.0};
          break;
        }
      if (c_iszero(pc)) pc = (cpx){1.0, 0.0};
      PC[sb->inbc_ln[i]] = c_add(PC[sb->inbc_ln[i]], pc);
    }
  }
  /* ITERATION_S_1ST */
  memcpy(R, Q, sizeof(cpx) * tfree);
  for (int i = 0; i < tfree; i++) PC[i] = !c_iszero(PC[i]) ? c_div((cpx){1.0, 0.0}, PC[i]) : (cpx){1.0, 0.0};
  double resi = 0.0;
  for (int i = 0; i < tfree; i++) {
    Z[i] = c_mul(R[i], PC[i]);
    P[i] = Z[i];
    double t = c_abs(R[i]);
    if (t > resi) resi = t;
  }
  *norm0 = resi;
  int last = resi < NEARLY_ZERO;
  double r0 = 1.0 / resi;
  cpx rz = {0.0, 0.0};
  for (int i = 0; i < tfree; i++) rz = c_add(rz, c_mul(R[i], Z[i]));
  for (int i = 0; i < tfree; i++) Q[i] = (cpx){0.0, 0.0};
  int loop = 1;
  while (!last) {
    for (int s = 0; s < nsub; s++) {
      const Sub *sb = &subs[s];
      for (int k = 0; k < sb->nbc; k++) vbc[k] = (cpx){0.0, 0.0};
      for (int i = 0, j = sb->nbc - sb->ninbc; i < sb->ninbc; i++, j++) vbc[j] = P[sb->inbc_ln[i]];
      solve_dom(&tmp[s], &fac[s], sb, vbc, 0, 0, x, vec);
      for (int i = 0; i < sb->ninbc; i++) Q[sb->inbc_ln[i]] = c_add(Q[sb->inbc_ln[i]], vec[sb->inbc_nfid[i]]);
    }
    cpx pq = {0.0, 0.0}, malpha, beta;
    for (int i = 0; i < tfree; i++) pq = c_add(pq, c_mul(P[i], Q[i]));
    if (c_abs(rz) < NEARLY_ZERO && c_abs(pq) < NEARLY_ZERO)
      malpha = (cpx){0.0, 0.0};
    else
      malpha = c_sub((cpx){0.0, 0.0}, c_div(rz, pq));
    resi = 0.0;
    for (int i = 0; i < tfree; i++) {
      U[i] = c_add(U[i], c_mul(malpha, P[i]));
      R[i] = c_add(R[i], c_mul(malpha, Q[i]));
      double t = c_abs(R[i]);
      if (t > resi) resi = t;
    }
    resi *= r0;
    if (hist) hist[loop - 1] = resi;
    for (int i = 0; i < tfree; i++) Z[i] = c_mul(R[i], PC[i]);
    cpx rzn = {0.0, 0.0};
    for (int i = 0; i < tfree; i++) rzn = c_add(rzn, c_mul(R[i], Z[i]));
    if (c_abs(rzn) < NEARLY_ZERO && c_abs(rz) < NEARLY_ZERO)
      beta = (cpx){0.0, 0.0};
    else
      beta = c_div(rzn, rz);
    rz = rzn;
    for (int i = 0; i < tfree; i++) P[i] = c_add(Z[i], c_mul(beta, P[i]));
    if (resi < hddm_eps) {
      last = 1;
      memcpy(P, U, sizeof(cpx) * tfree);
    }
    for (int i = 0; i < tfree; i++) Q[i] = (cpx){0.0, 0.0};
    if (loop == hddm_max_loop) last = 1;
    loop++;
  }
  /* last step */
  int64_t off = 0;
  for (int s = 0; s < nsub; s++) {
    const Sub *sb = &subs[s];
    for (int k = 0; k < sb->nbc; k++) vbc[k] = (cpx){0.0, 0.0};
    for (int i = 0, j = sb->nbc - sb->ninbc; i < sb->ninbc; i++, j++) vbc[j] = P[sb->inbc_ln[i]];
    solve_dom(&tmp[s], &fac[s], sb, vbc, 1, 1, x, vec);
    for (int i = 0; i < sb->nmp; i++) {
      x_out[2 * (off + i)] = x[i].re;
      x_out[2 * (off + i) + 1] = x[i].im;
    }
    off += sb->nmp;
  }
  for (int s = 0; s < nsub; s++) {
    tmp_free(&tmp[s]);
    sky_free(&fac[s]);
  }
  free(tmp);
  free(fac);
  free(subs);
  free(P);
  free(Q);
  free(R);
  free(Z);
  free(U);
  free(PC);
  free(x);
  free(vec);
  free(vbc);
  return rc < 0 ? rc : loop - 1;
}

/* ------------------------------------------------------------------------ */
/* element results of the post step                                         */

/* HDDM_post_em_E (main/fullwave/fullwave.c:639-763) for every element t of
 * the mesh: from the six edge values x of the element (global edge ids in
 * file order 01,02,03,12,23,13, taken in the edge-table order
 * 01,02,03,12,13,23 that the slot-8/9 swap of make_MESH.c:556-585 gives the
 * reference's nop), with
 *   nu    = 7.957747e+05 if the element's flag is in the Permittivity list
 *           (mtrl.flag_i), else 0          (fullwave.c:672-677)
 *   sigma = the first Conductor-list match, else 0   (:678-683)
 * and each edge value first scaled by nu/omega (:722, which the E and Je sums
 * below then also use):
 *   B  = (2/D)     sum_i i * xe_i * (X_i, Y_i, Z_i)      (:719-730)
 *   E  = (2/D)     sum_i xe_i * (Fx_i, Fy_i, Fz_i)       (:735-749)
 *   Je = (sigma/D) sum_i xe_i * (Fx_i, Fy_i, Fz_i)       (:752-762)
 * B, E, Je receive 3 complex (6 doubles) per element.  Returns the number of
 * elements with a zero-length edge (the reference stops there in
 * tetNedelec_Direction, tetrahedral.c:257-258). */
int orc_post_em_E(int nt, const int *tet_vertices, const int *tet_edges, const double *crd, const int *flag,
                  int nflag, const int *flag_i, int nR, const int *R_i, const double *R_sigma, double omega,
                  const double *xedge, double *B, double *E, double *Je) {
  static const int file_slot[6] = {0, 1, 2, 3, 5, 4};
  int bad = 0;
  for (int t = 0; t < nt; t++) {
    const int flg = flag[t];
    double nu = 0.0, sigma = 0.0;
    for (int i = 0; i < nflag; i++)
      if (flg == flag_i[i]) {
        nu = 7.957747e+05;
        break;
      }
    for (int i = 0; i < nR; i++)
      if (flg == R_i[i]) {
        sigma = R_sigma[i];
        break;
      }
    cpx xe[6];
    for (int i = 0; i < 6; i++) {
      const int e = tet_edges[6 * t + file_slot[i]];
      xe[i] = (cpx){xedge[2 * e], xedge[2 * e + 1]};
    }
    double x[4], y[4], z[4];
    for (int i = 0; i < 4; i++) {
      const int v = tet_vertices[4 * t + i];
      x[i] = crd[3 * v];
      y[i] = crd[3 * v + 1];
      z[i] = crd[3 * v + 2];
    }
    /* tet_Volume6 */
    double D = -x[0] * y[1] * z[2] + x[0] * y[1] * z[3] + x[0] * y[2] * z[1] - x[0] * y[2] * z[3] -
               x[0] * y[3] * z[1] + x[0] * y[3] * z[2] + x[1] * y[0] * z[2] - x[1] * y[0] * z[3] -
               x[1] * y[2] * z[0] + x[1] * y[2] * z[3] + x[1] * y[3] * z[0] - x[1] * y[3] * z[2] -
               x[2] * y[0] * z[1] + x[2] * y[0] * z[3] + x[2] * y[1] * z[0] - x[2] * y[1] * z[3] -
               x[2] * y[3] * z[0] + x[2] * y[3] * z[1] + x[3] * y[0] * z[1] - x[3] * y[0] * z[2] -
               x[3] * y[1] * z[0] + x[3] * y[1] * z[2] + x[3] * y[2] * z[0] - x[3] * y[2] * z[1];
    double X[6], Y[6], Z[6], Fx[6], Fy[6], Fz[6], g[3];
    g[0] = (x[0] + x[1] + x[2] + x[3]) * 0.25; /* tet_Center */
    g[1] = (y[0] + y[1] + y[2] + y[3]) * 0.25;
    g[2] = (z[0] + z[1] + z[2] + z[3]) * 0.25;
    for (int i = 0; i < 6; i++) {
      const int a = TET_N[i][0], b = TET_N[i][1], p = TET_N[i][2], q = TET_N[i][3];
      const double l = sqrt(pow(x[a] - x[b], 2) + pow(y[a] - y[b], 2) + pow(z[a] - z[b], 2));
      int si; /* tetNedelec_Direction */
      double pp = x[b] - x[a];
      if (pp > 0.0)
        si = 1;
      else if (pp < 0.0)
        si = -1;
      else {
        pp = y[b] - y[a];
        if (pp > 0.0)
          si = 1;
        else if (pp < 0.0)
          si = -1;
        else {
          pp = z[b] - z[a];
          si = pp > 0.0 ? 1 : (pp < 0.0 ? -1 : 0);
        }
      }
      if (si == 0) bad++;
      const double xi = x[q] - x[p], yi = y[q] - y[p], zi = z[q] - z[p]; /* tetNedelec_mk */
      const double d = l * (double)si;
      X[i] = d * xi; /* tetNedelec_XYZ */
      Y[i] = d * yi;
      Z[i] = d * zi;
      const double xy = x[p] * y[q] - x[q] * y[p]; /* tetNedelec_km_mk */
      const double yz = y[p] * z[q] - y[q] * z[p];
      const double zx = z[p] * x[q] - z[q] * x[p];
      Fx[i] = d * (yz - zi * g[1] + yi * g[2]); /* tetNedelec_Fxyz */
      Fy[i] = d * (zx - xi * g[2] + zi * g[0]);
      Fz[i] = d * (xy - yi * g[0] + xi * g[1]);
    }
    const cpx ci = {0.0, 1.0};
    cpx rb[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int i = 0; i < 6; i++) {
      xe[i] = (cpx){xe[i].re * (nu / omega), xe[i].im * (nu / omega)};
      const cpx cc = c_mul(xe[i], ci);
      rb[0] = c_add(rb[0], (cpx){cc.re * X[i], cc.im * X[i]});
      rb[1] = c_add(rb[1], (cpx){cc.re * Y[i], cc.im * Y[i]});
      rb[2] = c_add(rb[2], (cpx){cc.re * Z[i], cc.im * Z[i]});
    }
    cpx et[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int i = 0; i < 6; i++) {
      et[0] = c_add(et[0], (cpx){xe[i].re * Fx[i], xe[i].im * Fx[i]});
      et[1] = c_add(et[1], (cpx){xe[i].re * Fy[i], xe[i].im * Fy[i]});
      et[2] = c_add(et[2], (cpx){xe[i].re * Fz[i], xe[i].im * Fz[i]});
    }
    /* the Je sums repeat the E sums on the same xe and F (:752-762) */
    const double dd = 2.0 / D, ds = sigma / D;
    for (int k = 0; k < 3; k++) {
      B[6 * t + 2 * k] = rb[k].re * dd;
      B[6 * t + 2 * k + 1] = rb[k].im * dd;
      E[6 * t + 2 * k] = et[k].re * dd;
      E[6 * t + 2 * k + 1] = et[k].im * dd;
      Je[6 * t + 2 * k] = et[k].re * ds;
      Je[6 * t + 2 * k + 1] = et[k].im * ds;
    }
  }
  return bad;
}

/* ------------------------------------------------------------------------ */
/* element right-hand side                                                  */

static const int TET_M[4][4] = {{0, 1, 2, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}, {3, 1, 0, 2}};

/* The element right-hand side be (6 complex, edge-table order) of
 * tet_MakeElement_EM_E (lib/fem/make_elem_em.c:66-330) for one element with
 * vertex coordinates xyz (x0..x3, y0..y3, z0..z3) and conductivity sigma:
 *   n_gaps > 0 (volt.dat dg > 0, :302-329): DGe_j = (0, dV_k) for the last
 *     gap box k holding vertex j (boxes inclusive), 0 otherwise; if any
 *     vertex is in a box, be_i = (sigma omega) sum_j DGe_j gs_ij with
 *     gs = tetNedelec_gradside (tetrahedral.c:645-661), else be = 0;
 *   n_gaps = 0 (current input, :271-300): for an antenna element
 *     (antenna != 0) be = 0 + (be_JoA - 0) with be_JoA =
 *     tetNedelec_JoA_Complex (tetrahedral.c:794-858) of the vertex currents
 *     joe (vertex j, component c: re joe[2*(3j+c)], im joe[2*(3j+c)+1], the
 *     reference's Joe = (-Jo, -Jor)), and be = 0 otherwise.
 * be receives 12 doubles (re, im per edge). */
void orc_element_rhs(const double *xyz, double sigma, double omega, int n_gaps, const double *gap_box,
                     const double *gap_volt, int antenna, const double *joe, double *be) {
  const double *x = xyz, *y = xyz + 4, *z = xyz + 8;
  for (int i = 0; i < 12; i++) be[i] = 0.0;
  double l[6], b[4], c[4], d[4], Fx[6], Fy[6], Fz[6], g[3];
  int si[6];
  double D = -x[0] * y[1] * z[2] + x[0] * y[1] * z[3] + x[0] * y[2] * z[1] - x[0] * y[2] * z[3] -
             x[0] * y[3] * z[1] + x[0] * y[3] * z[2] + x[1] * y[0] * z[2] - x[1] * y[0] * z[3] -
             x[1] * y[2] * z[0] + x[1] * y[2] * z[3] + x[1] * y[3] * z[0] - x[1] * y[3] * z[2] -
             x[2] * y[0] * z[1] + x[2] * y[0] * z[3] + x[2] * y[1] * z[0] - x[2] * y[1] * z[3] -
             x[2] * y[3] * z[0] + x[2] * y[3] * z[1] + x[3] * y[0] * z[1] - x[3] * y[0] * z[2] -
             x[3] * y[1] * z[0] + x[3] * y[1] * z[2] + x[3] * y[2] * z[0] - x[3] * y[2] * z[1];
  g[0] = (x[0] + x[1] + x[2] + x[3]) * 0.25;
  g[1] = (y[0] + y[1] + y[2] + y[3]) * 0.25;
  g[2] = (z[0] + z[1] + z[2] + z[3]) * 0.25;
  for (int i = 0; i < 4; i++) { /* tet_simple_b, _c, _d */
    const int ii = TET_M[i][1], jj = TET_M[i][2], kk = TET_M[i][3];
    b[i] = -1.0 * (y[ii] * (z[jj] - z[kk]) + y[jj] * (z[kk] - z[ii]) + y[kk] * (z[ii] - z[jj]));
    c[i] = -1.0 * (z[ii] * (x[jj] - x[kk]) + z[jj] * (x[kk] - x[ii]) + z[kk] * (x[ii] - x[jj]));
    d[i] = -1.0 * (x[ii] * (y[jj] - y[kk]) + x[jj] * (y[kk] - y[ii]) + x[kk] * (y[ii] - y[jj]));
  }
  for (int i = 0; i < 6; i++) {
    const int a = TET_N[i][0], bb = TET_N[i][1], p = TET_N[i][2], q = TET_N[i][3];
    l[i] = sqrt(pow(x[a] - x[bb], 2) + pow(y[a] - y[bb], 2) + pow(z[a] - z[bb], 2));
    double pp = x[bb] - x[a];
    if (pp > 0.0)
      si[i] = 1;
    else if (pp < 0.0)
      si[i] = -1;
    else {
      pp = y[bb] - y[a];
      if (pp > 0.0)
        si[i] = 1;
      else if (pp < 0.0)
        si[i] = -1;
      else {
        pp = z[bb] - z[a];
        si[i] = pp > 0.0 ? 1 : (pp < 0.0 ? -1 : 0);
      }
    }
    const double xi = x[q] - x[p], yi = y[q] - y[p], zi = z[q] - z[p];
    const double xy = x[p] * y[q] - x[q] * y[p];
    const double yz = y[p] * z[q] - y[q] * z[p];
    const double zx = z[p] * x[q] - z[q] * x[p];
    const double dl = l[i] * (double)si[i];
    Fx[i] = dl * (yz - zi * g[1] + yi * g[2]);
    Fy[i] = dl * (zx - xi * g[2] + zi * g[0]);
    Fz[i] = dl * (xy - yi * g[0] + xi * g[1]);
  }
  if (n_gaps > 0) {
    cpx dge[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    int dvn = 0;
    for (int k = 0; k < n_gaps; k++) {
      const double *bx = gap_box + 6 * k;
      for (int j = 0; j < 4; j++)
        if ((bx[0] <= x[j] && x[j] <= bx[1]) && (bx[2] <= y[j] && y[j] <= bx[3]) &&
            (bx[4] <= z[j] && z[j] <= bx[5])) {
          dge[j] = (cpx){0.0, gap_volt[k]};
          dvn = 1;
        }
    }
    if (dvn) {
      const double dd = 1.0 / (6.0 * D);
      for (int i = 0; i < 6; i++) {
        cpx s = {0.0, 0.0};
        for (int j = 0; j < 4; j++) {
          const double gs = dd * (Fx[i] * b[j] + Fy[i] * c[j] + Fz[i] * d[j]);
          s = c_add(s, (cpx){dge[j].re * gs, dge[j].im * gs});
        }
        be[2 * i] = s.re * (sigma * omega);
        be[2 * i + 1] = s.im * (sigma * omega);
      }
    }
    return;
  }
  if (!antenna) return;
  static const double d0[6][4] = {{2.0, 1.0, 1.0, 1.0}, {2.0, 1.0, 1.0, 1.0}, {2.0, 1.0, 1.0, 1.0},
                                  {1.0, 2.0, 1.0, 1.0}, {1.0, 2.0, 1.0, 1.0}, {1.0, 1.0, 2.0, 1.0}};
  static const double d1[6][4] = {{-1.0, -2.0, -1.0, -1.0}, {-1.0, -1.0, -2.0, -1.0}, {-1.0, -1.0, -1.0, -2.0},
                                  {-1.0, -1.0, -2.0, -1.0}, {-1.0, -1.0, -1.0, -2.0}, {-1.0, -1.0, -1.0, -2.0}};
  for (int i = 0; i < 6; i++) {
    const int p0 = TET_N[i][0], p1 = TET_N[i][1];
    const double dd = (double)si[i] * l[i] / 120.0;
    double pn[12];
    for (int j = 0; j < 4; j++) {
      pn[j] = dd * (d0[i][j] * b[p1] + d1[i][j] * b[p0]);
      pn[4 + j] = dd * (d0[i][j] * c[p1] + d1[i][j] * c[p0]);
      pn[8 + j] = dd * (d0[i][j] * d[p1] + d1[i][j] * d[p0]);
    }
    cpx s = {0.0, 0.0};
    for (int cc = 0; cc < 3; cc++)
      for (int j = 0; j < 4; j++) {
        const double w = pn[4 * cc + j];
        s = c_add(s, (cpx){joe[2 * (3 * j + cc)] * w, joe[2 * (3 * j + cc) + 1] * w});
      }
    /* be = be + (be_JoA - be_gs), be_gs = sum of 0 * gs = +0 */
    be[2 * i] = 0.0 + (s.re - 0.0);
    be[2 * i + 1] = 0.0 + (s.im - 0.0);
  }
}
