/*
 * Reference harness: runs the reference's own s-mode full-wave HDDM solver
 * (lib/hddm, lib/fem, lib/mymt_aij_solver, main/fullwave/fullwave.c), built
 * from its sources by oracle/Makefile.ref, on a synthetic model written by
 * adventure_fullwave_b200.meshgen.write_hddm_model.  TEST INFRASTRUCTURE ONLY:
 * it is the oracle the CUDA path is checked against and the CPU baseline it
 * is timed against; the product never links or runs it.
 *
 * The flow is the reference's main() (main/fullwave/main.c:34-124) with one
 * change made through the reference's own plug-in table (HDDM_FUNC,
 * lib/std/types.h:629-730): the table from set_hddm_func_fullwave
 * (main/fullwave/fullwave.c:23-146) gets
 *   - make_TMP_AIJ wrapped to add the edge current source of <dir>/source.txt
 *     to the assembled right-hand side of the subdomain that owns the edge
 *     (the lowest-numbered subdomain holding it), and, when <dir>/antenna.txt
 *     exists, to hand the reference's element routine the antenna flags and
 *     vertex currents it reads (MTRL.antenna_def[k].flag, DomMesh.antenna[k]
 *     .enf/.Jo/.Jor; lib/fem/make_elem_em.c:110-115,287-300) in place of the
 *     correction-Jo pre-solve that fills them in main(), and
 *   - solve_dom_1st / iteration_s / solve_dom_last wrapped to record timings
 *     and, on request, dump the reference's intermediate data.
 * The correction-Jo pre-solve of main.c:92-98 runs only for antennas, which
 * synthetic models do not define.
 *
 * With FW_HARNESS_MAIN=1 the model is read by the reference's own hddm_Init
 * and the correction-Jo pre-solve of main.c:92-98 runs first, as in main();
 * the antenna currents it leaves are dumped to <prefix>.jo, and the
 * pre-solve's own systems and potentials to <prefix>.cojo.  This runs a
 * model directory of the reference as its main() would.
 *
 * Usage: fw_ref_harness [reference options] <model_dir>
 * Environment:
 *   FW_HARNESS_OUT   output prefix (default <model_dir>/ref)
 *   FW_HARNESS_COJO_ONLY  1 (with FW_HARNESS_MAIN=1): stop after the
 *                    correction-Jo pre-solve and its dumps
 *   FW_HARNESS_DUMP  0: timings + solution, 1: + integer maps and the
 *                    element results of the post step,
 *                    2: + assembled TMP_AIJ and skyline factors
 * Outputs: <prefix>.json (timings, counts), <prefix>.sol (solution),
 *          <prefix>.ints, <prefix>.post, <prefix>.post_drop, <prefix>.aij,
 *          <prefix>.fac (dumps), and the
 *          reference's own residual log under <model_dir>/calc_log/.
 */
#include "advfullwave_lib.h"
#include "libfem.h"
#include "libhddm.h"

#include "fullwave.h"

#include <stdint.h>

/* the program identity the reference's fullwave driver passes to its
   option parser (main/fullwave/main.c:13-19) */
#define LOCAL_MODULE_NAME "Full-Wave analysis with HDDM"
#define LOCAL_VERSION ADVFW_VERSION
#define LOCAL_WORK WORK_HDDM_ANALYSIS
#define LOCAL_FIELD FIELD_ELECTROMAGNETIC
#define LOCAL_ANALYSIS ANALYSIS_FULL_WAVECURRENT
#define LOCAL_N_ARGUMENT 0
#define LOCAL_USAGE ""
#include <time.h>

extern COM_WLD_ID COM_ID;
extern COM_GRP_ID COM_GID;
extern int nstart;
extern int nend;
extern int nrepeat;
extern HDDM_SW hddm_sw;
extern WORK_TIMES work_times;
extern double s_time;

static int g_dump = 0;
static char g_prefix[FILENAME_MAX];
static PartMesh *g_pm = NULL;

/* source edges owned per subdomain: (local edge id, value) */
typedef struct {
  int n;
  int *edge;
  double *re;
  double *im;
} SubSource;
static SubSource *g_src = NULL;
/* the same sources by global node id of the mid-node */
static int g_srcn = 0;
static int *g_srcg = NULL;
static double *g_srcv = NULL;

#ifdef FW_HARNESS_GPU
/* adventure_fullwave_b200/dropin/set_hddm_func_gpu.c: the reference's table
   with the subdomain and interface slots on the GPU library */
void set_hddm_func_fullwave_gpu(HDDM_FUNC *f, OPTIONS options);
void set_hddm_func_correct_Jor_gpu(HDDM_FUNC *f, OPTIONS options);
void set_hddm_func_correct_Joi_gpu(HDDM_FUNC *f, OPTIONS options);
void hddm_gpu_set_edge_source(int n, const int *mid_gnid, const double *re_im);
#endif

/* antenna currents of <dir>/antenna.txt: per antenna its element flag and the
   reference's Jo / Jor (3 per global vertex); per subdomain an ANTENNA array
   whose enf maps local vertex ids to global vertex ids, so that
   tet_MakeElement_EM_E reads Jo[3 * global vertex + c] */
static int g_nant = 0;
static MTRL_ANTENNA_DEFINITION *g_antdef = NULL;
static ANTENNA **g_dom_ant = NULL;

static double t_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static double t_assemble = 0.0, t_first = 0.0, t_last = 0.0, t_iter_total = 0.0;
static double t_iter_mark = -1.0;
static int n_iter = 0;
static FILE *f_aij = NULL, *f_fac = NULL;

/* the reference's fullwave table entries this harness wraps */
static void (*ref_make_TMP_AIJ)(DomMesh *, MTRL) = NULL;
static void (*ref_solve_dom_1st)(DomMesh *, HDDM_Opt, SolvOpt, int (*)(AIJ_MAT *, SolvOpt, FILE *),
                                 HDDM_DOM_VEC *, int (*)(TMP_AIJ, HDDM_DOM_VEC *), FILE *) = NULL;
static void (*ref_iteration_s)(PartMesh *, HDDM_VEC *, HDDM_Opt, int (*)(HDDM_VEC *)) = NULL;
static void (*ref_iteration_s_1st)(PartMesh *, HDDM_VEC *, HDDM_Opt, int (*)(HDDM_VEC *),
                                   void (*)(OPinfo **, HDDM_VEC *)) = NULL;
static FILE *f_hist = NULL, *f_itimes = NULL;
static void (*ref_solve_dom_last)(DomMesh *, SolvOpt, int (*)(AIJ_MAT *, SolvOpt, FILE *), HDDM_DOM_VEC *,
                                  FILE *) = NULL;

static void w_i32(FILE *f, int v) { fwrite(&v, 4, 1, f); }

static void harness_make_TMP_AIJ(DomMesh *dm, MTRL mtrl) {
  double t0 = t_now();
  if (g_nant > 0) {
    /* the reference's own element routine with the antennas in place */
    MTRL m2 = mtrl;
    ANTENNA *saved = dm->antenna;
    m2.nantenna = g_nant;
    m2.antenna_def = g_antdef;
    dm->antenna = g_dom_ant[dm->domid];
    ref_make_TMP_AIJ(dm, m2);
    dm->antenna = saved;
  } else {
    ref_make_TMP_AIJ(dm, mtrl);
  }
  SubSource *s = &g_src[dm->domid];
  for (int k = 0; k < s->n; k++) {
    Complex *b = &dm->tmp_aij.tmp_b_c[s->edge[k]];
    b->re += s->re[k];
    b->im += s->im[k];
  }
  t_assemble += t_now() - t0;
  if (g_dump >= 2 && f_aij) {
    TMP_AIJ *a = &dm->tmp_aij;
    w_i32(f_aij, a->nf);
    for (int i = 0; i < a->nf; i++) {
      w_i32(f_aij, a->tmp_ai[i]);
      fwrite(a->tmp_aij[i], 4, a->tmp_ai[i], f_aij);
      fwrite(a->tmp_vij_c[i], sizeof(Complex), a->tmp_ai[i], f_aij);
    }
    fwrite(a->tmp_b_c, sizeof(Complex), a->nf, f_aij);
  }
}

static void harness_solve_dom_1st(DomMesh *dm, HDDM_Opt hddm_opt, SolvOpt solvopt,
                                  int (*dom_solver)(AIJ_MAT *, SolvOpt, FILE *), HDDM_DOM_VEC *v,
                                  int (*makePC)(TMP_AIJ, HDDM_DOM_VEC *), FILE *fp_log) {
  double t0 = t_now();
  ref_solve_dom_1st(dm, hddm_opt, solvopt, dom_solver, v, makePC, fp_log);
  t_first += t_now() - t0;
  if (g_dump >= 2 && f_fac) {
    DMatrix *d = &dm->dmat;
    w_i32(f_fac, d->ndim);
    w_i32(f_fac, d->nlen);
    fwrite(d->idx1, 4, d->ndim, f_fac);
    fwrite(d->idx2, 4, d->ndim, f_fac);
    fwrite(d->mat_dc, sizeof(double _Complex), d->nlen, f_fac);
  }
}

/* max |r| over the parts' interface residuals, in the loop order and with
   the ComplexAbs of ITERATION_S (lib/hddm/hddm_solver_s.h:196-200,300-318) */
static double residual_max(HDDM_VEC *hv) {
  double m = 0.0;
  for (int part = 0; part < COM_GID.nparent; part++)
    for (int i = 0; i < hv[part].infree; i++) {
      const double t = ComplexAbs(hv[part].r_c[i]);
      if (t > m) m = t;
    }
  return m;
}

/* the residual history at full precision (the log prints 7 digits): the
   initial max-norm, then resi = max|r| * r0 after every iteration */
static void harness_iteration_s_1st(PartMesh *pm, HDDM_VEC *hv, HDDM_Opt hddm_opt, int (*setPC)(HDDM_VEC *),
                                    void (*gatherPC_s)(OPinfo **, HDDM_VEC *)) {
  ref_iteration_s_1st(pm, hv, hddm_opt, setPC, gatherPC_s);
  if (f_hist) {
    const double n0 = residual_max(hv);
    fwrite(&n0, sizeof(double), 1, f_hist);
  }
}

static void harness_iteration_s(PartMesh *pm, HDDM_VEC *hv, HDDM_Opt hddm_opt, int (*setPC)(HDDM_VEC *)) {
  ref_iteration_s(pm, hv, hddm_opt, setPC);
  if (f_hist) {
    double resi = residual_max(hv);
    resi *= hv[0].r0;
    fwrite(&resi, sizeof(double), 1, f_hist);
  }
  double t = t_now();
  if (t_iter_mark >= 0.0) {
    /* one whole interface iteration: the subdomain solves and this COCG step */
    const double dt = t - t_iter_mark;
    t_iter_total += dt;
    if (f_itimes) fwrite(&dt, sizeof(double), 1, f_itimes);
  }
  t_iter_mark = t;
  n_iter++;
}

static void harness_solve_dom_last(DomMesh *dm, SolvOpt solvopt, int (*s)(AIJ_MAT *, SolvOpt, FILE *),
                                   HDDM_DOM_VEC *v, FILE *fp_log) {
  double t0 = t_now();
  ref_solve_dom_last(dm, solvopt, s, v, fp_log);
  t_last += t_now() - t0;
}

static void set_hddm_func_harness(HDDM_FUNC *f, OPTIONS options) {
#ifdef FW_HARNESS_GPU
  /* the GPU table: only the once-per-step slots are timed; the
     per-subdomain slots of that table do nothing */
  set_hddm_func_fullwave_gpu(f, options);
  ref_iteration_s = f->iteration_s;
  ref_iteration_s_1st = f->iteration_s_1st;
  ref_solve_dom_last = f->solve_dom_last;
  f->iteration_s_1st = harness_iteration_s_1st;
  f->iteration_s = harness_iteration_s;
  f->solve_dom_last = harness_solve_dom_last;
  return;
#endif
  set_hddm_func_fullwave(f, options);
  ref_make_TMP_AIJ = f->make_TMP_AIJ;
  ref_solve_dom_1st = f->solve_dom_1st;
  ref_iteration_s = f->iteration_s;
  ref_iteration_s_1st = f->iteration_s_1st;
  ref_solve_dom_last = f->solve_dom_last;
  f->iteration_s_1st = harness_iteration_s_1st;
  f->make_TMP_AIJ = harness_make_TMP_AIJ;
  f->solve_dom_1st = harness_solve_dom_1st;
  f->iteration_s = harness_iteration_s;
  f->solve_dom_last = harness_solve_dom_last;
}

/* global node id of each subdomain-local edge DOF */
static int *edge_gnid(PartMesh *pm, DomMesh *dm) {
  int *g = (int *)malloc(sizeof(int) * (dm->nmp > 0 ? dm->nmp : 1));
  for (int e = 0; e < dm->nmp; e++) g[e] = pm->pnid2gnid[dm->snid2pnid[dm->mpid2snid[e]]];
  return g;
}

static void load_sources(const char *dir, PartMesh *pm) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s/source.txt", dir);
  g_src = (SubSource *)calloc(pm->ndomain, sizeof(SubSource));
  FILE *f = fopen(path, "r");
  if (!f) return;
  int nrhs = 0, n = 0;
  if (fscanf(f, "%d", &nrhs) != 1 || nrhs < 1 || fscanf(f, "%d", &n) != 1) {
    fclose(f);
    return;
  }
  /* only the first right-hand side drives the reference run */
  for (int k = 0; k < n; k++) {
    int gnid;
    double re, im;
    if (fscanf(f, "%d %lf %lf", &gnid, &re, &im) != 3) break;
    g_srcg = (int *)realloc(g_srcg, sizeof(int) * (g_srcn + 1));
    g_srcv = (double *)realloc(g_srcv, sizeof(double) * 2 * (g_srcn + 1));
    g_srcg[g_srcn] = gnid;
    g_srcv[2 * g_srcn] = re;
    g_srcv[2 * g_srcn + 1] = im;
    g_srcn++;
    for (int d = 0; d < pm->ndomain; d++) {
      DomMesh *dm = &pm->dm[d];
      int *g = edge_gnid(pm, dm);
      int found = -1;
      for (int e = 0; e < dm->nmp; e++)
        if (g[e] == gnid) {
          found = e;
          break;
        }
      free(g);
      if (found >= 0) {
        SubSource *s = &g_src[d];
        s->edge = (int *)realloc(s->edge, sizeof(int) * (s->n + 1));
        s->re = (double *)realloc(s->re, sizeof(double) * (s->n + 1));
        s->im = (double *)realloc(s->im, sizeof(double) * (s->n + 1));
        s->edge[s->n] = found;
        s->re[s->n] = re;
        s->im[s->n] = im;
        s->n++;
        break;
      }
    }
  }
  fclose(f);
}

static void load_antennas(const char *dir, PartMesh *pm) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s/antenna.txt", dir);
  FILE *f = fopen(path, "r");
  if (!f) return;
  int nant = 0, nv = 0;
  if (fscanf(f, "%d %d", &nant, &nv) != 2 || nant < 1 || nv < 1) {
    fclose(f);
    return;
  }
  g_antdef = (MTRL_ANTENNA_DEFINITION *)calloc(nant, sizeof(MTRL_ANTENNA_DEFINITION));
  double **jo = (double **)calloc(nant, sizeof(double *));
  double **jor = (double **)calloc(nant, sizeof(double *));
  for (int k = 0; k < nant; k++) {
    if (fscanf(f, "%d", &g_antdef[k].flag) != 1) break;
    jo[k] = (double *)calloc(3 * (size_t)nv, sizeof(double));
    jor[k] = (double *)calloc(3 * (size_t)nv, sizeof(double));
    for (int v = 0; v < nv; v++)
      if (fscanf(f, "%lf %lf %lf %lf %lf %lf", &jo[k][3 * v], &jo[k][3 * v + 1], &jo[k][3 * v + 2], &jor[k][3 * v],
                 &jor[k][3 * v + 1], &jor[k][3 * v + 2]) != 6)
        break;
  }
  fclose(f);
  g_dom_ant = (ANTENNA **)calloc(pm->ndomain, sizeof(ANTENNA *));
  for (int d = 0; d < pm->ndomain; d++) {
    DomMesh *dm = &pm->dm[d];
    int *enf = (int *)malloc(sizeof(int) * (dm->nap > 0 ? dm->nap : 1));
    for (int v = 0; v < dm->nap; v++) enf[v] = pm->pnid2gnid[dm->snid2pnid[dm->apid2snid[v]]];
    g_dom_ant[d] = (ANTENNA *)calloc(nant, sizeof(ANTENNA));
    for (int k = 0; k < nant; k++) {
      g_dom_ant[d][k].antenna = k;
      g_dom_ant[d][k].enf = enf;
      g_dom_ant[d][k].Jo = jo[k];
      g_dom_ant[d][k].Jor = jor[k];
    }
  }
  g_nant = nant;
}

/* The antenna currents Jo, Jor after the correction-Jo pre-solve, per
   antenna and subdomain: every local vertex with an antenna node
   (enf >= 0) as (global node id, Jo x y z, Jor x y z). */
static void dump_jo(PartMesh *pms, int nparts) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s.jo", g_prefix);
  FILE *f = fopen(path, "w");
  if (!f) return;
  const int nant = pms[0].mtrl.nantenna;
  fprintf(f, "%d\n", nant);
  for (int k = 0; k < nant; k++) {
    int count = 0;
    for (int q = 0; q < nparts; q++)
      for (int d = 0; d < pms[q].ndomain; d++) {
        ANTENNA *a = &pms[q].dm[d].antenna[k];
        if (!a->enf) continue;
        for (int v = 0; v < pms[q].dm[d].nap; v++) count += a->enf[v] > -1;
      }
    fprintf(f, "%d %d\n", pms[0].mtrl.antenna_def[k].flag, count);
    for (int q = 0; q < nparts; q++)
    for (int d = 0; d < pms[q].ndomain; d++) {
      PartMesh *pm = &pms[q];
      DomMesh *dm = &pm->dm[d];
      ANTENNA *a = &dm->antenna[k];
      if (!a->enf) continue;
      for (int v = 0; v < dm->nap; v++) {
        const int j = a->enf[v];
        if (j < 0) continue;
        fprintf(f, "%d %.17e %.17e %.17e %.17e %.17e %.17e\n", pm->pnid2gnid[dm->snid2pnid[dm->apid2snid[v]]],
                a->Jo[3 * j], a->Jo[3 * j + 1], a->Jo[3 * j + 2], a->Jor[3 * j], a->Jor[3 * j + 1], a->Jor[3 * j + 2]);
      }
    }
  }
  fclose(f);
}

/* The correction-Jo pre-solve's systems and results (main.c:92-98 with
   lib/hddm/set_hddm_func.c:90-233): per antenna, per subdomain in part
   order, "nf nbc ninbc", the global node id of each antenna DOF
   (enf order), the Dirichlet list dbc.ibc, the interface entries (nfid,
   ln_part) and the potentials Ihr and Ihi the two real-symmetric HDDM runs
   leave (HDDM_get_result_sp_correct_Jor/Joi, set_hddm_func.c:626-667). */
static void dump_cojo(PartMesh *pms, int nparts) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s.cojo", g_prefix);
  FILE *f = fopen(path, "w");
  if (!f) return;
  const int nant = pms[0].mtrl.nantenna;
  int nsub = 0;
  for (int q = 0; q < nparts; q++) nsub += pms[q].ndomain;
  fprintf(f, "%d %d\n", nant, nsub);
  for (int k = 0; k < nant; k++) {
    fprintf(f, "%d %d\n", pms[0].mtrl.antenna_def[k].flag, pms[0].pantenna ? pms[0].pantenna[k].total_free : 0);
    for (int q = 0; q < nparts; q++)
      for (int d = 0; d < pms[q].ndomain; d++) {
        PartMesh *pm = &pms[q];
        DomMesh *dm = &pm->dm[d];
        ANTENNA *a = &dm->antenna[k];
        const int nf = a->enf ? a->nf : 0;
        fprintf(f, "%d %d %d\n", nf, nf ? a->dbc.nbc : 0, nf ? a->ninbc : 0);
        if (!nf) continue;
        int *gid = (int *)calloc(nf, sizeof(int));
        for (int v = 0; v < dm->nap; v++)
          if (a->enf[v] >= 0) gid[a->enf[v]] = pm->pnid2gnid[dm->snid2pnid[dm->apid2snid[v]]];
        for (int i = 0; i < nf; i++) fprintf(f, "%d%c", gid[i], i + 1 < nf ? ' ' : '\n');
        free(gid);
        for (int i = 0; i < a->dbc.nbc; i++) fprintf(f, "%d ", a->dbc.ibc[i]);
        fprintf(f, "\n");
        for (int i = 0; i < a->ninbc; i++) fprintf(f, "%d %d ", a->inbc[i].nfid, a->inbc[i].ln_part);
        fprintf(f, "\n");
        for (int i = 0; i < nf; i++) fprintf(f, "%.17e ", a->Ihr ? a->Ihr[i] : 0.0);
        fprintf(f, "\n");
        for (int i = 0; i < nf; i++) fprintf(f, "%.17e ", a->Ihi ? a->Ihi[i] : 0.0);
        fprintf(f, "\n");
      }
  }
  fclose(f);
}

/* every part's subdomains, parts in order; the header counts all of them and
   gives the first part's interface sizes */
static void dump_ints(PartMesh *pms, int nparts) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s.ints", g_prefix);
  FILE *f = fopen(path, "wb");
  if (!f) return;
  int total = 0;
  for (int q = 0; q < nparts; q++) total += pms[q].ndomain;
  w_i32(f, total);
  w_i32(f, pms[0].infree);
  w_i32(f, pms[0].outfree);
  w_i32(f, pms[0].total_free);
  for (int q = 0; q < nparts; q++)
  for (int d = 0; d < pms[q].ndomain; d++) {
    PartMesh *pm = &pms[q];
    DomMesh *dm = &pm->dm[d];
    w_i32(f, dm->nmp);
    w_i32(f, dm->nap);
    w_i32(f, dm->nel);
    fwrite(dm->nop, 4, dm->nel * dm->nd_elem, f);
    w_i32(f, dm->dbc_Axn0.nbc);
    fwrite(dm->dbc_Axn0.ibc, 4, dm->dbc_Axn0.nbc, f);
    w_i32(f, dm->ninbc);
    for (int i = 0; i < dm->ninbc; i++) {
      w_i32(f, dm->inbc[i].nfid);
      w_i32(f, dm->inbc[i].ln_part);
    }
    int *g = edge_gnid(pm, dm);
    fwrite(g, 4, dm->nmp, f);
    free(g);
  }
  fclose(f);
}

/* every part's subdomains, parts in order */
static void dump_solution(PartMesh *pms, int nparts) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s.sol", g_prefix);
  FILE *f = fopen(path, "wb");
  if (!f) return;
  int total = 0;
  for (int q = 0; q < nparts; q++) total += pms[q].ndomain;
  w_i32(f, total);
  for (int q = 0; q < nparts; q++) {
    PartMesh *pm = &pms[q];
    for (int d = 0; d < pm->ndomain; d++) {
      DomMesh *dm = &pm->dm[d];
      w_i32(f, dm->nmp);
      int *g = edge_gnid(pm, dm);
      fwrite(g, 4, dm->nmp, f);
      free(g);
      fwrite(dm->x_c, sizeof(Complex), dm->nmp, f);
    }
  }
  fclose(f);
}

/* The reference's element results of HDDM_post_dom_em_E
   (main/fullwave/fullwave.c:607-634), which hddm_solver_CS runs through the
   post_sp slot after the last solve: per subdomain its element count, the
   global element ids (seid2geid) and el_B_c, el_E_c, el_Je_c (3 Complex per
   element each). */
static void dump_post(PartMesh *pm, const char *suffix) {
  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s.%s", g_prefix, suffix);
  FILE *f = fopen(path, "wb");
  if (!f) return;
  w_i32(f, pm->ndomain);
  for (int d = 0; d < pm->ndomain; d++) {
    DomMesh *dm = &pm->dm[d];
    w_i32(f, dm->nel);
    fwrite(dm->seid2geid, 4, dm->nel, f);
    fwrite(dm->rvalue.el_B_c, sizeof(Complex), 3 * dm->nel, f);
    fwrite(dm->rvalue.el_E_c, sizeof(Complex), 3 * dm->nel, f);
    fwrite(dm->rvalue.el_Je_c, sizeof(Complex), 3 * dm->nel, f);
  }
  fclose(f);
}

/* HDDM_post_dom_em_E once more on the converged solution with the first
   entry of the Permittivity list (flag_i) and of the Conductor list (R_i)
   left out, so that those elements take the nu = 0 and sigma = 0 branches
   (fullwave.c:672-683).  The MTRL is a shallow copy; the model is unchanged. */
static void dump_post_dropped(PartMesh *pm) {
  MTRL m = pm->mtrl;
  if (m.nflag > 0) {
    m.nflag -= 1;
    m.flag_i += 1;
    m.flag_nu += 1;
  }
  if (m.nR > 0) {
    m.nR -= 1;
    m.R_i += 1;
    m.R_sigma += 1;
  }
  for (int d = 0; d < pm->ndomain; d++) HDDM_post_dom_em_E(&pm->dm[d], m);
  dump_post(pm, "post_drop");
}

int main(int argc, char **argv) {
  OPTIONS options;
  double t0 = t_now();
  const char *model_dir = argc > 1 ? argv[argc - 1] : ".";
  const char *out = getenv("FW_HARNESS_OUT");
  const char *dump = getenv("FW_HARNESS_DUMP");
  g_dump = dump ? atoi(dump) : 0;
  if (out)
    snprintf(g_prefix, sizeof(g_prefix), "%s", out);
  else
    snprintf(g_prefix, sizeof(g_prefix), "%s/ref", model_dir);

  hddm_time_Init();
  /* the solver selection main() hard-codes (main/fullwave/main.c:46-60) */
  options.solvopt.solver_dom = SOLVER_LU;
  options.solvopt.solver_pc = SOLVER_PC_ICC;
  options.solvopt.solver_eps = 1.0e-09;
  options.solvopt.solver_log = NO_NEED;
  options.solvopt.coJo_sol = SOLVER_CGMETHOD;
  options.solvopt.coJo_sol_pc = SOLVER_PC_ICC;
  options.solvopt.coJo_sol_log = NO_NEED;
  options.hddm_opt.hddm_solver = HDDM_COCG;
  options.hddm_opt.hddm_pc = HDDM_PC_DIAG;
  options.hddm_opt.hddm_log = NEED;
  options.hddm_opt.coJo_hddm_sol = HDDM_CGMETHOD;
  options.hddm_opt.coJo_hddm_pc = HDDM_PC_DIAG;
  options.hddm_opt.coJo_hddm_log = NEED;
  main_Init(argc, argv, &options);
  if (make_outdata_directory(options.datasw) > 0) return 1;
  if (make_calclog_directory(options.datasw) > 0) return 1;

  const char *main_mode = getenv("FW_HARNESS_MAIN");
  if (main_mode && atoi(main_mode) == 1) {
    /* main()'s own flow (main/fullwave/main.c:75-100): hddm_Init, then the
       correction-Jo pre-solve of every antenna */
    hddm_Init(&g_pm, options);
    hddm_sw.t_loop = -2;
    for (int i = 0; i < g_pm[0].mtrl.nantenna; i++) {
      hddm_sw.antenna = i;
#ifdef FW_HARNESS_GPU
      /* the pre-solve's slots on the GPU library */
      hddm_solver_RS(g_pm, options, set_hddm_func_correct_Jor_gpu);
      hddm_solver_RS(g_pm, options, set_hddm_func_correct_Joi_gpu);
#else
      hddm_solver_RS(g_pm, options, set_hddm_func_correct_Jor);
      hddm_solver_RS(g_pm, options, set_hddm_func_correct_Joi);
#endif
    }
    dump_jo(g_pm, nrepeat);
    dump_cojo(g_pm, nrepeat);
    /* FW_HARNESS_COJO_ONLY=1: stop after the pre-solve */
    const char *cojo_only = getenv("FW_HARNESS_COJO_ONLY");
    if (cojo_only && atoi(cojo_only) == 1) return 0;
  } else {
  /* hddm_Init (lib/hddm/make_PartMesh.c:58-117) in s-mode, calling
     make_PartMesh_FW directly: make_PartMesh's material check
     (make_MESH_check_flag_2nd, lib/fem/make_MESH.c:78-130) insists on an
     antenna definition, and synthetic models drive the solve through an edge
     current instead. */
    char fname[FILENAME_MAX];
    nstart = 0;
    nend = COM_GID.nparent;
    nrepeat = COM_GID.nparent;
    g_pm = (PartMesh *)Malloc(sizeof(PartMesh), nrepeat);
    for (int i = nstart, j = 0; i < nend; i++, j++) {
      init_PartMesh(&g_pm[j], options);
      make_modeldata_filename(fname, options.datasw, i);
      read_modeldata_file(fname, &g_pm[j], options);
    }
    make_mtrldat_filename(fname, options.datasw, 0);
    read_mtrldat_file(fname, &g_pm[0].mtrl, options);
    for (int i = 1; i < COM_GID.nparent; i++) Copy_MTRL(&g_pm[i].mtrl, g_pm[0].mtrl);
    make_PartMesh_FW(g_pm, options);
  }
  double t_init = t_now() - t0;
  load_sources(model_dir, &g_pm[0]);
  load_antennas(model_dir, &g_pm[0]);
  if (g_dump >= 1) dump_ints(g_pm, nrepeat);
  if (g_dump >= 2) {
    char path[FILENAME_MAX];
    snprintf(path, sizeof(path), "%s.aij", g_prefix);
    f_aij = fopen(path, "wb");
    snprintf(path, sizeof(path), "%s.fac", g_prefix);
    f_fac = fopen(path, "wb");
  }

  hddm_sw.t_loop = -2;
  hddm_sw.antenna = -1;
#ifdef FW_HARNESS_GPU
  hddm_gpu_set_edge_source(g_srcn, g_srcg, g_srcv);
#endif
  {
    char path[FILENAME_MAX];
#ifndef FW_HARNESS_GPU
    /* the residuals are read from the reference's own interface vectors */
    snprintf(path, sizeof(path), "%s.hist", g_prefix);
    f_hist = fopen(path, "wb");
#endif
    snprintf(path, sizeof(path), "%s.itimes", g_prefix);
    f_itimes = fopen(path, "wb");
  }
  double t1 = t_now();
  hddm_solver_CS(g_pm, options, set_hddm_func_harness);
  double t_solve = t_now() - t1;
  if (f_hist) fclose(f_hist);
  if (f_itimes) fclose(f_itimes);
  if (f_aij) fclose(f_aij);
  if (f_fac) fclose(f_fac);
  dump_solution(g_pm, nrepeat);
  if (g_dump >= 1) {
    dump_post(&g_pm[0], "post");
    dump_post_dropped(&g_pm[0]);
  }

  char path[FILENAME_MAX];
  snprintf(path, sizeof(path), "%s.json", g_prefix);
  FILE *f = fopen(path, "w");
  if (f) {
    fprintf(f,
            "{\"ndomain\": %d, \"total_free\": %d, \"iterations\": %d, \"t_init_s\": %.6f, "
            "\"t_assemble_s\": %.6f, \"t_first_s\": %.6f, \"t_iter_total_s\": %.6f, "
            "\"t_iter_count\": %d, \"t_last_s\": %.6f, \"t_solve_s\": %.6f}\n",
            g_pm[0].ndomain, g_pm[0].total_free, n_iter, t_init, t_assemble, t_first, t_iter_total,
            n_iter > 0 ? n_iter - 1 : 0, t_last, t_solve);
    fclose(f);
  }
  return 0;
}
