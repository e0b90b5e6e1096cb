/*
 * set_hddm_func_gpu.c -- the reference's plug-in table for the full-wave
 * HDDM solve (HDDM_FUNC, lib/std/types.h:629-730) with its subdomain and
 * interface slots on the B200 library (include/fwgpu.h).
 *
 * A maintainer of the reference builds this file with the reference's
 * headers and passes set_hddm_func_fullwave_gpu where main() passes
 * set_hddm_func_fullwave (main/fullwave/main.c:105):
 *
 *     hddm_solver_CS(pm, options, set_hddm_func_fullwave_gpu);
 *
 * The reference's driver (hddm_solver_CS, lib/hddm/hddm_solver.h:25-183, and
 * the s-mode loop of lib/hddm/hddm_solver_s.h) walks the table unchanged.
 * The library solves all parts and subdomains at once, so the slots the
 * driver calls once per subdomain do nothing, and the batched work sits in
 * the slots it calls once per step:
 *
 *   general_func_2nd   the library context from the PartMesh (mesh, material
 *                      flags, PEC wall, partition, element sources)
 *   iteration_s_1st    assembly, factors, first solves, first COCG step
 *                      (fwgpu_make_tmp_aij, fwgpu_solve_dom_1st,
 *                      fwgpu_iteration_s_1st)
 *   iteration_s        one interface iteration (fwgpu_iteration_s)
 *   solve_dom_last     the last solves, once per solve (fwgpu_solve_dom_last)
 *   get_result_sp      every subdomain's dm->x_c from the edge solution
 *   general_func_5th   the context released
 *
 * The loop stays the reference's: hddm_sw.status is set from the library's
 * COCG status after each step, and the driver's own hddm_max_loop test ends
 * the loop as before.  Every other slot (the post step, result files, PC
 * options) is the reference's own.  Errors of the library are reported the
 * reference's way: a message and exit (lib/std/errormessage.c).
 *
 * Every subdomain keeps the PartMesh's own local numbering (its apid and
 * mpid order), so the library's skyline profiles are the reference's.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "advfullwave_lib.h"
#include "libfem.h"
#include "libhddm.h"

#include "fullwave.h"
#include "fwgpu.h"

extern COM_GRP_ID COM_GID;
extern HDDM_SW hddm_sw;

/* the reference's entries this table keeps and calls through */
static void (*ref_general_func_2nd)(PartMesh *, HDDM_VEC *, OPTIONS, HDDM_Opt, SolvOpt) = NULL;
static void (*ref_general_func_5th)(PartMesh *, HDDM_VEC *, OPTIONS, HDDM_Opt, SolvOpt) = NULL;

static fwgpu_context *g_ctx = NULL;
static int g_last_done = 0;      /* the last solves of this solve have run */
static double *g_x = NULL;       /* edge solution, 2 doubles per edge */
static int *g_edge_of = NULL;    /* global node id of a mid-node -> library edge id (-1 else) */
static int g_n_gnid = 0;
/* extra edge currents given by the caller (mid-node global ids) */
static int g_nsrc = 0;
static int *g_src_gnid = NULL;
static double *g_src_val = NULL;

static void gpu_fail(const char *what, int rc) {
  fprintf(stderr, "set_hddm_func_fullwave_gpu: %s failed (%d): %s\n", what, rc, fwgpu_last_error());
  exit(1);
}

#define GPU_CALL(what, expr)          \
  do {                                \
    int rc_ = (expr);                 \
    if (rc_ != FWGPU_OK) gpu_fail(what, rc_); \
  } while (0)

void hddm_gpu_set_edge_source(int n, const int *mid_gnid, const double *re_im) {
  free(g_src_gnid);
  free(g_src_val);
  g_nsrc = n;
  g_src_gnid = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  g_src_val = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  if (n > 0) {
    memcpy(g_src_gnid, mid_gnid, sizeof(int) * n);
    memcpy(g_src_val, re_im, sizeof(double) * 2 * n);
  }
}

static int gnid_of(PartMesh *pm, DomMesh *dm, int snid) { return pm->pnid2gnid[dm->snid2pnid[snid]]; }

/* file order of the six mid-nodes (01,02,03,12,23,13) in the nop slots the
   reference leaves after make_MESH_change_nop: slots 4..7, then 9 and 8 */
static const int kMidSlot[6] = {4, 5, 6, 7, 9, 8};

static int read_volt(fwgpu_element_source *es, double **box, double **volt) {
  FILE *f = fopen("./MODEL/volt.dat", "r");
  char buf[256];
  int dg = 0;
  if (!f) return 0;
  if (fgets(buf, sizeof(buf), f)) sscanf(buf, "%d", &dg);
  if (dg > 0) {
    *box = (double *)calloc(6 * dg, sizeof(double));
    *volt = (double *)calloc(dg, sizeof(double));
    for (int i = 0; i < dg; i++) {
      for (int a = 0; a < 3; a++)
        if (fgets(buf, sizeof(buf), f)) sscanf(buf, "%lf %lf", &(*box)[6 * i + 2 * a], &(*box)[6 * i + 2 * a + 1]);
      if (fgets(buf, sizeof(buf), f)) sscanf(buf, "%lf", &(*volt)[i]);
    }
    es->n_gaps = dg;
    es->gap_box = *box;
    es->gap_volt = *volt;
  }
  fclose(f);
  return dg;
}

/* The library's mesh arrays built from the PartMesh after hddm_Init. */
typedef struct {
  int nv, ne, nt, nsub, ng;
  double *crd;
  int32_t *tv, *te, *flag, *sub, *vptr, *vord, *eptr, *eord;
  uint8_t *pec;
  int *vtx_of;  /* global node id -> library vertex, -1 for none */
  int *edge_of; /* global node id -> library edge, -1 for none */
} MeshArrays;

static void mesh_free(MeshArrays *a) {
  free(a->crd);
  free(a->tv);
  free(a->te);
  free(a->flag);
  free(a->sub);
  free(a->pec);
  free(a->vptr);
  free(a->vord);
  free(a->eptr);
  free(a->eord);
  free(a->vtx_of);
  free(a->edge_of);
  memset(a, 0, sizeof(*a));
}

/* Every part's subdomains, in part order, become the library's subdomains;
   vertices and edges are numbered in ascending global node id, and each
   subdomain keeps its own apid and mpid order. */
static void mesh_from_partmesh(PartMesh *pm, MeshArrays *A) {
  const int npart = COM_GID.nparent;
  int nsub = 0, nt = 0, maxg = -1;
  for (int q = 0; q < npart; q++)
    for (int d = 0; d < pm[q].ndomain; d++) {
      DomMesh *dm = &pm[q].dm[d];
      nsub++;
      nt += dm->nel;
      for (int a = 0; a < dm->nap; a++) {
        const int g = gnid_of(&pm[q], dm, dm->apid2snid[a]);
        if (g > maxg) maxg = g;
      }
      for (int m = 0; m < dm->nmp; m++) {
        const int g = gnid_of(&pm[q], dm, dm->mpid2snid[m]);
        if (g > maxg) maxg = g;
      }
    }
  /* vertices and edges numbered in ascending global node id */
  const int ng = maxg + 1;
  int *vtx_of = (int *)malloc(sizeof(int) * (ng > 0 ? ng : 1));
  int *edge_of = (int *)malloc(sizeof(int) * (ng > 0 ? ng : 1));
  for (int g = 0; g < ng; g++) vtx_of[g] = edge_of[g] = -1;
  for (int q = 0; q < npart; q++)
    for (int d = 0; d < pm[q].ndomain; d++) {
      DomMesh *dm = &pm[q].dm[d];
      for (int a = 0; a < dm->nap; a++) vtx_of[gnid_of(&pm[q], dm, dm->apid2snid[a])] = 0;
      for (int m = 0; m < dm->nmp; m++) edge_of[gnid_of(&pm[q], dm, dm->mpid2snid[m])] = 0;
    }
  int nv = 0, ne = 0;
  for (int g = 0; g < ng; g++) {
    if (vtx_of[g] == 0) vtx_of[g] = nv++;
    if (edge_of[g] == 0) edge_of[g] = ne++;
  }
  double *crd = (double *)calloc(3 * (size_t)(nv > 0 ? nv : 1), sizeof(double));
  int32_t *tv = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)(nt > 0 ? nt : 1));
  int32_t *te = (int32_t *)malloc(sizeof(int32_t) * 6 * (size_t)(nt > 0 ? nt : 1));
  int32_t *flag = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nt > 0 ? nt : 1));
  int32_t *sub = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nt > 0 ? nt : 1));
  uint8_t *pec = (uint8_t *)calloc(ne > 0 ? ne : 1, 1);
  /* each subdomain's local order: its apid and mpid order */
  int32_t *vptr = (int32_t *)malloc(sizeof(int32_t) * (nsub + 1));
  int32_t *eptr = (int32_t *)malloc(sizeof(int32_t) * (nsub + 1));
  vptr[0] = eptr[0] = 0;
  {
    int k = 0;
    for (int q = 0; q < npart; q++)
      for (int d = 0; d < pm[q].ndomain; d++, k++) {
        vptr[k + 1] = vptr[k] + pm[q].dm[d].nap;
        eptr[k + 1] = eptr[k] + pm[q].dm[d].nmp;
      }
  }
  int32_t *vord = (int32_t *)malloc(sizeof(int32_t) * (vptr[nsub] > 0 ? vptr[nsub] : 1));
  int32_t *eord = (int32_t *)malloc(sizeof(int32_t) * (eptr[nsub] > 0 ? eptr[nsub] : 1));
  int t = 0, s = 0;
  for (int q = 0; q < npart; q++)
    for (int d = 0; d < pm[q].ndomain; d++, s++) {
      DomMesh *dm = &pm[q].dm[d];
      for (int a = 0; a < dm->nap; a++) {
        const int v = vtx_of[gnid_of(&pm[q], dm, dm->apid2snid[a])];
        for (int k = 0; k < 3; k++) crd[3 * v + k] = dm->crd[3 * a + k];
        vord[vptr[s] + a] = v;
      }
      for (int m = 0; m < dm->nmp; m++) eord[eptr[s] + m] = edge_of[gnid_of(&pm[q], dm, dm->mpid2snid[m])];
      for (int el = 0; el < dm->nel; el++, t++) {
        const int *ne_ = &dm->nop[el * dm->nd_elem];
        for (int i = 0; i < 4; i++) tv[4 * t + i] = vtx_of[gnid_of(&pm[q], dm, dm->apid2snid[ne_[i]])];
        for (int i = 0; i < 6; i++) te[6 * t + i] = edge_of[gnid_of(&pm[q], dm, dm->mpid2snid[ne_[kMidSlot[i]]])];
        flag[t] = dm->flag[el];
        sub[t] = s;
      }
      /* the PEC wall: Dirichlet mid-nodes that are not interface DOFs */
      char *is_if = (char *)calloc(dm->nmp > 0 ? dm->nmp : 1, 1);
      for (int i = 0; i < dm->ninbc; i++)
        if (dm->inbc[i].nfid >= 0 && dm->inbc[i].nfid < dm->nmp) is_if[dm->inbc[i].nfid] = 1;
      for (int i = 0; i < dm->dbc_Axn0.nbc; i++) {
        const int m = dm->dbc_Axn0.ibc[i];
        if (m >= 0 && m < dm->nmp && !is_if[m]) pec[edge_of[gnid_of(&pm[q], dm, dm->mpid2snid[m])]] = 1;
      }
      free(is_if);
    }
  A->nv = nv;
  A->ne = ne;
  A->nt = nt;
  A->nsub = nsub;
  A->ng = ng;
  A->crd = crd;
  A->tv = tv;
  A->te = te;
  A->flag = flag;
  A->sub = sub;
  A->pec = pec;
  A->vptr = vptr;
  A->vord = vord;
  A->eptr = eptr;
  A->eord = eord;
  A->vtx_of = vtx_of;
  A->edge_of = edge_of;
}

static fwgpu_mesh mesh_view(const MeshArrays *a) {
  fwgpu_mesh m = {a->nv, a->crd, a->nt, a->tv, a->te, a->flag, a->ne, a->pec, a->nsub, a->sub,
                  a->vptr, a->vord, a->eptr, a->eord};
  return m;
}

/* The library context from the PartMesh after hddm_Init. */
static void gpu_general_func_2nd(PartMesh *pm, HDDM_VEC *hv, OPTIONS options, HDDM_Opt hddm_opt, SolvOpt solvopt) {
  if (ref_general_func_2nd) ref_general_func_2nd(pm, hv, options, hddm_opt, solvopt);
  const int npart = COM_GID.nparent;
  MeshArrays A;
  mesh_from_partmesh(pm, &A);
  const int nv = A.nv, ne = A.ne;
  const int *vtx_of = A.vtx_of;
  /* the edge map outlives the mesh arrays: sources and results use it */
  g_edge_of = A.edge_of;
  g_n_gnid = A.ng;
  A.edge_of = NULL;
  const MTRL *mt = &pm[0].mtrl;
  fwgpu_mesh mesh = mesh_view(&A);
  fwgpu_material mat = {mt->nflag, mt->flag_i, mt->flag_nu, mt->nR, mt->R_i, mt->R_sigma, mt->antenna_omega};
  fwgpu_options o;
  memset(&o, 0, sizeof(o));
  o.hddm_eps = hddm_opt.hddm_eps;
  /* the driver ends the loop at its own hddm_max_loop */
  o.hddm_max_loop = 0x7fffffff;
  o.precision = getenv("FW_GPU_FP32_IR") ? FWGPU_PREC_FP32_IR : FWGPU_PREC_FP64;
  o.ir_max_steps = 1;
  o.graph_iterations = 1;
  GPU_CALL("fwgpu_create", fwgpu_create(&mesh, &mat, &o, &g_ctx));

  /* element sources: volt.dat gaps, else the antennas' vertex currents */
  fwgpu_element_source es;
  memset(&es, 0, sizeof(es));
  double *box = NULL, *volt = NULL, *jo = NULL, *jor = NULL;
  int32_t *aflag = NULL;
  if (read_volt(&es, &box, &volt) == 0 && mt->nantenna > 0) {
    const int na = mt->nantenna;
    aflag = (int32_t *)malloc(sizeof(int32_t) * na);
    jo = (double *)calloc(3 * (size_t)nv * na, sizeof(double));
    jor = (double *)calloc(3 * (size_t)nv * na, sizeof(double));
    for (int k = 0; k < na; k++) aflag[k] = mt->antenna_def[k].flag;
    for (int q = 0; q < npart; q++)
      for (int d = 0; d < pm[q].ndomain; d++) {
        DomMesh *dm = &pm[q].dm[d];
        if (!dm->antenna) continue;
        for (int k = 0; k < na; k++) {
          const ANTENNA *an = &dm->antenna[k];
          if (!an->enf || !an->Jo || !an->Jor) continue;
          for (int a = 0; a < dm->nap; a++) {
            const int e = an->enf[a];
            if (e < 0) continue;
            const size_t v = (size_t)k * nv + vtx_of[gnid_of(&pm[q], dm, dm->apid2snid[a])];
            for (int j = 0; j < 3; j++) {
              jo[3 * v + j] = an->Jo[3 * e + j];
              jor[3 * v + j] = an->Jor[3 * e + j];
            }
          }
        }
      }
    es.n_antennas = na;
    es.antenna_flag = aflag;
    es.antenna_Jo = jo;
    es.antenna_Jor = jor;
  }
  if (es.n_gaps > 0 || es.n_antennas > 0) GPU_CALL("fwgpu_set_element_source", fwgpu_set_element_source(g_ctx, &es));
  free(box);
  free(volt);
  free(jo);
  free(jor);
  free(aflag);
  mesh_free(&A);
  g_x = (double *)calloc(2 * (size_t)(ne > 0 ? ne : 1), sizeof(double));
  g_last_done = 0;
}

static void gpu_noop_dom(DomMesh *dm, MTRL mtrl) {
  (void)dm;
  (void)mtrl;
}
static void gpu_noop_solve_1st(DomMesh *dm, HDDM_Opt o, SolvOpt so, int (*s)(AIJ_MAT *, SolvOpt, FILE *),
                               HDDM_DOM_VEC *v, int (*pc)(TMP_AIJ, HDDM_DOM_VEC *), FILE *fp) {
  (void)dm, (void)o, (void)so, (void)s, (void)v, (void)pc, (void)fp;
}
static void gpu_noop_solve(DomMesh *dm, SolvOpt so, int (*s)(AIJ_MAT *, SolvOpt, FILE *), HDDM_DOM_VEC *v,
                           FILE *fp) {
  (void)dm, (void)so, (void)s, (void)v, (void)fp;
}
static void gpu_noop_com(HDDM_VEC *hv, HDDM_DOM_VEC v, DomMesh dm, HDDM_Opt o) {
  (void)hv, (void)v, (void)dm, (void)o;
}
static void gpu_noop_renewal(DomMesh *dm, HDDM_VEC hv) {
  (void)dm, (void)hv;
}

static void set_status(int32_t st) { hddm_sw.status = st != 0 ? __HDDM_SW_LAST__ : __HDDM_SW_ITERATION__; }

static void gpu_iteration_s_1st(PartMesh *pm, HDDM_VEC *hv, HDDM_Opt o, int (*setPC)(HDDM_VEC *),
                                void (*gatherPC_s)(OPinfo **, HDDM_VEC *)) {
  (void)pm, (void)hv, (void)o, (void)setPC, (void)gatherPC_s;
  fwgpu_source src = {0, NULL, NULL};
  int32_t *edge = NULL;
  if (g_nsrc > 0) {
    edge = (int32_t *)malloc(sizeof(int32_t) * g_nsrc);
    for (int i = 0; i < g_nsrc; i++) {
      const int g = g_src_gnid[i];
      edge[i] = (g >= 0 && g < g_n_gnid) ? g_edge_of[g] : -1;
      if (edge[i] < 0) gpu_fail("edge source on a node that is no mid-node", FWGPU_ERR_ARG);
    }
    src.n_entries = g_nsrc;
    src.edge = edge;
    src.value = g_src_val;
  }
  int32_t st = 0;
  GPU_CALL("fwgpu_make_tmp_aij", fwgpu_make_tmp_aij(g_ctx, &src));
  GPU_CALL("fwgpu_solve_dom_1st", fwgpu_solve_dom_1st(g_ctx));
  GPU_CALL("fwgpu_iteration_s_1st", fwgpu_iteration_s_1st(g_ctx, &st));
  free(edge);
  set_status(st);
  g_last_done = 0;
}

static void gpu_iteration_s(PartMesh *pm, HDDM_VEC *hv, HDDM_Opt o, int (*setPC)(HDDM_VEC *)) {
  (void)pm, (void)hv, (void)o, (void)setPC;
  int32_t st = 0;
  GPU_CALL("fwgpu_iteration_s", fwgpu_iteration_s(g_ctx, &st));
  set_status(st);
}

/* the last solves of every subdomain at once, on the first subdomain's call */
static void gpu_solve_dom_last(DomMesh *dm, SolvOpt so, int (*s)(AIJ_MAT *, SolvOpt, FILE *), HDDM_DOM_VEC *v,
                               FILE *fp) {
  (void)dm, (void)so, (void)s, (void)v, (void)fp;
  if (g_last_done) return;
  GPU_CALL("fwgpu_solve_dom_last", fwgpu_solve_dom_last(g_ctx));
  GPU_CALL("fwgpu_get_edge_solution", fwgpu_get_edge_solution(g_ctx, g_x));
  g_last_done = 1;
}

/* every subdomain's local solution, as HDDM_get_result_sp_fullwave leaves it
   (main/fullwave/fullwave.c:500-514) */
static void gpu_get_result_sp(PartMesh *pm) {
  for (int d = 0; d < pm->ndomain; d++) {
    DomMesh *dm = &pm->dm[d];
    Complex *x = (Complex *)Calloc(sizeof(Complex), dm->nmp > 0 ? dm->nmp : 1);
    for (int m = 0; m < dm->nmp; m++) {
      const int e = g_edge_of[gnid_of(pm, dm, dm->mpid2snid[m])];
      x[m].re = g_x[2 * e];
      x[m].im = g_x[2 * e + 1];
    }
    dm->x_c = x;
  }
}

static void gpu_general_func_5th(PartMesh *pm, HDDM_VEC *hv, OPTIONS options, HDDM_Opt hddm_opt, SolvOpt solvopt) {
  if (g_ctx) fwgpu_destroy(g_ctx);
  g_ctx = NULL;
  if (ref_general_func_5th) ref_general_func_5th(pm, hv, options, hddm_opt, solvopt);
}

void set_hddm_func_fullwave_gpu(HDDM_FUNC *f, OPTIONS options) {
  set_hddm_func_fullwave(f, options);
  ref_general_func_2nd = f->general_func_2nd;
  ref_general_func_5th = f->general_func_5th;
  f->general_func_2nd = gpu_general_func_2nd;
  f->general_func_5th = gpu_general_func_5th;
  f->make_TMP_AIJ = gpu_noop_dom;
  f->solve_dom_1st = gpu_noop_solve_1st;
  f->COM_res_sp_1st = gpu_noop_com;
  f->iteration_s_1st = gpu_iteration_s_1st;
  f->renewal_bc_sp = gpu_noop_renewal;
  f->solve_dom = gpu_noop_solve;
  f->COM_res_sp = gpu_noop_com;
  f->iteration_s = gpu_iteration_s;
  f->solve_dom_last = gpu_solve_dom_last;
  f->get_result_sp = gpu_get_result_sp;
}

/* ------------------------------------------------------------------------
 * The correction-Jo pre-solve of main() (main/fullwave/main.c:92-98), the
 * same way:
 *
 *     hddm_solver_RS(pm, options, set_hddm_func_correct_Jor_gpu);
 *     hddm_solver_RS(pm, options, set_hddm_func_correct_Joi_gpu);
 *
 * in place of set_hddm_func_correct_Jor / _Joi
 * (lib/hddm/set_hddm_func.c:195-233).  general_func_2nd keeps the
 * reference's own entry first, which leaves the pass's current in every
 * subdomain's antenna->Jo (HDDM_general_func_make_Jo_correct_Jo, :769-888),
 * and then builds the antenna's library context (fwgpu_cojo_create) with
 * that current.  The iteration slots run the library's batched steps, and
 * get_result_sp leaves each subdomain's potentials in antenna->Ihr (first
 * pass) or antenna->Ihi (second), as HDDM_get_result_sp_correct_Jor / _Joi
 * (:626-667) do.  The reference's own init_bc allocates dbc.vbc, which
 * get_result_sp releases as the reference's does.
 */
static fwgpu_context *g_cj = NULL;
static int g_cj_last_done = 0;
static double *g_phi = NULL;    /* potential, 2 doubles per library vertex */
static int *g_cj_vtx_of = NULL; /* global node id -> library vertex */
static int g_cj_pass = -1;      /* -1: Ihr (real part of the current), -2: Ihi */
static void (*ref_cojo_2nd)(PartMesh *, HDDM_VEC *, OPTIONS, HDDM_Opt, SolvOpt) = NULL;
static void (*ref_cojo_5th)(PartMesh *, HDDM_VEC *, OPTIONS, HDDM_Opt, SolvOpt) = NULL;

static void cojo_general_func_2nd(PartMesh *pm, HDDM_VEC *hv, OPTIONS options, HDDM_Opt hddm_opt, SolvOpt solvopt) {
  if (ref_cojo_2nd) ref_cojo_2nd(pm, hv, options, hddm_opt, solvopt);
  const int npart = COM_GID.nparent;
  const int k = hddm_sw.antenna;
  MeshArrays A;
  mesh_from_partmesh(pm, &A);
  const int nv = A.nv;
  /* the pass's current per vertex, and the vertex Dirichlet nodes of the
     antenna: its Dirichlet list before the interface DOFs (a subdomain's
     pinned DOF 0 is one too, and is held at zero the same way) */
  double *J = (double *)calloc(3 * (size_t)(nv > 0 ? nv : 1), sizeof(double));
  uint8_t *pecv = (uint8_t *)calloc(nv > 0 ? nv : 1, 1);
  for (int q = 0; q < npart; q++)
    for (int d = 0; d < pm[q].ndomain; d++) {
      DomMesh *dm = &pm[q].dm[d];
      ANTENNA *an = dm->antenna ? &dm->antenna[k] : NULL;
      if (!an || !an->enf || an->nf <= 0) continue;
      int *v_of = (int *)malloc(sizeof(int) * an->nf);
      for (int a = 0; a < dm->nap; a++)
        if (an->enf[a] >= 0) v_of[an->enf[a]] = A.vtx_of[gnid_of(&pm[q], dm, dm->apid2snid[a])];
      for (int i = 0; i < an->dbc.nbc - an->ninbc; i++) pecv[v_of[an->dbc.ibc[i]]] = 1;
      if (an->Jo)
        for (int e = 0; e < an->nf; e++)
          for (int j = 0; j < 3; j++) J[3 * (size_t)v_of[e] + j] = an->Jo[3 * e + j];
      free(v_of);
    }
  fwgpu_mesh mesh = mesh_view(&A);
  fwgpu_options o;
  memset(&o, 0, sizeof(o));
  o.hddm_eps = hddm_opt.hddm_eps;
  o.hddm_max_loop = 0x7fffffff; /* the driver ends the loop at its own hddm_max_loop */
  o.precision = FWGPU_PREC_FP64;
  o.ir_max_steps = 1;
  o.graph_iterations = 1;
  GPU_CALL("fwgpu_cojo_create", fwgpu_cojo_create(&mesh, pm[0].mtrl.antenna_def[k].flag, pecv, &o, &g_cj));
  GPU_CALL("fwgpu_cojo_set_current", fwgpu_cojo_set_current(g_cj, J));
  free(J);
  free(pecv);
  g_phi = (double *)calloc(2 * (size_t)(nv > 0 ? nv : 1), sizeof(double));
  g_cj_vtx_of = A.vtx_of;
  A.vtx_of = NULL;
  mesh_free(&A);
  g_cj_last_done = 0;
}

static void cojo_iteration_s_1st(PartMesh *pm, HDDM_VEC *hv, HDDM_Opt o, int (*setPC)(HDDM_VEC *),
                                 void (*gatherPC_s)(OPinfo **, HDDM_VEC *)) {
  (void)pm, (void)hv, (void)o, (void)setPC, (void)gatherPC_s;
  int32_t st = 0;
  GPU_CALL("fwgpu_make_tmp_aij", fwgpu_make_tmp_aij(g_cj, NULL));
  GPU_CALL("fwgpu_solve_dom_1st", fwgpu_solve_dom_1st(g_cj));
  GPU_CALL("fwgpu_iteration_s_1st", fwgpu_iteration_s_1st(g_cj, &st));
  set_status(st);
  g_cj_last_done = 0;
}

static void cojo_iteration_s(PartMesh *pm, HDDM_VEC *hv, HDDM_Opt o, int (*setPC)(HDDM_VEC *)) {
  (void)pm, (void)hv, (void)o, (void)setPC;
  int32_t st = 0;
  GPU_CALL("fwgpu_iteration_s", fwgpu_iteration_s(g_cj, &st));
  set_status(st);
}

static void cojo_solve_dom_last(DomMesh *dm, SolvOpt so, int (*s)(AIJ_MAT *, SolvOpt, FILE *), HDDM_DOM_VEC *v,
                                FILE *fp) {
  (void)dm, (void)so, (void)s, (void)v, (void)fp;
  if (g_cj_last_done) return;
  GPU_CALL("fwgpu_solve_dom_last", fwgpu_solve_dom_last(g_cj));
  GPU_CALL("fwgpu_get_edge_solution", fwgpu_get_edge_solution(g_cj, g_phi));
  g_cj_last_done = 1;
}

static void cojo_get_result_sp(PartMesh *pm) {
  const int k = hddm_sw.antenna;
  for (int d = 0; d < pm->ndomain; d++) {
    DomMesh *dm = &pm->dm[d];
    ANTENNA *an = dm->antenna ? &dm->antenna[k] : NULL;
    if (!an) continue;
    if (an->enf && an->nf > 0) {
      double *ih = (double *)Malloc(sizeof(double), an->nf);
      for (int a = 0; a < dm->nap; a++)
        if (an->enf[a] >= 0) ih[an->enf[a]] = g_phi[2 * (size_t)g_cj_vtx_of[gnid_of(pm, dm, dm->apid2snid[a])]];
      if (g_cj_pass == -1)
        an->Ihr = ih;
      else
        an->Ihi = ih;
    }
    if (an->dbc.vbc) {
      Free(sizeof(double) * an->dbc.nbc, an->dbc.vbc);
      an->dbc.vbc = NULL;
    }
  }
}

static void cojo_general_func_5th(PartMesh *pm, HDDM_VEC *hv, OPTIONS options, HDDM_Opt hddm_opt, SolvOpt solvopt) {
  if (g_cj) fwgpu_destroy(g_cj);
  g_cj = NULL;
  free(g_phi);
  free(g_cj_vtx_of);
  g_phi = NULL;
  g_cj_vtx_of = NULL;
  if (ref_cojo_5th) ref_cojo_5th(pm, hv, options, hddm_opt, solvopt);
}

static void cojo_table(HDDM_FUNC *f, int pass) {
  g_cj_pass = pass;
  ref_cojo_2nd = f->general_func_2nd;
  ref_cojo_5th = f->general_func_5th;
  f->general_func_2nd = cojo_general_func_2nd;
  f->general_func_5th = cojo_general_func_5th;
  f->make_TMP_AIJ = gpu_noop_dom;
  f->solve_dom_1st = gpu_noop_solve_1st;
  f->COM_res_sp_1st = gpu_noop_com;
  f->iteration_s_1st = cojo_iteration_s_1st;
  f->renewal_bc_sp = gpu_noop_renewal;
  f->solve_dom = gpu_noop_solve;
  f->COM_res_sp = gpu_noop_com;
  f->iteration_s = cojo_iteration_s;
  f->solve_dom_last = cojo_solve_dom_last;
  f->get_result_sp = cojo_get_result_sp;
}

void set_hddm_func_correct_Jor_gpu(HDDM_FUNC *f, OPTIONS options) {
  set_hddm_func_correct_Jor(f, options);
  cojo_table(f, -1);
}

void set_hddm_func_correct_Joi_gpu(HDDM_FUNC *f, OPTIONS options) {
  set_hddm_func_correct_Joi(f, options);
  cojo_table(f, -2);
}
