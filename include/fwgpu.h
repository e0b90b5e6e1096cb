/*
 * fwgpu.h -- C ABI of the B200 HDDM hot path of ADVENTURE_FullWave.
 *
 * One context holds every part and subdomain of a full-wave HDDM problem
 * resident on one GPU.  The reference's per-subdomain loops over
 * (part, subdomain) in lib/hddm/hddm_solver_s.h become one batched call each;
 * every entry point below replaces one slot of the reference's plug-in table
 * HDDM_FUNC (lib/std/types.h:629-730) as filled by set_hddm_func_fullwave
 * (main/fullwave/fullwave.c:23-146), or the driver that walks it
 * (hddm_solver_CS, lib/hddm/hddm_solver.h:25-183).
 *
 * Conventions
 *   - plain C types only; complex numbers are interleaved (re, im) doubles,
 *     the layout of the reference's Complex (lib/std/types.h).
 *   - every function returns FWGPU_OK (0) or a negative FWGPU_ERR_* code and
 *     never exits the process (the reference calls emessage()/exit()).
 *   - the caller owns every buffer passed in; the library owns device state
 *     behind the opaque context.  A context is used by one host thread at a
 *     time and runs on its own CUDA stream.
 *   - there is no CPU fallback: without a CUDA device every call that needs
 *     the GPU returns FWGPU_ERR_CUDA.
 */
#ifndef FWGPU_H
#define FWGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FWGPU_ABI_VERSION 4

enum {
  FWGPU_OK = 0,
  FWGPU_ERR_ARG = -1,           /* invalid argument or inconsistent sizes */
  FWGPU_ERR_CUDA = -2,          /* CUDA runtime error or no device */
  FWGPU_ERR_STATE = -3,         /* call out of order (e.g. solve before factor) */
  FWGPU_ERR_NOT_CONVERGED = -4, /* COCG hit hddm_max_loop before hddm_eps */
  FWGPU_ERR_BREAKDOWN = -5,     /* zero or non-finite pivot in a subdomain factor */
  FWGPU_ERR_NOMEM = -6,         /* device allocation failed */
  FWGPU_ERR_MESH = -7,          /* degenerate or negatively oriented element */
  FWGPU_ERR_NONFINITE = -8,     /* the interface residual or (r, z) became NaN or infinite (e.g. a
                                   non-finite right-hand side); the loop stopped at once, where the
                                   reference would run on to hddm_max_loop */
  FWGPU_ERR_TIMEOUT = -9        /* a subdomain solve gave up waiting for one of its staged copies
                                   (every wait on the device is bounded); the solution is invalid */
};

/* precision of the subdomain factors */
enum {
  FWGPU_PREC_FP64 = 0,    /* factor stored and applied in complex FP64 (the reference) */
  FWGPU_PREC_FP32_IR = 1  /* factor stored and applied in complex FP32, FP64 iterative
                             refinement of every subdomain solve */
};

/* Model input: the fullwave driver's mesh, material flags, PEC wall and
 * partition, i.e. what lib/hddm/make_PartMesh.c:58-117 (hddm_Init) reads
 * from the part files, for one part.  Global numbering: vertices
 * 0..n_vertices-1, edges 0..n_edges-1. */
typedef struct {
  int32_t n_vertices;
  const double *vertex_crd;   /* 3*n_vertices */
  int32_t n_tets;
  const int32_t *tet_vertices; /* 4*n_tets, positively oriented (tet_Volume6 > 0) */
  const int32_t *tet_edges;    /* 6*n_tets global edge ids in file order 01,02,03,12,23,13 */
  const int32_t *tet_flag;     /* n_tets material flags */
  int32_t n_edges;
  const uint8_t *pec_edge;     /* n_edges, 1 = edge on the PEC wall (DirichletBCs_Axn0) */
  int32_t n_subdomains;
  const int32_t *sub_of_tet;   /* n_tets, subdomain of each element */
  /* Optional (all four NULL: ascending global id in every subdomain): each
   * subdomain's own local order, the node order (snid) of the reference's
   * part files.  The reference numbers a subdomain's vertices and then its
   * mid-nodes by their rank in that order (make_MESH_make_ap,
   * make_MESH_change_ap, lib/fem/make_MESH.c:237-272,539-552), which sets
   * the skyline profiles and with them the factors' rounding.  Subdomain s
   * lists its vertices in sub_vertex_order[sub_vertex_ptr[s] ..
   * sub_vertex_ptr[s+1]) and its edges in sub_edge_order[sub_edge_ptr[s] ..
   * sub_edge_ptr[s+1]); each list must hold every vertex (edge) of the
   * subdomain's elements exactly once. */
  const int32_t *sub_vertex_ptr;   /* n_subdomains+1 */
  const int32_t *sub_vertex_order; /* global vertex ids */
  const int32_t *sub_edge_ptr;     /* n_subdomains+1 */
  const int32_t *sub_edge_order;   /* global edge ids */
} fwgpu_mesh;

/* Material table: the reference's MTRL (lib/std/types.h:257-279) as read
 * from mtrl.dat by read_mtrldat_file (lib/std/fileio.c:3474-3572). */
typedef struct {
  int32_t n_eps;
  const int32_t *eps_flag;   /* Permittivity flags */
  const double *eps;         /* absolute permittivity [F/m] per flag */
  int32_t n_sigma;
  const int32_t *sigma_flag; /* Conductor flags */
  const double *sigma;       /* conductivity [S/m] per flag */
  double omega;              /* AntennaOmega [rad/s] */
} fwgpu_material;

/* Right-hand side: edge currents added to the assembled right-hand side of
 * the lowest-numbered subdomain holding each edge (after any element source,
 * fwgpu_set_element_source). */
typedef struct {
  int32_t n_entries;
  const int32_t *edge;     /* global edge ids */
  const double *value;     /* 2*n_entries (re, im) */
} fwgpu_source;

/* Element sources of the right-hand side: the two inputs of the element
 * routine tet_MakeElement_EM_E (lib/fem/make_elem_em.c:66-330), which the
 * reference selects by the first line dg of ./MODEL/volt.dat.
 *   n_gaps > 0  delta-gap voltages (dg > 0, :302-329): every element with a
 *               vertex inside a gap box (bounds inclusive; a later gap wins
 *               for a vertex in several) gets be_i = (sigma omega) *
 *               sum_j (0, dV) gs_ij, gs = tetNedelec_gradside
 *               (lib/fem/tetrahedral.c:645-661); the antennas are ignored.
 *   n_gaps = 0  antenna currents (dg = 0, :271-300): every element whose flag
 *               is an antenna's flag (the first match) gets
 *               be = tetNedelec_JoA_Complex (tetrahedral.c:794-858) of the
 *               vertex currents Joe = (-Jo, -Jor) of that antenna.
 * The element vectors are summed into each subdomain's right-hand side in
 * element order (SetFe, aij_matrix_func.h:327-338); an fwgpu_source passed
 * to make_tmp_aij / solve / resolve is added after them. */
typedef struct {
  int32_t n_gaps;
  const double *gap_box;        /* 6*n_gaps: x0 x1 y0 y1 z0 z1 per gap (volt.dat) */
  const double *gap_volt;       /* n_gaps: dV per gap */
  int32_t n_antennas;           /* mtrl.nantenna */
  const int32_t *antenna_flag;  /* n_antennas: antenna_def[k].flag */
  const double *antenna_Jo;     /* 3*n_vertices per antenna (k-major): antenna[k].Jo (x, y, z) per vertex */
  const double *antenna_Jor;    /* same layout: antenna[k].Jor */
} fwgpu_element_source;
typedef struct {
  double hddm_eps;       /* -hddm-eps, max-norm relative residual (default 1e-3) */
  int32_t hddm_max_loop; /* -hddm-max-loop (default 4000) */
  int32_t precision;     /* FWGPU_PREC_* */
  int32_t ir_max_steps;  /* FP32_IR: refinement steps per subdomain solve (>=1) */
  double ir_tol;         /* FP32_IR: stop refining when the subdomain residual drops below
                            ir_tol * |rhs| (0 = always ir_max_steps) */
  int32_t graph_iterations; /* COCG iterations captured per CUDA graph launch */
  int32_t device;        /* CUDA device ordinal */
  int32_t solve_kernel;  /* FWGPU_SOLVE_*: batched subdomain-solve kernel (0 = timed choice) */
  int32_t stage_cap;     /* WARP kernel: envelope elements per staging buffer (0 = timed choice) */
  double ir_relax;       /* FP32_IR: interface iterations refine only while the COCG relative
                            residual is above ir_relax (0 = always); the first and last
                            subdomain solves always refine */
  int32_t shard_begin;   /* sharded solve: this context solves subdomains [shard_begin, shard_end) */
  int32_t shard_end;     /* (0, 0 = every subdomain, unsharded); a given range, even all of them,
                            makes a sharded context: drive it with the fwgpu_shard_* calls */
  int32_t stage_warps;   /* WARP kernel: warps sharing a subdomain's sweeps, 1, 2 or 4 (0 = timed choice) */
  int32_t stall_copy_test; /* test hook, 0 in normal use: 1 makes the staged subdomain solves' first wait
                              for a copy poll a barrier that nothing completes, give up after a few polls
                              and raise FWGPU_ERR_TIMEOUT (each CTA still waits for its copies in flight
                              before it exits) */
} fwgpu_options;

/* Batched subdomain-solve kernels.  AUTO runs the WARP kernel (FP64
 * factors) or the BLOCKINV kernel (FP32 factors) at the staging capacity
 * that a rule on the envelope gives, and times 1, 2 and 4 warps per
 * subdomain, which sum in the same order; WARP also times its staging
 * capacities, which changes the order of the sums. */
#define FWGPU_SOLVE_AUTO 0
#define FWGPU_SOLVE_WARP 1   /* one warp per subdomain, vectors in shared memory */
#define FWGPU_SOLVE_CTA 2    /* one 256-thread CTA per subdomain */
#define FWGPU_SOLVE_GLOBAL 3 /* one warp per subdomain, vectors in global memory (any size) */
#define FWGPU_SOLVE_BLOCKINV 4 /* the WARP kernel on a second layout of the factor: each row block's own
                                  triangle stored as its inverse, applied as a product */

typedef struct fwgpu_context fwgpu_context;

/* Sizes a caller needs to allocate result buffers and to compute the
 * roofline of the substitution kernels. */
typedef struct {
  int32_t n_subdomains;
  int32_t total_free;       /* interface DOFs ("DOF on interface", hddm_solver.h:90) */
  int64_t total_dofs;       /* sum over subdomains of local edge DOFs */
  int64_t total_interior;   /* sum of non-Dirichlet local DOFs */
  int64_t nlen_reference;   /* sum of the reference's skyline lengths (advlas_skyline.c:24) */
  int64_t nlen_interior;    /* sum of stored interior envelope lengths */
  int64_t nnz_lower;        /* sum of stored lower-triangle entries of the assembled matrices */
  int64_t nnz_interface_rows; /* entries of the interface-row operator used per iteration */
  int64_t nnz_coupling;     /* entries of the interior-interface coupling used per iteration */
  int64_t nnz_interior;     /* entries of the interior operator used by refinement */
  int64_t total_iface_slots; /* sum over subdomains of interface DOFs */
  int32_t max_local_dofs;
  int32_t max_interior;
} fwgpu_sizes;

typedef struct {
  int32_t iterations;      /* COCG iterations done (hddm_sw.loop - 1 at exit) */
  int32_t converged;       /* 1 if resi < hddm_eps */
  double initial_norm;     /* max|r0| ("# Norm", hddm_solver_s.h:205) */
  double final_resi;       /* max|r|/max|r0| at exit */
  double final_resi_l2;    /* ||r||_2/||r0||_2 at exit */
  double t_setup_ms;       /* assembly + factor + first solve, device time */
  double t_iterate_ms;     /* COCG loop, device time */
  double t_last_ms;        /* final subdomain solves, device time */
  int64_t kernel_launches; /* kernels this library launched for the call */
  int32_t solve_kernel;    /* FWGPU_SOLVE_* used for the subdomain solves */
  int32_t stage_cap;       /* WARP kernel: envelope elements per staging buffer, else 0 */
  int32_t stage_warps;     /* WARP kernel: warps per subdomain, else 0 */
  int32_t reserved;
} fwgpu_result;

/* -- lifecycle ----------------------------------------------------------- */

/* Builds every subdomain's local numbering, Dirichlet list and interface maps
 * on the host (make_PartMesh_FW, lib/hddm/make_PartMesh.c:1201-1241, with
 * make_PartMesh_FW_TetQ :1628-1707 and the inner-BC renumbering :158-858 for
 * one part) and uploads mesh and material to the device. */
int fwgpu_create(const fwgpu_mesh *mesh, const fwgpu_material *mtrl, const fwgpu_options *opts,
                 fwgpu_context **out);
int fwgpu_destroy(fwgpu_context *ctx);
int fwgpu_get_sizes(const fwgpu_context *ctx, fwgpu_sizes *sizes);
/* Last CUDA/library error as text (never NULL). */
const char *fwgpu_last_error(void);
int fwgpu_abi_version(void);

/* -- host-only integer setup --------------------------------------------- */

/* The integer part of fwgpu_create without any device work:
 * make_PartMesh_FW for one part (lib/hddm/make_PartMesh.c:1201-1241).  Lets a
 * host without a GPU inspect the subdomain numbering. */
typedef struct fwgpu_partition fwgpu_partition;
int fwgpu_partition_build(const fwgpu_mesh *mesh, fwgpu_partition **out);
int fwgpu_partition_destroy(fwgpu_partition *part);
/* n_subdomains and total_free (interface DOFs) */
int fwgpu_partition_info(const fwgpu_partition *part, int32_t *n_subdomains, int32_t *total_free);
/* Same layout as fwgpu_get_subdomain_maps. */
int fwgpu_partition_maps(const fwgpu_partition *part, int32_t s, int32_t *nel, int32_t *nmp, int32_t *nbc,
                         int32_t *ninbc, int32_t *nop, int32_t *ibc, int32_t *inbc_nfid, int32_t *inbc_ln_part,
                         int32_t *edge_gid);

/* -- reference plug-in slots, batched over all subdomains ----------------- */

/* make_TMP_AIJ: HDDM_make_TMP_AIJ_em_E (main/fullwave/fullwave.c:221-259):
 * element matrices tet_MakeElement_EM_E (lib/fem/make_elem_em.c:14-400)
 * summed into each subdomain's lower-triangle rows in element order, exact
 * zeros removed (aij_matrix_func.h:260-391), plus the source right-hand side. */
int fwgpu_make_tmp_aij(fwgpu_context *ctx, const fwgpu_source *src);
/* Sets (or, with NULL, clears) the element source every later assembly of a
 * right-hand side adds: make_tmp_aij, hddm_solve, hddm_resolve and each source
 * of hddm_solve_multi.  The adjoint solve of fwgpu_adjoint_gradient does not
 * use it.  Arrays are copied. */
int fwgpu_set_element_source(fwgpu_context *ctx, const fwgpu_element_source *es);

/* solve_dom_1st: hddm_solver_CS_solve_dom_1st_d (lib/hddm/hddm_solver.h:461-555)
 * for every subdomain: Dirichlet elimination, skyline envelope
 * (advlas_skyline.c:12-60), LDL^T factor (advlas_skyline.c:79-128), first
 * solve, vec = A x - b, the diagonal preconditioner (hddm_pc.h:52-86), and
 * the scatter-add into Q and PC (hddm_solver_sp.h:8-25). */
int fwgpu_solve_dom_1st(fwgpu_context *ctx);

/* iteration_s_1st: ITERATION_S_1ST (lib/hddm/hddm_solver_s.h:158-256) with
 * DIAG_GATHER_S (hddm_pc.h:108-137). */
int fwgpu_iteration_s_1st(fwgpu_context *ctx, int32_t *status);

/* One HDDM step: renewal_bc_sp + solve_dom + COM_res_sp for every subdomain
 * (hddm_solver_s.h:69-112, hddm_solver.h:559-622, hddm_solver_sp.h:28-69)
 * followed by iteration_s (hddm_solver_s.h:260-400).  status receives 1 when
 * the residual reached hddm_eps. */
int fwgpu_iteration_s(fwgpu_context *ctx, int32_t *status);

/* solve_dom_last: hddm_solver_CS_solve_dom_last_d (hddm_solver.h:626-693)
 * with the converged interface values, then get_result_sp
 * (main/fullwave/fullwave.c:500-514). */
int fwgpu_solve_dom_last(fwgpu_context *ctx);

/* -- batched driver ------------------------------------------------------- */

/* hddm_solver_CS (lib/hddm/hddm_solver.h:25-183, s-mode loop
 * hddm_solver_s.h): make_tmp_aij, solve_dom_1st, iteration_s_1st, iterations
 * captured in CUDA graphs until hddm_eps or hddm_max_loop, solve_dom_last.
 * Returns FWGPU_ERR_NOT_CONVERGED (with the result filled) when the loop
 * hits hddm_max_loop. */
int fwgpu_hddm_solve(fwgpu_context *ctx, const fwgpu_source *src, fwgpu_result *result);

/* Re-run only the interface iteration and last step for a new right-hand side
 * on the existing factors (multi-source runs). */
int fwgpu_hddm_resolve(fwgpu_context *ctx, const fwgpu_source *src, fwgpu_result *result);

/* -- correction-Jo pre-solve of an antenna ------------------------------- */

/* The real-symmetric HDDM that main() runs for every antenna before the
 * full-wave solve (main/fullwave/main.c:92-98: hddm_solver_RS with
 * set_hddm_func_correct_Jor, then set_hddm_func_correct_Joi,
 * lib/hddm/set_hddm_func.c:90-233).  Its unknown is a potential at the
 * vertices of the antenna's elements, its element matrix (grad N_i, grad N_j)
 * and its element vector (J, grad N_i) of the vertex currents J
 * (tet_MakeElement_correct_Jo, lib/fem/make_elem.c:10-66); interface DOFs
 * are the antenna vertices two or more subdomains hold that are on no
 * Dirichlet list (make_PartMesh.c:393-421), and a subdomain with
 * no Dirichlet or interface DOF holds its first DOF at zero
 * (make_PartMesh.c:973-1063,1288-1340,1546-1575).  The interface problem is
 * solved by the same batched kernels as the full-wave one (the reference's
 * RS and CS drivers are one template, hddm_solver.h and hddm_solver_s.h,
 * here with real values), the subdomain systems by the envelope LDL^T
 * factor where the reference iterates (mymt_RS_AIJ_Solver_CG with ICC to
 * coJo-l-sol-eps 1e-12).  Pass the reference's coJo options in opts:
 * hddm_eps = coJo-hddm-eps (1e-10), hddm_max_loop = coJo-hddm-max-loop
 * (4000); precision must be FWGPU_PREC_FP64.
 *
 * fwgpu_cojo_create: the integer setup of the antenna with element flag
 * antenna_flag (only subdomains with antenna elements take part) and the
 * device context.  pec_vertex: one flag per vertex marking vertex nodes of
 * the Dirichlet (DirichletBCs_Axn0) lists, or NULL for none. */
int fwgpu_cojo_create(const fwgpu_mesh *mesh, int32_t antenna_flag, const uint8_t *pec_vertex,
                      const fwgpu_options *opts, fwgpu_context **out);
/* One pass: current = 3 doubles per global vertex (the real part Jor for the
 * first pass, the imaginary part Jo for the second); potential receives one
 * double per global vertex (Ihr / Ihi of every subdomain holding it; 0 off
 * the antenna).  The first call assembles and factors, later calls reuse the
 * factors.  Returns FWGPU_ERR_NOT_CONVERGED (result and potential filled)
 * at hddm_max_loop. */
int fwgpu_cojo_solve(fwgpu_context *ctx, const double *current, fwgpu_result *result, double *potential);
/* The current of the next right-hand side, without solving: with it the
 * slot-by-slot calls (fwgpu_make_tmp_aij with a NULL or empty source,
 * fwgpu_solve_dom_1st, fwgpu_iteration_s_1st, fwgpu_iteration_s,
 * fwgpu_solve_dom_last) run a pass behind the reference's own hddm_solver_RS
 * loop, and fwgpu_get_edge_solution then gives 2 doubles per vertex. */
int fwgpu_cojo_set_current(fwgpu_context *ctx, const double *current);
/* The original subdomain id of each of the problem's subdomains (n first;
 * sub_ids may be NULL to query n). */
int fwgpu_cojo_subdomains(const fwgpu_context *ctx, int32_t *n, int32_t *sub_ids);
/* The integer setup alone, without a GPU; fwgpu_partition_info and
 * fwgpu_partition_maps then describe the problem's subdomains (edge_gid
 * holds the global vertex of each local DOF, nop the local DOFs of each
 * antenna element in slots 0-3 and 4-7, -1 in 8-9). */
int fwgpu_cojo_partition_build(const fwgpu_mesh *mesh, int32_t antenna_flag, const uint8_t *pec_vertex,
                               fwgpu_partition **out);
int fwgpu_cojo_partition_subdomains(const fwgpu_partition *part, int32_t *sub_ids);

/* -- adjoint ------------------------------------------------------------- */

/* Backward of fwgpu_hddm_solve (the forward).  No reference counterpart.
 * For J = sum_p |x_p|^2 over the probe edges of the forward solution x, one
 * adjoint HDDM solve A lambda = conj(x_P) on the forward factors (A = A^T)
 * gives, per listed element e with edge values x_e, lambda_e and mass
 * matrix SS_e (recomputed, lib/fem/tetrahedral.c:362-422),
 *   grad_eps[k]   = dJ/d eps_e   = 2 omega Re(lambda_e^T SS_e x_e)   [per F/m]
 *   grad_sigma[k] = dJ/d sigma_e = 2 Im(lambda_e^T SS_e x_e)         [per S/m]
 * for the element matrix (nu/omega) RR - (eps omega) SS + i sigma SS
 * (lib/fem/make_elem_em.c:227-265).  J receives the objective, the adjoint
 * solve's COCG figures go to adjoint_result; fwgpu_get_edge_solution still
 * returns the forward solution afterwards. */
int fwgpu_adjoint_gradient(fwgpu_context *ctx, int32_t n_probe, const int32_t *probe_edges, int32_t n_design,
                           const int32_t *design_tets, double *J, double *grad_eps, double *grad_sigma,
                           fwgpu_result *adjoint_result);

/* -- post step ------------------------------------------------------------ */
/* post_sp: HDDM_post_sp_em_E (main/fullwave/fullwave.c:518-529), that is
 * HDDM_post_dom_em_E (:607-634) over every subdomain with HDDM_post_em_E
 * (:639-763) per element.  From each element's six edge values it gives the
 * reference's element results (ResultValue, lib/std/types.h:330-345):
 *   el_B  = (2/D) sum_i i xe_i (X_i, Y_i, Z_i)     i (nu/omega) rot E
 *   el_E  = (2/D) sum_i xe_i (Fx_i, Fy_i, Fz_i)    E at the centroid
 *   el_Je = (sigma/D) sum_i xe_i (Fx_i, Fy_i, Fz_i)
 * where xe_i is the edge value times nu/omega, nu = 7.957747e+05 for an
 * element whose flag is in the Permittivity list and 0 otherwise, sigma the
 * element's Conductor entry (0 if none): the reference scales the edge values
 * before all three sums.  3 complex (6 doubles) per element, in global
 * element order (the reference keeps them per subdomain in local element
 * order; each element lies in one subdomain).
 *   x      2*n_edges doubles, or NULL for the context's last edge solution
 *          (fwgpu_solve_dom_last, fwgpu_hddm_solve, fwgpu_hddm_resolve, or the
 *          source last read with fwgpu_get_edge_solution_multi); a sharded
 *          context holds only its own edges and needs x.
 *   el_B, el_E, el_Je   6*n_tets doubles each; NULL skips that result.
 * Every pointer may be host memory or 16-byte aligned device memory of the
 * context's device; device results are written in place, without a copy.
 * Returns FWGPU_ERR_MESH for a degenerate element (the reference stops in
 * tetNedelec_Direction, lib/fem/tetrahedral.c:257-258). */
int fwgpu_post_em_E(fwgpu_context *ctx, const double *x, double *el_B, double *el_E, double *el_Je);
/* -- measurement ---------------------------------------------------------- */

typedef struct {
  double subsolve_ms;   /* one batched subdomain-solve launch of the interface iteration, average */
  double interface_ms;  /* the interface (COCG) kernels of one iteration, average */
  double iteration_ms;  /* one iteration replayed from the CUDA graph, average */
  int32_t reps;
} fwgpu_kernel_profile;

/* Times the kernels of one interface iteration with CUDA events on the
 * context's stream.  Needs factors (after fwgpu_hddm_solve); overwrites the
 * iteration state, so the solution must be recomputed with
 * fwgpu_hddm_resolve afterwards.  No reference counterpart (the reference
 * times whole phases with gettimeofday, lib/std/timefunc.c:17-111). */
int fwgpu_profile_iteration(fwgpu_context *ctx, int32_t reps, fwgpu_kernel_profile *out);
/* Average device time of one post-step kernel launch (fwgpu_post_em_E, all
 * three results into device memory) over reps launches on the context's last
 * edge solution, each timed alone with CUDA events after a write of 256 MiB
 * that evicts the L2.  No reference counterpart. */
int fwgpu_profile_post(fwgpu_context *ctx, int32_t reps, double *kernel_ms);

/* -- several sources on one set of factors --------------------------------- */

/* Right-hand sides one batched solve takes at most. */
#define FWGPU_MAX_RHS 16

/* Solves n_src (1..FWGPU_MAX_RHS) sources together: one assembly and one
 * factorisation, then all sources' interface COCGs in lockstep on the same
 * factors, each with its own scalars and stopping test.  results[k] is
 * source k's (the times are the batch's).  The reference solves one source
 * per hddm_solver_CS run (hddm_solver.h:25-183); this is n_src such runs
 * sharing the factors.  Needs the staged solve kernel (not available when a
 * subdomain is too large for its shared memory). */
int fwgpu_hddm_solve_multi(fwgpu_context *ctx, int32_t n_src, const fwgpu_source *sources, fwgpu_result *results);
/* Edge solution of source k of the last fwgpu_hddm_solve_multi (2*n_edges doubles). */
int fwgpu_get_edge_solution_multi(fwgpu_context *ctx, int32_t k, double *x);
/* The adjoint of every source of the last fwgpu_hddm_solve_multi at once: for
 * source k, J[k] = sum over the probes of |x_k|^2, and its gradient with
 * respect to the permittivity and conductivity of each design element, as
 * fwgpu_adjoint_gradient gives it for one source.  The n_src adjoint
 * right-hand sides conj(x_k at the probes) are solved together, as one
 * batched solve on the forward factors (A = A^T); then one gradient launch
 * per source.  grad_eps and grad_sigma hold n_src * n_design values, source
 * by source (NULL to skip); adjoint_results (NULL to skip) gets n_src
 * results.  Afterwards fwgpu_get_edge_solution_multi(k) returns source k's
 * adjoint solution.  No counterpart in the reference (as
 * fwgpu_adjoint_gradient). */
int fwgpu_adjoint_gradient_multi(fwgpu_context *ctx, int32_t n_probe, const int32_t *probe_edges, int32_t n_design,
                                 const int32_t *design_tets, double *J, double *grad_eps, double *grad_sigma,
                                 fwgpu_result *adjoint_results);

/* -- sharded solve over several GPUs (one context per rank) ---------------- */

/* A context created with shard_begin < shard_end solves the subdomains of
 * that range only: the reference's "part" (lib/hddm/hddm_solver_ph.h:112-329,
 * one part per rank).  Each shard runs the COCG on the interface DOFs its
 * subdomains hold; every DOF has one owner (the shard of the first subdomain
 * holding it), and the dot products and the max-norm sum or max the owned
 * DOFs over the shards.  Only the DOFs held by two or more shards cross
 * between the ranks, packed in ascending DOF order (the same positions on
 * every rank).  Per iteration the caller sums, over the ranks, in place on
 * the context's device: the packed partial Q, then (p, q), then (r, z) and
 * |r|^2 together with the max of max|r| -- the reference's neighbour exchange
 * and its scalar all-reduces.  Order per solve:
 *   fwgpu_shard_set_layout; fwgpu_shard_set_exchange (once per context);
 *   fwgpu_make_tmp_aij; fwgpu_shard_first; [sum pack];
 *   fwgpu_shard_first_sums; [sum scal[0..2], max scal[4]];
 *   fwgpu_shard_first_finish; then until *status != 0:
 *     fwgpu_shard_iterate; [sum pack[0 .. 2*n_shared)];
 *     fwgpu_shard_iterate_pq; [sum scal[0..1]];
 *     fwgpu_shard_iterate_update; [sum scal[0..2], max scal[4]];
 *     fwgpu_shard_iterate_finish;
 *   fwgpu_solve_dom_last; fwgpu_get_edge_solution gives this shard's edges
 *   (zero elsewhere): their sum over ranks is the solution.
 * Every call returns after its kernels finished, so the caller's collective
 * may read the buffers at once.  The whole-solve calls (fwgpu_hddm_solve,
 * fwgpu_iteration_s*) refuse a sharded context. */

/* The subdomain ranges of all n_shards shards: shard k solves subdomains
 * shard_first[k] .. shard_first[k+1]-1 (shard_first[0] = 0,
 * shard_first[n_shards] = n_subdomains); this context's range must be one
 * of them.  *n_shared receives the number of interface DOFs held by two or
 * more shards, the length of the packed exchange. */
int fwgpu_shard_set_layout(fwgpu_context *ctx, int32_t n_shards, const int32_t *shard_first, int32_t *n_shared);
/* Caller-owned device buffers on the context's device: d_pack 4*n_shared
 * doubles (two packed complex vectors: Q, and on the first step the
 * preconditioner diagonal), d_scal 8 doubles. */
int fwgpu_shard_set_exchange(fwgpu_context *ctx, double *d_pack, double *d_scal);
/* solve_dom_1st on this shard; packed partial Q and diagonal */
int fwgpu_shard_first(fwgpu_context *ctx);
/* the first step of ITERATION_S_1ST on the held DOFs, from the summed pack;
 * local sums of the owned DOFs into scal */
int fwgpu_shard_first_sums(fwgpu_context *ctx);
/* its scalars from the summed scal; *status as fwgpu_iteration_s_1st */
int fwgpu_shard_first_finish(fwgpu_context *ctx, int32_t *status);
/* the subdomain solves of one iteration; packed partial Q */
int fwgpu_shard_iterate(fwgpu_context *ctx);
/* Q from the summed pack; the owned DOFs' (p, q) into scal[0..1] */
int fwgpu_shard_iterate_pq(fwgpu_context *ctx);
/* alpha from the summed (p, q); u, r, z; the owned DOFs' (r, z), |r|^2, max|r| into scal */
int fwgpu_shard_iterate_update(fwgpu_context *ctx);
/* resi, beta and the stopping test from the summed scal, then p;
 * *status as fwgpu_iteration_s */
int fwgpu_shard_iterate_finish(fwgpu_context *ctx, int32_t *status);

/* -- batched skyline substitution without device allocation -------------- */

/* Rows of the fixed device work array behind fwgpu_skyline_solve_noalloc:
 * 262,144 complex FP64 values (4 MiB), held by every GPU that loads the
 * library until the process exits. */
#define FWGPU_NOALLOC_MAX_ROWS 262144

/* Solves L D L^T x = b for a batch of skyline-factored systems on the
 * current device without allocating any device memory.  No counterpart in
 * the reference: it is for callers that cannot call cudaMalloc when they
 * solve (a host framework that owns the device memory through its own pool,
 * or a real-time loop that must not enter the allocator), so every buffer
 * is theirs and the work vectors live in a fixed device array.
 *
 * Systems use the reference's skyline layout (advlas_skyline.c:12-128):
 * system s has rows d_row_off[s]..d_row_off[s+1]-1 of d_idx1/d_idx2 (its
 * own row numbering), entries d_mat[2*(d_mat_off[s] + idx2[i] + j)] for
 * j = idx1[i]..i, unit L off the diagonal and 1/d on it (what
 * fwgpu_get_factor returns).  d_b and d_x hold 2*total_rows doubles
 * (interleaved complex).  All pointers are device memory; the kernel runs on
 * `stream` (a cudaStream_t, NULL for the default stream) and the call
 * returns without synchronising.
 *
 * d_row_off must be non-decreasing with d_row_off[0] >= 0 and
 * d_row_off[n_systems] <= total_rows; a system whose rows fall outside
 * [0, total_rows) is skipped and its rows of d_x keep what they held.
 * idx1[i] must lie in [0, i]; a value outside is clamped, which keeps the
 * other systems' results intact but makes that system's result
 * meaningless.  d_b may equal d_x (an in-place solve).
 *
 * total_rows may not exceed FWGPU_NOALLOC_MAX_ROWS (FWGPU_ERR_ARG
 * otherwise).  Every call looks up the work array's address in the context
 * current on the calling thread; the first call in a context (also after a
 * cudaDeviceReset) loads the library's device code into it, so make it
 * before any stream capture.  All calls share the work array: calls whose
 * kernels overlap on one GPU race and must be ordered by the caller. */
int fwgpu_skyline_solve_noalloc(int32_t n_systems, int32_t total_rows, const int32_t *d_row_off,
                                const int64_t *d_mat_off, const int32_t *d_idx1, const int32_t *d_idx2,
                                const double *d_mat, const double *d_b, double *d_x, void *stream);

/* -- results -------------------------------------------------------------- */

/* Edge solution per global edge (2*n_edges doubles).  Every subdomain holding
 * an edge computes the same value; the lowest-numbered one is returned. */
int fwgpu_get_edge_solution(fwgpu_context *ctx, double *x_edges);
/* Residual history: resi per iteration (hddm_solver_s.h:319-323),
 * up to max_n entries; n_out receives the count. */
int fwgpu_get_history(fwgpu_context *ctx, double *resi, int32_t max_n, int32_t *n_out);

/* -- introspection for parity tests -------------------------------------- */

/* Integer maps of subdomain s as the reference's make_PartMesh leaves them:
 * nop (10*nel, after make_MESH_change_nop), Dirichlet list ibc (nbc, PEC
 * then interface), inbc (nfid, ln_part pairs), and the global edge id of each
 * local edge DOF.  Pass NULL buffers to query the counts. */
int fwgpu_get_subdomain_maps(const fwgpu_context *ctx, int32_t s, int32_t *nel, int32_t *nmp, int32_t *nbc,
                             int32_t *ninbc, int32_t *nop, int32_t *ibc, int32_t *inbc_nfid,
                             int32_t *inbc_ln_part, int32_t *edge_gid);
/* The reference's skyline profile of subdomain s after Dirichlet elimination:
 * idx1[n], idx2[n] and nlen (advlas_skyline.c:12-25). */
int fwgpu_get_skyline_profile(fwgpu_context *ctx, int32_t s, int32_t *idx1, int32_t *idx2, int32_t *nlen);
/* Assembled lower rows of subdomain s (row_ptr[n+1], col[nnz], val[2*nnz]) and
 * right-hand side b[2n]; pass NULL to query nnz through *nnz. */
int fwgpu_get_tmp_aij(fwgpu_context *ctx, int32_t s, int32_t *nnz, int32_t *row_ptr, int32_t *col, double *val,
                      double *b);
/* FP64 factor of subdomain s in the reference's skyline layout
 * (mat[idx2[i]+j], 1/d on the diagonal); nlen complex values. */
int fwgpu_get_factor(fwgpu_context *ctx, int32_t s, double *mat);

#ifdef __cplusplus
}
#endif
#endif /* FWGPU_H */
