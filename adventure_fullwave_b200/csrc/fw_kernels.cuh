// Device kernels of the HDDM hot path (declarations shared by fw_capi.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fw {

// COCG scalars of one interface problem, resident on the device.  Mirrors the
// scalars of ITERATION_S / ITERATION_S_1ST (lib/hddm/hddm_solver_s.h:158-400)
// and hddm_sw (lib/std/types.h:732-741).
struct CocgScalars {
  double2 rz;        // (r, z) bilinear
  double2 rz_new;
  double2 malpha;    // -alpha
  double2 beta;
  double norm0;      // max|r0|
  double r0inv;      // 1 / max|r0|
  double l2_0;       // ||r0||_2
  double resi;       // max|r| / max|r0|
  double resi_l2;    // ||r||_2 / ||r0||_2
  double eps;        // hddm_eps
  int32_t status;    // 0 iterating, 1 last iteration done (p := u), 2 finished
  int32_t loop;      // hddm_sw.loop
  int32_t max_loop;  // hddm_max_loop
  int32_t converged;
  int32_t factor_status;  // non-zero: a pivot was zero or not finite
  int32_t copy_timeout;   // non-zero: a subdomain solve gave up waiting for a copy (cleared by the host only)
  int32_t nonfinite;      // non-zero: the interface residual or (r, z) was not finite; the loop stopped
  int32_t unused;
  uint32_t ticket[4];  // CTAs of a reduction kernel that wrote their partials (last one reduces)
};

// Per-problem device pointers used by the iteration kernels.
struct DevProblem {
  int32_t nsub;                  // subdomains this context solves (all, or a shard's range)
  int32_t nfree;                 // interface DOFs
  const int32_t *sub_order;      // warps take subdomains in this order (nsub entries)
  const int64_t *int_off;        // nsub+1
  const int64_t *if_off;         // nsub+1
  // interior envelope (compressed)
  const int32_t *env_lo;         // sum nI: first stored column (interior index)
  const int64_t *env_ptr;        // sum nI: position of column env_lo in the value arrays
  const double2 *L64;
  const float2 *L32;
  // operators
  const int32_t *cpl_ptr;        // sum(nI+1) relative
  const int64_t *cpl_off;        // nsub+1 base of cpl arrays
  const int32_t *cpl_col;
  const double2 *cpl_val;
  const int32_t *ifr_ptr;        // sum(nG+1) relative
  const int64_t *ifr_off;
  const int32_t *ifr_col;
  const double2 *ifr_val;
  const int32_t *aii_ptr;        // sum(nI+1) relative
  const int64_t *aii_off;
  const int32_t *aii_col;
  const double2 *aii_val;
  const int32_t *if_ln;          // sum nG
  const double2 *fI;             // sum nI, interior right-hand side
  const double2 *fG;             // sum nG, interface right-hand side
  // work
  double2 *Y;                    // sum nI, interior solution
  double2 *B;                    // sum nI, right-hand side copy (refinement)
  float2 *Y32;                   // sum nI, FP32 work (refinement)
  double2 *V;                    // sum nG, interface values
  double2 *qloc;                 // sum nG
  // interface vectors
  double2 *P, *Q, *R, *Z, *U, *PC;
  const int32_t *gq_ptr;         // nfree+1
  const int64_t *gq_slot;
  CocgScalars *sc;
  double *hist;                  // residual history
  double *part;                  // reduction partials, 4 * n_part_blocks
  int32_t n_part_blocks;
  int32_t ir_steps;
  double ir_tol;
  double ir_relax;               // interface iterations refine only while sc->resi > ir_relax
  int32_t cta_smem;              // dynamic shared bytes of the CTA-per-subdomain solve (0: not available)
  int32_t hist_cap;              // entries of hist
  int32_t solve_variant;         // SolveVariant of the batched subdomain solve
  int32_t stall_test;            // test hook: the staged solves' first copy wait gives up (bounded)
  int32_t max_interior;          // largest subdomain: interior rows
  int32_t max_iface;             // largest subdomain: interface DOFs
  // staged solve (kSolveWarp): row blocks and grid-wide operator products
  const int32_t *blk_off;        // nsub+1: first block-table entry of each subdomain
  const int2 *blk_tab;           // per subdomain nblk+1 x (first row, first envelope element)
  int32_t max_blocks;            // most blocks of one subdomain
  int32_t stage_cap;             // envelope elements per staging buffer
  int32_t stage_warps;           // warps sharing one subdomain's sweeps (1, 2 or 4)
  // staged solve on the block-inverse layout (kSolveInv): per block of rows,
  // the rows' entries left of the block, then N = (I + L_bb)^-1 - I strictly
  // lower and row-major (row t at t(t-1)/2), then the block's pivots 1/d
  const int64_t *inv_ptr;        // sum nI: position of each row's left entries in Linv
  const double2 *Linv64;
  const float2 *Linv32;
  const int32_t *inv_blk_off;    // nsub+1
  const int2 *inv_blk_tab;       // per subdomain nblk+1 x (first row, first element relative to inv_ptr[row 0])
  int32_t inv_max_blocks;
  int32_t inv_cap;               // elements per staging buffer
  int64_t row0, n_interior;      // interior rows of the subdomains this context solves
  int64_t slot0, n_slots;        // interface slots of the subdomains this context solves
  // sharded solve: this shard's partial interface sums go to the exchange
  // buffer (summed over ranks by the caller) and the COCG reads them back
  const int64_t *cpl_rowptr;     // n_interior+1 into cpl_val
  const int32_t *cpl_gcol;       // interface DOF (index into P) of each coupling entry
  const int64_t *ifr_rowptr;     // n_slots+1 into ifr_val
  const int32_t *ifr_gcol;       // >=0: global interior row; <0: -(interface DOF)-1
  const int64_t *aii_rowptr;     // n_interior+1 into aii_val
  const int32_t *aii_gcol;       // global interior row of each interior entry
  double2 *Rres;                 // n_interior: refinement residual
  // sharded solve with the exchange packed to the shared interface DOFs: the
  // interface DOFs this shard's subdomains hold (ascending), whether it owns
  // each (every DOF has one owner, so sums over owned DOFs add up once over
  // the shards), each one's place in the packed exchange (-1: held by this
  // shard alone), the packed buffer (2 x n_shared complex) and the scalar
  // buffer ([0..2] summed, [4] maxed over the shards)
  const int32_t *dist_dof;
  const uint8_t *dist_own;
  const int32_t *dist_pos;
  int32_t dist_n;
  int32_t n_shared;
  double2 *dist_pack;
  double *dist_scal;
};

// Batched subdomain solve kernels: one warp per subdomain with TMA-staged row
// blocks and grid-wide operator products, one CTA per subdomain, or one warp
// per subdomain with the vectors in global memory (any size).
enum SolveVariant { kSolveWarp = 0, kSolveCta = 1, kSolveGlobal = 2, kSolveInv = 3 };

enum SolveMode { kModeFirst = 0, kModeIter = 1, kModeLast = 2 };

// ---- batched right-hand sides ----------------------------------------------
// Up to kMaxRhs sources share one set of factors: every vector is stored
// right-hand-side minor ([row][kMaxRhs]), and each source runs its own COCG
// (its own scalars and stopping) in lockstep with the others.
constexpr int kMaxRhs = 16;
constexpr int kMaxBuckets = 8;

struct MultiScalars {
  CocgScalars s[kMaxRhs];
  int32_t all_status;  // 0: some right-hand side iterates; 2: every one finished
  int32_t err;         // non-zero: a subdomain solve gave up waiting for a copy
  uint32_t ticket[4];
};

struct MultiProblem {
  DevProblem p;                 // structure, factors, operators, row ranges
  const double2 *fI, *fG;       // [n_interior][kMaxRhs], [n_slots][kMaxRhs]
  double2 *Y;                   // [n_interior][kMaxRhs]: right-hand sides in, interior solutions out
  double2 *B, *Rres;            // FP32 + refinement: right-hand side copy, residual
  void *Zs;                     // [n_interior][kMaxRhs] z stash in the factor's precision
  double2 *V, *qloc;            // [n_slots][kMaxRhs]
  double2 *P, *Q, *R, *Z, *U;   // [nfree][kMaxRhs]
  double2 *PC;                  // [nfree]
  MultiScalars *ms;
  double *part;                 // [fields][n_part_blocks][kMaxRhs]
  // sweep launches by subdomain size: bucket k covers sub_order[first[k] ..
  // first[k] + count[k]) with shared memory for its largest subdomain
  int n_buckets;
  int bucket_first[kMaxBuckets], bucket_count[kMaxBuckets];
  int bucket_max_interior[kMaxBuckets], bucket_max_blocks[kMaxBuckets];
};

size_t multi_smem_bytes(int max_interior, int max_blocks, int cap, bool fp32);
int configure_multi(size_t smem, bool fp32);
void launch_multi_subsolve(const MultiProblem &m, int mode, bool fp32, cudaStream_t stream);
void launch_multi_set_status(MultiScalars *ms, double eps, int32_t max_loop, cudaStream_t stream);
void launch_multi_first(const MultiProblem &m, const double2 *pcloc, cudaStream_t stream);
void launch_multi_iteration(const MultiProblem &m, bool fp32, cudaStream_t stream);
void launch_multi_edge_solution(const MultiProblem &m, int k, int64_t ne, const int64_t *edge_src, double2 *x,
                                cudaStream_t stream);
int multi_iteration_launches(bool fp32, int ir_steps, int n_buckets);

void launch_element_matrices(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                             const double *el_eps, const double *el_sigma, double omega, double *out,
                             int32_t *status, cudaStream_t stream);
// correction-Jo problem: linear-tetrahedron (grad, grad) matrices in the
// 6x6 slot layout, and element vectors (J, grad N_i) from vertex currents J
void launch_cojo_element_matrices(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices,
                                  const double *crd, double *out, int32_t *status, cudaStream_t stream);
void launch_cojo_element_rhs(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                             const double *J, double2 *be, cudaStream_t stream);
void launch_gather_values(int64_t nnz, const int64_t *contrib_ptr, const int64_t *contrib, const double2 *elmat,
                          double2 *aval, cudaStream_t stream);
void launch_profile(int32_t nsub, const int64_t *dof_off, const int64_t *nnz_off, const int32_t *row_ptr_rel,
                    const int32_t *col, const double2 *aval, const uint8_t *isbc, int32_t *idx1,
                    cudaStream_t stream);
void launch_scatter_envelope(int64_t nnz, const int64_t *dst, const double2 *aval, double2 *L, cudaStream_t stream);
void launch_gather_ops(int64_t n, const int64_t *src, const double2 *aval, double2 *dst, cudaStream_t stream);
void launch_diag_pc(int64_t n, const int64_t *diag_src, const double2 *aval, double2 *pcloc, cudaStream_t stream);
void launch_factor(const DevProblem &p, const int64_t *int_off, const int32_t *env_lo, const int64_t *env_ptr,
                   double2 *L, int32_t *status, cudaStream_t stream);
void launch_to_fp32(int64_t n, const double2 *src, float2 *dst, cudaStream_t stream);
void launch_subsolve(const DevProblem &p, int mode, bool fp32, cudaStream_t stream);
size_t subsolve_smem_bytes(int max_interior, int max_iface, bool fp32);
int configure_subsolve(size_t smem, bool fp32);
size_t subsolve_staged_smem_bytes(int max_interior, int max_blocks, int cap, bool fp32);
int configure_subsolve_staged(size_t smem, bool fp32);
int configure_subsolve_inv(size_t smem, bool fp32);
// the block-inverse layout (DevProblem inv_*) from the FP64 factor L64 in the
// envelope layout, in FP32 (Linv32) or FP64 (Linv64)
void launch_inv_relayout(const DevProblem &p, const double2 *L64, bool fp32, cudaStream_t stream);
// Raises (never lowers) the dynamic shared-memory limit of kernel `func` on
// the current device; `slot` names the kernel (0..7).
// Slots of the process-wide dynamic shared-memory limits (raise_smem_limit):
// one per kernel instantiation that runs above the 48 KB default.
enum SmemSlot {
  kSlotStaged32 = 0,
  kSlotStaged64 = 1,
  kSlotCta32 = 2,
  kSlotCta64 = 3,
  kSlotInv32 = 4,
  kSlotInv64 = 5,
  kSlotMulti32 = 6,
  kSlotMulti64 = 7,
  kSmemSlots = 8
};
int raise_smem_limit(const void *func, int slot, size_t smem);
// kernels one launch_subsolve call issues
int subsolve_launches(const DevProblem &p, bool fp32);
void launch_cocg_first(const DevProblem &p, const double2 *pcloc, cudaStream_t stream);
void launch_cocg_iteration(const DevProblem &p, cudaStream_t stream);
// the COCG part of an iteration (after the subdomain solves): Q, alpha, updates, beta, p
void launch_cocg_update(const DevProblem &p, cudaStream_t stream);
void launch_edge_solution(const DevProblem &p, int64_t ne, const int64_t *edge_src, const double2 *Y,
                          const double2 *V, double2 *x, cudaStream_t stream);
void launch_set_status(CocgScalars *sc, double eps, int32_t max_loop, cudaStream_t stream);
void launch_element_rhs(int64_t n_el, const int32_t *el_order, const int32_t *tet_vertices, const double *crd,
                        const double *el_sigma, double omega, int32_t n_gaps, const double *gap,
                        const int32_t *el_antenna, const double *Jo, const double *Jor, int64_t n_vertices,
                        double2 *be, cudaStream_t stream);
void launch_rhs_gather(int64_t n_dof, const int64_t *ptr, const int32_t *src, const double2 *be,
                       const double2 *b_edge, double2 *b, cudaStream_t stream);
void launch_rhs_split(int64_t n, const int64_t *pos, const double2 *b, double2 *f, cudaStream_t stream);
void launch_post_em_E(int64_t nt, const int32_t *tet_vertices, const int32_t *tet_edges, const double *crd,
                      const uint8_t *el_has_nu, const double *el_sigma, double omega, const double2 *x, double2 *B,
                      double2 *E, double2 *Je, int32_t *status, cudaStream_t stream);
void launch_adjoint_gradient(int32_t n_design, const int32_t *design_tets, const int32_t *tet_vertices,
                             const int32_t *tet_edges, const double *crd, double omega, const double2 *x,
                             const double2 *lam, double *g_eps, double *g_sigma, cudaStream_t stream);
void launch_profile_reset(CocgScalars *sc, cudaStream_t stream);
// sharded solve, packed exchange (DevProblem dist_*): pack the shard's
// partial Q (and PC diagonal) of its shared DOFs; the first COCG step up to
// the local sums; its scalars from the exchanged sums; an iteration's (p, q),
// its update up to the local sums, and its scalars and p
void launch_dist_pack(const DevProblem &p, const double2 *pcloc, bool with_pc, bool status_check, cudaStream_t stream);
void launch_dist_first(const DevProblem &p, const double2 *pcloc, cudaStream_t stream);
void launch_dist_first_finish(const DevProblem &p, cudaStream_t stream);
void launch_dist_pq(const DevProblem &p, cudaStream_t stream);
void launch_dist_update(const DevProblem &p, cudaStream_t stream);
void launch_dist_finish(const DevProblem &p, cudaStream_t stream);

}  // namespace fw
