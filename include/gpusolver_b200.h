/*
 * gpusolver_b200 -- C ABI of the B200-native AMG-preconditioned CG path.
 *
 * Plain C: pointers, sizes and status codes; no C++ or torch types cross it
 * and no exception escapes it. Every function returns GS_OK (0) on success;
 * otherwise the reason is available from gs_last_error() (thread-local).
 * Each entry point names the reference interface it replaces (file:line in
 * theofbraune/GPU-Conjugate-Gradient-Solver); the C++ classes under
 * include/GPUSolver/ are thin wrappers over these calls and re-throw
 * failures as std::runtime_error, as the reference does.
 *
 * Numbering conventions follow the reference: CSR with int32 row pointers
 * and column indices, permutations as (old_to_new, new_to_old) pairs
 * (include/GPUSolver/Permutation.h:10-33).
 */
#ifndef GPUSOLVER_B200_H
#define GPUSOLVER_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_OK 0
#define GS_ERR_INVALID 1    /* bad argument, shape or matrix (std::runtime_error in the reference) */
#define GS_ERR_CUDA 2       /* CUDA runtime failure */
#define GS_ERR_NOT_FINITE 3 /* NaN/Inf residual: CGSolver's "solver diverged" */
#define GS_ERR_NO_DEVICE 4  /* no CUDA device: the library has no CPU fallback */

/* solve status reported in gs_solve_stats.status */
#define GS_STATUS_CONVERGED 1
#define GS_STATUS_MAX_ITER 2
#define GS_STATUS_BREAKDOWN 4
#define GS_STATUS_INITIAL_CONVERGED 5
#define GS_STATUS_ZERO_RHS 6

/* ABI version, 100 * major + minor: 101 added the device memory, copy and
 * stream entry points (gs_device_malloc ... gs_stream_synchronize); 102
 * appended gs_solver_options.sweep_launch; 103 added gs_solver_node_features
 * and gs_solver_set_node_weights and gs_hierarchy_refresh and appended
 * gs_solver_options.half_sweeps and coarse_half; 104 added
 * gs_solver_level_launch, gs_solver_setup_phases and gs_relaxed_coloring
 * (gs_solver_options.coloring 2). */
#define GS_VERSION 104

const char *gs_last_error(void);
/* GS_VERSION of the library that was loaded. */
int gs_version(void);

/* ------------------------------------------------------------------------
 * Host setup (integer work, bit-exact with the reference)
 * --------------------------------------------------------------------- */

/* GraphColoring::compute (src/GraphColoring.cc:9-72): greedy first-fit in
 * natural order. colors[n], color_vertices[n] (grouped by colour, ascending
 * inside a colour), color_offsets[num_colors + 1] (caller allocates n + 1).
 * Each vertex avoids the colours of the already coloured vertices its row
 * lists, as the reference's does: the colouring is proper for structurally
 * symmetric patterns (an entry whose mirror is missing may join two rows of
 * one colour, in the reference too). */
int gs_greedy_coloring(int n, const int *row_ptr, const int *col_idx, int *colors,
                       int *color_vertices, int *color_offsets, int *num_colors);
/* The same first-fit colouring in smallest-last vertex order (no reference
 * counterpart): usually fewer colours; same output layout. Proper for every
 * pattern: one that is not structurally symmetric is coloured on its
 * symmetrised pattern. */
int gs_smallest_last_coloring(int n, const int *row_ptr, const int *col_idx, int *colors,
                              int *color_vertices, int *color_offsets, int *ncolors);
/* Colouring of the strong couplings only (no reference counterpart; the
 * colouring of the coarse levels under gs_solver_options.coloring 2): the
 * entries with |a_ij| >= theta sqrt(|a_ii a_jj|) are coloured first-fit (row
 * order, or smallest-last order where that gives fewer colours), then rows
 * whose same-colour off-diagonal mass reaches rho |a_ii| move to a colour
 * that keeps it below (0 < rho < 1; the exact greedy colouring if 64 passes
 * do not settle). A Gauss-Seidel pass over it reads same-colour neighbours
 * from the iterate its sweep started with. The pattern must be structurally
 * symmetric. Same output layout as gs_greedy_coloring. */
int gs_relaxed_coloring(int n, const int *row_ptr, const int *col_idx, const double *values, double theta,
                        double rho, int *colors, int *color_vertices, int *color_offsets, int *ncolors);
/* The same for the nodes of a 3x3-blocked matrix (n rows, n / 3 nodes; the
 * colouring of block Gauss-Seidel levels under coloring 2): node pairs are
 * strong when ||A_IJ||_F >= theta sqrt(||A_II||_F ||A_JJ||_F), and a node keeps
 * sum ||A_IJ||_F over its same-colour nodes below rho / ||A_II^-1||_F. Outputs
 * per node (colors[n / 3], color_vertices[n / 3], color_offsets up to
 * n / 3 + 1). */
int gs_relaxed_block_coloring(int n, const int *row_ptr, const int *col_idx, const double *values, double theta,
                              double rho, int *colors, int *color_vertices, int *color_offsets, int *ncolors);

/* RCMReordering::compute (src/ReorderingStrategies/RCMReordering.cc:11-110). */
int gs_rcm(int n, const int *row_ptr, const int *col_idx, int *old_to_new, int *new_to_old);

/* HostCSRMatrix::applyPermutation (src/HostSparseMatrix.cc:118-249):
 * A' = P A P^T, rows reordered, column order inside a row kept. */
int gs_apply_permutation(int n, const int *row_ptr, const int *col_idx, const double *val,
                         const int *old_to_new, const int *new_to_old, int *out_row_ptr,
                         int *out_col_idx, double *out_val);

/* permuteMatrix (src/SparseMatrixUtils.cc:8-31): columns sorted per row. */
int gs_permute_matrix(int rows, int cols, const int *row_ptr, const int *col_idx,
                      const double *val, const int *row_old_to_new, const int *col_old_to_new,
                      int *out_row_ptr, int *out_col_idx, double *out_val);

/* HostELLMatrix (src/HostELLMatrix.cc:10-206): slot-major ELL of `width`
 * slots (index = slot * n + row, padding col 0 / value 0) plus the overflow
 * CSR. ovf_col / ovf_val must hold nnz entries. */
int gs_ell_build(int n, int cols, const int *row_ptr, const int *col_idx, const double *val,
                 int width, int *ell_col, double *ell_val, int *ovf_row_ptr, int *ovf_col,
                 double *ovf_val, int *ovf_nnz);

/* buildBlockGraph (src/BlockUtils.cc:126-216): node i linked to node j != i
 * when an entry of block row i lies in block column j or the reverse; sorted,
 * no duplicates. g_col must hold nnz entries, which suffices for every
 * structurally symmetric matrix; GS_ERR_INVALID (nothing written) if the
 * graph of an unsymmetric pattern needs more. */
int gs_block_graph(int n, const int *row_ptr, const int *col_idx, int block, int *g_row_ptr,
                   int *g_col, int *g_nnz);

/* extractInverseDiagonalBlocks3x3 (src/BlockUtils.cc:218-277): 9 doubles
 * per node, row-major; GS_ERR_INVALID if a block is not SPD. */
int gs_block_inverses3x3(int n, const int *row_ptr, const int *col_idx, const double *val,
                         double *dinv);

/* expandBlockPermutation (src/BlockUtils.cc:7-55). */
int gs_expand_block_permutation(int nodes, int block, const int *node_old_to_new,
                                const int *node_new_to_old, int *old_to_new, int *new_to_old);

/* ------------------------------------------------------------------------
 * Host CSR container (synthetic problems)
 * --------------------------------------------------------------------- */
typedef struct gs_host_csr gs_host_csr;

#define GS_PROBLEM_POISSON7 0        /* ip = {nx, ny, nz} */
#define GS_PROBLEM_VARCOEF_GRF 1     /* ip = {nx, ny, nz}, dp = {corr_len, sigma} */
#define GS_PROBLEM_VARCOEF_LOGUNI 2  /* ip = {nx, ny, nz}, dp = {lo, hi} */
#define GS_PROBLEM_KUHN_P1 3         /* ip = {cells per side}, dp = {jitter fraction of h} */
#define GS_PROBLEM_ELASTICITY_P1 4   /* ip = {vertices per side}, dp = {poisson ratio}; has rhs */

int gs_problem_create(int kind, const int *ip, const double *dp, unsigned long long seed,
                      gs_host_csr **out);
int gs_host_csr_create(int rows, int cols, const int *row_ptr, const int *col_idx,
                       const double *val, gs_host_csr **out);
int gs_host_csr_info(const gs_host_csr *m, int *rows, int *cols, int *nnz, int *has_rhs);
int gs_host_csr_copy(const gs_host_csr *m, int *row_ptr, int *col_idx, double *val);
int gs_host_csr_rhs(const gs_host_csr *m, double *rhs);
void gs_host_csr_destroy(gs_host_csr *m);
/* Right-hand side uniform in [-1, 1] from SplitMix64(seed). */
int gs_uniform_rhs(int n, unsigned long long seed, double *out);

/* ------------------------------------------------------------------------
 * AMG hierarchy: AMGHierarchy (include/GPUSolver/AMGHierarchy.h:13-21)
 * --------------------------------------------------------------------- */
typedef struct gs_hierarchy gs_hierarchy;

typedef struct {
  int rows, cols;
  const int *row_ptr;
  const int *col_idx;
  const double *val;
} gs_csr;

/* AMGHierarchyBuilder(SmoothedAggregationCoarsener(block_size, eps_strong),
 * max_levels, min_dofs).build(A)
 * (examples/amgSolver/src/AMGHierarchyBuilder.cc:59-150,
 *  examples/amgSolver/src/SmoothedAggregationCoarsener.cc:64-108). */
int gs_hierarchy_build(const gs_host_csr *a, int block_size, double eps_strong, int max_levels,
                       int min_dofs, gs_hierarchy **out);
/* The same builder with a choice of aggregation and of where it runs (no
 * reference counterpart: the reference's setup is amgcl on the host).
 * aggregation 0: gs_hierarchy_build's sequential aggregation (host only);
 *             1: aggregates grown from a distance-2 maximal independent set of
 *                the strength graph (parallel rounds), everything else as 0.
 * device < 0 builds on the host, device >= 0 on that GPU (aggregation 1 only;
 * every row of `a` needs sorted, duplicate-free column indices). Host and GPU
 * builds of aggregation 1 are identical bit for bit. stats may be NULL. */
typedef struct {
  double total_ms;    /* wall clock of the whole build */
  double upload_ms;   /* GPU build: finest matrix to the device */
  double build_ms;    /* GPU build: the coarsening steps */
  double download_ms; /* GPU build: levels back to the host */
  int mis_rounds;     /* independent-set rounds, all levels */
} gs_setup_stats;
int gs_hierarchy_build_ex(const gs_host_csr *a, int block_size, double eps_strong, int max_levels,
                          int min_dofs, int aggregation, int device, gs_setup_stats *stats,
                          gs_hierarchy **out);
/* New values on the finest level, same sparsity: *out holds every coarser
 * level recomputed as A_{k+1} = R_k A_k P_k with h's transfer operators
 * (DeviceCSRMatrix::updateValues, src/cuda/CudaDeviceCSRMatrix.cc:99-116,
 * extended to the Galerkin hierarchy). device >= 0: the sparse products run
 * on that GPU (the setup's own kernels); device < 0: on the host. Both give
 * the same bits. values: nnz of the finest level, in its CSR order. */
int gs_hierarchy_refresh(const gs_hierarchy *h, const double *values, int device, gs_hierarchy **out);
/* A hierarchy given level by level (A[L], P[L-1], R[L-1]). */
int gs_hierarchy_from_levels(int num_levels, const gs_csr *A, const gs_csr *P, const gs_csr *R,
                             int block_size, gs_hierarchy **out);
int gs_hierarchy_num_levels(const gs_hierarchy *h);
/* which: 0 = A[level], 1 = P[level], 2 = R[level] */
int gs_hierarchy_matrix_info(const gs_hierarchy *h, int level, int which, int *rows, int *cols,
                             int *nnz);
int gs_hierarchy_matrix(const gs_hierarchy *h, int level, int which, int *row_ptr, int *col_idx,
                        double *val);
/* aggregate of every node of `level` (-1: isolated, no coarse dof) */
int gs_hierarchy_aggregates(const gs_hierarchy *h, int level, int *agg);
/* HierarchicalReordering::compute
 * (src/ReorderingStrategies/HierarchicalReordering.cc:217-278): one permutation
 * per level (finest first) to pass to gs_solver_create; old_to_new[k] and
 * new_to_old[k] are caller arrays of rows_k ints. */
int gs_hierarchical_reordering(const gs_hierarchy *h, int *const *old_to_new, int *const *new_to_old);
void gs_hierarchy_destroy(gs_hierarchy *h);

/* ------------------------------------------------------------------------
 * AMG-preconditioned CG on one GPU
 * (CGSolver, src/CGSolver.cc:87-306, with MultigridGaussSeidelPreconditioner
 *  src/Preconditioners/MultigridGaussSeidelPreconditioner.cc:6-54 or
 *  MultigridBlockGaussSeidelPreconditioner
 *  src/Preconditioners/MultigridBlockGaussSeidelPreconditioner.cc:8-60)
 * --------------------------------------------------------------------- */
typedef struct gs_solver gs_solver;

typedef struct {
  int smoother;      /* finest level (and every level unless coarse_smoother >= 0):
                        0 multicolour symmetric GS, 1 3x3 block symmetric GS,
                        2 damped Jacobi, 3 3x3 block Jacobi, 4 identity (one-level
                        hierarchies only) -- the reference's SmootherType */
  int pre_steps;     /* >= 1 */
  int post_steps;    /* >= 1 */
  int coarse_steps;  /* smoothing steps on the coarsest level when coarse_solver == 0 */
  int vcycles;       /* V-cycles per application, >= 1 */
  double omega;      /* relaxation weight in (0, 2) */
  int coarse_solver; /* 0 smoother on the coarsest level (the reference), 1 dense Cholesky */
  int precision;     /* 0 FP64 V-cycle, 1 FP32 V-cycle inside the FP64 CG */
  int flexible;      /* 0 beta = rho'/rho (the reference), 1 Polak-Ribiere */
  int use_graph;     /* 1 replay the iteration as a CUDA graph with a device-side stop flag */
  int check_every;   /* reserved */
  double tol;        /* relative recurrence residual; default 1e-6 as CGSolver */
  int max_iter;      /* default 1000 as CGSolver */
  int reference_vcycle; /* 1: the reference's V-cycle bit for bit, including its
                           correction/solution buffer aliasing below the finest
                           level (src/Smoothers/MultigridSmoother.cc:394-404);
                           0 (default): x_k += P x_{k+1} */
  int autotune;      /* 1 (default): threads per row chosen per level by timing
                        the candidates at setup; 0: one lane per row everywhere */
  int coarse_tail;   /* levels below the finest with <= 65536 rows run their part of
                        the V-cycle as one cluster-resident kernel: 0 never,
                        1 (default) when timed faster at setup, 2 always */
  int lanes;         /* > 0: threads per row forced everywhere (1, 4, 8, 16, 32);
                        0 (default): the autotuner decides */
  int sliced_lanes;  /* > 0: every level's smoother and residual use the sliced layout
                        (SELL-32 / BELL-32) with 1, 2, 4 or 8 lanes per row or node,
                        and so does the outer CG's 3x3 block operator, overriding the
                        autotuner for them; 0 (default): autotuned */
  int coarse_rows;   /* > 0 with coarse_solver 1: the dense coarsest solve moves up to the
                        first level below the finest with at most this many rows and the
                        levels under it are not used (no reference counterpart);
                        0 (default): the hierarchy's own coarsest level */
  int coarse_smoother; /* smoother of every level below the finest (same codes);
                          -1 (default): the same as `smoother`. 1 with smoother 1 and
                          3 below is MultigridHybridBlockPreconditioner */
  int overlap_launch; /* 2 (default): every V-cycle kernel, in captured CUDA graphs too,
                         uses programmatic dependent launch: each becomes resident while its
                         predecessor drains, loads its matrix operands and waits in-kernel
                         for its predecessor's results; 1: only kernels launched on the
                         stream (graph captures use plain edges); 0: plain stream order */
  int packed_rows;    /* dense coarsest levels with more rows keep only the lower triangle
                         of their inverse, tiled, read once per solve for both halves (half
                         the bytes); default 8192 */
  int coloring;       /* 0 (default): the reference's greedy first-fit colouring in row order;
                         1: first-fit in smallest-last order where it uses fewer colours (fewer
                         passes), else the greedy colouring; 2: as 1 on the finest level, and on
                         the coarser scalar Gauss-Seidel levels a colouring of the strong
                         couplings only (gs_relaxed_coloring, theta 0.05, rho 0.5), each pass
                         reading its own colour's neighbours from the iterate its sweep started
                         with (no reference counterpart: 5 instead of 16 colours on P128's
                         level 1) */
  int sweep_launch;   /* symmetric Gauss-Seidel steps of a scalar level: 0 one launch per
                         colour pass (the reference's structure); 1 (default) one cooperative
                         launch per smoothing step, grid barriers between colours, where timed
                         faster at setup; 2 cooperative on every such level. Colour passes of
                         a 3x3 block level in the BELL-1 layout: 1 with each slice's blocks
                         bulk-copied to shared memory where timed faster, 2 on every such
                         level whose widest slice fits, 0 never. Same iterates bit for bit
                         (no reference counterpart) */
  int half_sweeps;    /* 1: pre-smoothing is pre_steps forward colour sweeps and post-smoothing
                         post_steps backward sweeps (the symmetric pair S, S^T: half the colour
                         passes, still symmetric positive definite; no reference counterpart;
                         one launch per colour pass, whatever sweep_launch says);
                         0 (default): symmetric Gauss-Seidel steps on both sides (the reference) */
  int coarse_half;    /* 1 (FP32 V-cycle, packed dense coarsest level): its inverse stored in FP16
                         tiles with one FP32 scale each (half the bytes of the coarse solve; no
                         reference counterpart); 0 (default): tiles in the V-cycle's precision */
} gs_solver_options;

typedef struct {
  int iterations; /* CGSolver::getNbOfIterations semantics (0-based converging iteration) */
  int status;     /* GS_STATUS_* */
  int spmv;       /* outer iterations executed */
  double ratio;   /* final ||r||^2 / ||b||^2 of the recurrence residual */
  double rhs_norm2;
  double solve_ms; /* device time of the solve, CUDA events */
} gs_solve_stats;

void gs_solver_options_default(gs_solver_options *opt);
/* Path of the autotuner's decision cache used by solvers created afterwards
 * on this thread (NULL or "" = no cache). The reference has no autotuner. */
int gs_set_tune_cache(const char *path);
/* old_to_new / new_to_old: one permutation per level (the reference's
 * std::vector<Permutation>), or NULL for identity on every level. */
int gs_solver_create(const gs_hierarchy *h, const int *const *old_to_new,
                     const int *const *new_to_old, const gs_solver_options *opt, int device,
                     gs_solver **out);
/* Host arrays, FP64: copies in, solves, copies out. x: initial guess in,
 * solution out. */
int gs_solver_solve(gs_solver *s, const double *b, double *x, gs_solve_stats *stats);
/* Host arrays in FP32, the reference's CGSolver::solve(VectorXf, VectorXf). */
int gs_solver_solve_f32(gs_solver *s, const float *b, float *x, gs_solve_stats *stats);
/* Device arrays (FP64, caller order) on `stream` (a cudaStream_t, NULL for
 * the legacy default stream). Returns when the solve has finished. */
int gs_solver_solve_device(gs_solver *s, const double *b, double *x, void *stream,
                           gs_solve_stats *stats);
/* Preconditioner::apply: z = M r (device arrays, caller order). */
int gs_solver_apply_preconditioner(gs_solver *s, const double *r, double *z, void *stream);
/* CGSolver::setTolerance / setMaxIterations */
int gs_solver_set_tolerance(gs_solver *s, double tol, int max_iter);
/* Per-(level, colour) relaxation weights in (0, 2): w[level_offsets[k] + c];
 * pass w = NULL to go back to the constant omega. */
int gs_solver_set_colour_weights(gs_solver *s, const double *w, const int *level_offsets,
                                 int num_levels);
int gs_solver_num_levels(const gs_solver *s);
int gs_solver_level_info(const gs_solver *s, int level, int *rows, int *nnz, int *colors,
                         int *slices, long long *stored);
/* Threads per row the kernels of `level` use: A's smoother and residual,
 * the prolongation P (level <- level+1) and the restriction R (level ->
 * level+1); 1 means one lane per row (SELL-32). No reference counterpart. */
int gs_solver_level_format(const gs_solver *s, int level, int *lanes, int *p_lanes, int *r_lanes);
/* CTAs of the cluster-resident coarse kernel (one launch for the whole
 * coarse part of the V-cycle) if `level` runs inside it, else 0. No
 * reference counterpart. */
int gs_solver_level_in_tail(const gs_solver *s, int level);
/* Layout of `level`'s smoother and residual: 1 sliced (SELL-32 / BELL-32 with
 * gs_solver_level_format's `lanes` lanes per row or node), 0 CSR-vector with
 * `lanes` lanes per row; -1 on a bad argument. No reference counterpart. */
int gs_solver_level_layout(const gs_solver *s, int level);
/* How `level`'s colour passes are launched: 0 one kernel per colour pass,
 * 1 one cooperative kernel per smoothing step (grid barriers between the
 * colours), 2 one kernel per colour pass that bulk-copies each BELL-1
 * slice's blocks to shared memory (gs_solver_options.sweep_launch chooses);
 * -1 on a bad argument. No reference counterpart. */
int gs_solver_level_launch(const gs_solver *s, int level);
/* Average device milliseconds of one launch of a kernel, CUDA events on
 * `stream`: kind 0 outer SpMV (+ p.Ap), 1 one forward GS sweep of the finest
 * level over all colours, 2 its V-cycle residual, 3 the dense coarsest solve
 * (tile pass + reduction when the inverse is packed). */
int gs_solver_time_kernel(gs_solver *s, int kind, int reps, void *stream, double *ms);
/* One operation of `level` (a level with a coarser one below): op 0 forward
 * Gauss-Seidel sweep over all colours, 1 residual, 2 restriction,
 * 3 prolongation; `lanes` threads per row (1 = SELL-32 / BELL-32; 4, 8, 16,
 * 32 = CSR-vector; 0 = the solver's own choice). Average device ms on
 * `stream`. No reference counterpart (measurement aid for the autotuner's
 * choices). */
int gs_solver_time_level(gs_solver *s, int level, int op, int lanes, int reps, void *stream, double *ms);
/* Host wall-clock milliseconds of gs_solver_create's phases: ms4[0] levels
 * (permutation, colouring, layouts, uploads, coarsest inverse), ms4[1]
 * autotuner, ms4[2] coarse-tail decision, ms4[3] total. */
int gs_solver_setup_times(const gs_solver *s, double *ms4);
/* The same phases and, inside the levels, where their time went: ms[0..3]
 * as gs_solver_setup_times, ms[4] colouring, ms[5] permutations, ms[6]
 * smoother features, ms[7] smoother and residual layouts (build and
 * upload), ms[8] transfer layouts, ms[9] dense coarsest inverse; the first
 * `count` entries are written (entries past 9 are 0). No reference
 * counterpart (setup profiling). */
int gs_solver_setup_phases(const gs_solver *s, double *ms, int count);
/* Number of CUDA kernels this solver has launched (graph replays counted
 * kernel by kernel); no reference counterpart, used to account for the GPU
 * work inside a timed region. */
int gs_solver_launch_count(const gs_solver *s, long long *count);
void gs_solver_destroy(gs_solver *s);
/* New values for the finest-level matrix, same sparsity (`values`: nnz
 * doubles in the order of the CSR the hierarchy was built from), for
 * time-stepping callers. The coarser levels are recomputed as R A P with the
 * transfer operators kept, and every device copy is overwritten in place;
 * colouring, layouts, autotuner decisions and captured CUDA graphs stay
 * valid. Counterpart of DeviceCSRMatrix::updateValues
 * (include/GPUSolver/DeviceSparseMatrix.h:12, src/cuda/CudaDeviceCSRMatrix.cc:99-116)
 * extended to the whole hierarchy. GS_ERR_INVALID if the refreshed matrix
 * loses a diagonal or its coarsest level is not SPD. */
int gs_solver_update_matrix(gs_solver *s, const double *values);
/* Dense inverse of an SPD matrix (CSR in, n x n row-major FP64 out, host
 * arrays) on the GPU: tiled FP64 Cholesky factorisation and inverse from
 * the factor in the library's own kernels, the routine behind the dense
 * coarsest levels of more than 1000 rows. The reference's only Cholesky is
 * the per-block 3x3 LLT of extractInverseDiagonalBlocks3x3
 * (src/BlockUtils.cc:218-277). No reference counterpart (the reference smooths its coarsest
 * level); GS_ERR_INVALID if not SPD. */
int gs_dense_spd_inverse(int n, const int *row_ptr, const int *col_idx, const double *val,
                         double *inverse, int device);

/* ------------------------------------------------------------------------
 * Batched solves: many independent systems of uneven sizes, each with 1-4
 * right-hand sides, advanced together on one GPU (no reference
 * counterpart: the reference solves one system per CGSolver,
 * src/CGSolver.cc:87-306). Every (system, right-hand side) pair follows
 * that solve's semantics -- recurrence-residual stop test, 0-based
 * iteration count, zero right-hand side and already-converged exits --
 * with its own AMG V-cycle (src/Smoothers/MultigridSmoother.cc:337-420,
 * multicolour symmetric Gauss-Seidel, identity permutations) and its own
 * dense coarsest solve. One launch carries the same step of all systems
 * (work lists of (system, row slice) items); with use_graph the whole
 * iteration is one CUDA graph. The systems' R right-hand sides share each
 * matrix read.
 * Options: pre/post_steps, vcycles, omega, precision, flexible, use_graph,
 * tol, max_iter, autotune, lanes (1, 2, 4, 8, 16 or 32 here). Required:
 * smoother 0, coarse_solver 1, reference_vcycle 0, and at least two levels
 * per hierarchy.
 * --------------------------------------------------------------------- */
typedef struct gs_batch gs_batch;

/* per-pair status when the residual became NaN/Inf (batched solves report
 * it per pair instead of failing the call) */
#define GS_STATUS_NOT_FINITE 3

int gs_batch_create(int num_systems, const gs_hierarchy *const *hierarchies, int nrhs,
                    const gs_solver_options *opt, int device, gs_batch **out);
/* Host arrays, FP64. Layout of b and x: system after system; right-hand
 * side j of system s starts at (n_0 + ... + n_{s-1}) * nrhs + j * n_s and
 * holds n_s values in the caller's row order. x: initial guesses in,
 * solutions out. stats: num_systems * nrhs entries, system-major (may be
 * NULL); solve_ms is the device time of the whole batch. */
int gs_batch_solve(gs_batch *b, const double *rhs, double *x, gs_solve_stats *stats);
/* The same on device arrays, ordered on `stream` (a cudaStream_t). */
int gs_batch_solve_device(gs_batch *b, const double *rhs, double *x, void *stream,
                          gs_solve_stats *stats);
int gs_batch_set_tolerance(gs_batch *b, double tol, int max_iter);
int gs_batch_info(const gs_batch *b, int *num_systems, int *nrhs, long long *unknowns, int *levels);
int gs_batch_system_rows(const gs_batch *b, int *rows);
/* Level `level` of the batch (every system that has it): rows, nonzeros,
 * systems, colour passes per sweep, threads per row of A, P and R. */
int gs_batch_level_info(const gs_batch *b, int level, int *rows, long long *nnz, int *systems,
                        int *max_colors, int *lanes, int *p_lanes, int *r_lanes);
int gs_batch_launch_count(const gs_batch *b, long long *count);
/* Average device milliseconds of: kind 0 the outer FP64 SpMV (+ p.Ap) over
 * every system and right-hand side, 1 one forward Gauss-Seidel sweep of
 * level 0, 2 one preconditioner application; CUDA events, ordered after
 * `stream`. */
int gs_batch_time_kernel(gs_batch *b, int kind, int reps, void *stream, double *ms);
/* One operation of `level` (a level with a coarser one below): op 0 forward
 * Gauss-Seidel sweep over all colour passes, 1 residual, 2 restriction,
 * 3 prolongation; `lanes` threads per row (1 = SELL-32; 4, 8, 16, 32 =
 * CSR-vector; 0 = the batch's own choice). Average device milliseconds. */
int gs_batch_time_level(gs_batch *b, int level, int op, int lanes, int reps, void *stream, double *ms);
void gs_batch_destroy(gs_batch *b);
/* Host-only check of the batch's work lists (no GPU needed): colours every
 * level, lays the systems out and verifies that each colour of each system
 * is swept exactly once per direction and that no item crosses a system or
 * a colour. Returns the batch depth, colour passes per V-cycle sweep pair
 * and SELL-32 items. */
int gs_batch_plan_check(int num_systems, const gs_hierarchy *const *hierarchies, int *levels,
                        int *passes, long long *items);

/* ------------------------------------------------------------------------
 * Learned relaxation weights (no reference counterpart): an MLP
 * 8 -> 32 (tanh) -> 32 (tanh) -> 1, omega = 2 sigmoid(z) in (0, 2), one
 * sample per (level, colour). All arrays are device arrays of the caller;
 * parameters flat FP32 (gs_mlp_param_count values: W1[32][8], b1, W2[32][32],
 * b2, W3[32], b3); `cache` and `delta` hold 65 floats per sample.
 * --------------------------------------------------------------------- */
int gs_mlp_param_count(void);
/* omega[s] for the n samples of feats (8 floats each); cache may be NULL. */
int gs_mlp_forward(const float *params, const float *feats, int n, float *omega, float *cache,
                   void *stream);
/* grad = sum over samples of d(upstream[s] * omega[s]) / d params, given
 * the forward cache; deterministic (samples summed in order). */
int gs_mlp_backward(const float *params, const float *feats, int n, const float *cache,
                    const float *upstream, float *delta, float *grad, void *stream);
/* One Adam step (step counts from 1) on params with moments m, v. */
int gs_mlp_adam(float *params, const float *grad, float *m, float *v, int n_params, double lr,
                double beta1, double beta2, double eps, int step, void *stream);
/* The solver's 8 features per (level, colour), level-major (host array of
 * capacity floats; *count receives the number of samples). */
int gs_solver_colour_features(const gs_solver *s, float *out, int capacity, int *count);
/* Eight features per node (3x3 block row) of every level of a block
 * hierarchy, in the caller's node order, level after level: the inputs of the
 * learned per-block scalings (no reference counterpart). *count = nodes;
 * out (capacity floats, >= 8 * nodes) may be NULL to ask for the count. */
int gs_solver_node_features(const gs_solver *s, float *out, long long capacity, long long *count);
/* Per-block scalings of the 3x3 block Gauss-Seidel smoother (no reference
 * counterpart; the reference relaxes every block with one omega,
 * src/Smoothers/BlockGaussSeidelSmoother.cc:111-210): one weight in (0, 2)
 * per node of every level, in the order of gs_solver_node_features, used in
 * every forward and backward pass (the V-cycle stays symmetric positive
 * definite). n = 0 restores the colour weights / omega. */
int gs_solver_set_node_weights(gs_solver *s, const double *w, long long n);
/* ||e1||_A / ||e0||_A of one preconditioner step, e1 = e0 - M A e0, with the
 * current weights; e0 a device FP64 array in the caller's order. */
int gs_solver_error_reduction(gs_solver *s, const double *e0, void *stream, double *ratio);

/* ------------------------------------------------------------------------
 * Kernel-level operations: the reference's Backend interface
 * (include/GPUSolver/Backend.h:47-114, CUDA implementation
 * src/cuda/CudaBackend.cc and the .cu files of kernels/cuda) on device pointers.
 * Every call is asynchronous on `stream` (a cudaStream_t, NULL = legacy
 * default stream), like the reference's encode* calls; dtype selects
 * FP32 (the reference's precision) or FP64.
 * --------------------------------------------------------------------- */
#define GS_F32 0
#define GS_F64 1

typedef struct gs_device_csr gs_device_csr;

/* Backend::createCSRMatrix (src/cuda/CudaDeviceCSRMatrix.cc:28-56): copies
 * host CSR arrays (values of `dtype`) to the device. GS_ERR_INVALID, before
 * any upload, for row pointers that do not start at 0 or decrease and for
 * column indices outside [0, cols). */
int gs_device_csr_create(int rows, int cols, const int *row_ptr, const int *col_idx,
                         const void *val, int dtype, gs_device_csr **out);
/* DeviceCSRMatrix::updateValues (src/cuda/CudaDeviceCSRMatrix.cc:99-116). */
int gs_device_csr_update_values(gs_device_csr *m, const void *val, long long count);
void gs_device_csr_destroy(gs_device_csr *m);

/* encodeSpmv (src/cuda/CudaBackend.cc:397-445): y = A x. */
int gs_spmv(const gs_device_csr *A, const void *x, void *y, void *stream);
/* encodeGaussSeidelColor (src/cuda/CudaBackend.cc:447-506,
 * kernels/cuda/GaussSeidelKernels.cu:10-63): for the rows
 * color_vertices[start .. start+count) (device array), x_i <- (1-w) x_i
 * + w (b_i - sum_{j!=i} a_ij x_j) / a_ii, in place. GS_ERR_INVALID if the
 * matrix has a zero or missing diagonal entry. color_vertices lives on the
 * device and is read as given: its entries in the range must be row indices
 * in [0, rows), as for the reference's kernel. */
int gs_gauss_seidel_color(const gs_device_csr *A, const int *color_vertices, long long start,
                          long long count, const void *rhs, void *x, double omega, void *stream);
/* encodeBlockGaussSeidelColor3x3 (src/cuda/CudaBackend.cc:702-783) with the
 * (colorStart, colorCount) reading BlockGaussSeidelSmoother passes
 * (src/Smoothers/BlockGaussSeidelSmoother.cc:149-166); dinv: 9 values per
 * node, row-major (extractInverseDiagonalBlocks3x3). color_blocks lives on
 * the device and is read as given: its entries in the range must be node
 * indices in [0, rows / 3). */
int gs_block_gauss_seidel_color3x3(const gs_device_csr *A, const int *color_blocks,
                                   long long start, long long count, const void *dinv,
                                   const void *rhs, void *x, double omega, void *stream);
/* encodeApplyBlockInverses3x3 (kernels/cuda/BlockKernels.cu:9-57): c = D^-1 r,
 * n = vector length (3 per node). */
int gs_apply_block_inverses3x3(long long n, const void *dinv, const void *r, void *c, int dtype,
                               void *stream);
/* encodeDot (src/cuda/CudaBackend.cc:508-548): *result (device) = x . y,
 * accumulated in FP64, deterministic order. Uses a per-device scratch of a
 * few kilobytes that the library allocates on the first call on a device. */
int gs_dot(long long n, const void *x, const void *y, void *result, int dtype, void *stream);

/* gs_dot without any allocation, for callers that cannot allocate device
 * memory at the point where they need a dot product -- for example a code
 * that hands all of the GPU's memory to its own pool at start-up, or a
 * time-critical loop that cannot take cudaMalloc's implicit device
 * synchronisation. No counterpart in the reference.
 * Same result contract as gs_dot (FP64 accumulation, *result on the device),
 * same tolerance; the summation blocks differ, so the last bits may too.
 * Scratch: a fixed 32 KB + 256 B array inside the library's device image;
 * n is limited to 8,388,608 elements (GS_ERR_INVALID above that; use
 * gs_dot). The array takes device memory on a GPU when the library's device
 * image is loaded there: with CUDA's default lazy module loading that is the
 * library's first GPU call on that device (this one or any other gs_* call
 * that touches the GPU), which may need a little device memory. Make that
 * first call before your memory pool claims the GPU (or set
 * CUDA_MODULE_LOADING=EAGER); from then on the GPU holds the array until the
 * process exits and no call allocates. Each call looks up the array's device
 * address with the current device; make the first call on a device before
 * any stream capture. All calls share the one array: calls that can overlap
 * on the GPU (different streams, or different host threads) race on it --
 * serialise them on one stream. */
int gs_dot_noalloc(long long n, const void *x, const void *y, void *result, int dtype,
                   void *stream);

#define GS_VEC_AXPY 0            /* y += alpha x      encodeAxpy */
#define GS_VEC_SCALE 1           /* y *= alpha        encodeScale */
#define GS_VEC_COPY 2            /* y = x             encodeCopy */
#define GS_VEC_SET_ZERO 3        /* y = 0             encodeSetZero */
#define GS_VEC_SCALE_BY_VECTOR 4 /* y *= x (elementwise) encodeScaleVector */
/* Vector operations of src/cuda/CudaBackend.cc:199-394; alpha from the host,
 * or from the device scalar alpha_dev when it is not NULL (the DeviceScalar
 * overloads). */
int gs_vector_op(int op, long long n, const void *x, void *y, double alpha, const void *alpha_dev,
                 int dtype, void *stream);

#define GS_SCALAR_DIVIDE 0   /* out = a / b */
#define GS_SCALAR_MULTIPLY 1 /* out = a * b */
#define GS_SCALAR_SET 2      /* out = value */
#define GS_SCALAR_COPY 3     /* out = a */
#define GS_SCALAR_NEGATE 4   /* out = -a */
#define GS_SCALAR_SQRT 5     /* out = sqrt(a) */
/* encodeScalar{Divide,Multiply,Set,Copy,Negate,Sqrt}
 * (kernels/cuda/ScalarKernels.cu:9-62) on device scalars. */
int gs_scalar_op(int op, const void *a, const void *b, void *out, double value, int dtype,
                 void *stream);

/* ---------------------------------------------------------------------
 * Device memory, copies and streams, for callers that do not link a CUDA
 * runtime of their own: the C++ mirror's Device* handles and encoders
 * (include/GPUSolver/cuda/CudaBackend.h). The reference's CudaDevice*
 * classes and CudaEncoder call the CUDA runtime directly
 * (src/cuda/CudaDeviceVector.cc, src/cuda/CudaDeviceScalar.cc,
 * src/cuda/CudaEncoder.cc:7-15); these are the same calls behind the ABI.
 * The calling thread's current device is left as it was.
 * --------------------------------------------------------------------- */
/* cudaMalloc on `device`; bytes == 0 gives *ptr = NULL. */
int gs_device_malloc(int device, unsigned long long bytes, void **ptr);
/* cudaFree; NULL is a no-op. */
int gs_device_free(void *ptr);
#define GS_COPY_H2D 0
#define GS_COPY_D2H 1
#define GS_COPY_D2D 2
/* stream NULL: a synchronous cudaMemcpy, ordered after the work of every
 * blocking stream like the reference's; otherwise cudaMemcpyAsync on it. */
int gs_memcpy(void *dst, const void *src, unsigned long long bytes, int kind, void *stream);
/* cudaMemset (stream NULL) or cudaMemsetAsync of `bytes` bytes to byte_value. */
int gs_memset(void *dst, int byte_value, unsigned long long bytes, void *stream);
/* cudaStreamCreate on `device` (a blocking stream, as the reference's
 * encoder creates), cudaStreamDestroy, cudaStreamSynchronize. */
int gs_stream_create(int device, void **stream);
int gs_stream_destroy(void *stream);
int gs_stream_synchronize(void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GPUSOLVER_B200_H */
