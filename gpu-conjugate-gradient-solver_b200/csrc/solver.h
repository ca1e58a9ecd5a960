// AMG-preconditioned CG on one GPU: the device-side counterpart of the
// reference's CGSolver (src/CGSolver.cc:87-306) driving a multigrid
// preconditioner (src/Smoothers/MultigridSmoother.cc:337-420) with
// multicolour symmetric Gauss-Seidel or 3x3 block Gauss-Seidel smoothing.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "setup.h"

namespace gsb {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};
void cuda_check(cudaError_t e, const char *what);

struct SolverOptions {
  // Smoother of the finest level (and of every level unless coarse_smoother
  // is set): 0 multicolour SGS, 1 3x3 block SGS, 2 damped Jacobi, 3 3x3 block
  // Jacobi, 4 identity (single-level hierarchies only: IdentityPreconditioner).
  int smoother = 0;
  // Smoother of every level below the finest (MultigridSmoother's second
  // type, src/Smoothers/MultigridSmoother.cc:78-135); -1: the same as smoother.
  int coarse_smoother = -1;
  int pre = 1, post = 1;   // symmetric smoothing steps before / after the coarse correction
  int coarse_steps = 2;    // smoothing steps on the coarsest level when coarse == 0
  int vcycles = 1;         // V-cycles per preconditioner application
  double omega = 1.0;      // relaxation weight, in (0, 2)
  int coarse = 1;          // 0: smoother on the coarsest level (the reference), 1: dense Cholesky
  int mixed = 0;           // 0: FP64 V-cycle, 1: FP32 V-cycle (storage and arithmetic)
  int flexible = 0;        // 0: beta = rho'/rho (the reference), 1: Polak-Ribiere
  int graph = 0;           // 1: capture the CG iteration in a CUDA graph, device-side stop
  int check_every = 8;     // reserved
  // 1: reproduce the reference V-cycle exactly, including its buffer
  // aliasing below the finest level (the coarse correction overwrites the
  // pre-smoothed iterate and is added to itself,
  // src/Smoothers/MultigridSmoother.cc:394-404); 0: x_k += P x_{k+1}.
  int reference_vcycle = 0;
  // 1: pick threads-per-row per level and transfer operator by timing the
  // candidates at setup; 0: one lane per row (SELL-32) everywhere.
  int autotune = 1;
  // > 0: threads per row forced on every level and transfer operator
  // (1, 4, 8, 16 or 32), overriding the autotuner; 0: the autotuner decides.
  int lanes = 0;
  // > 0: the smoother and residual of every level use the sliced layout
  // (SELL-32 / BELL-32) with this many lanes per row or node (1, 2, 4 or 8),
  // and so does the outer CG's 3x3 block operator, overriding the autotuner
  // for them; 0: the autotuner decides.
  int sliced_lanes = 0;
  // File of cached autotuner decisions ("" = no cache). A hierarchy seen
  // before (same level sizes, nonzeros, colours and precision) reuses the
  // recorded threads-per-row instead of timing the candidates again.
  std::string tune_cache;
  // Levels (below the finest) whose rows are all at most this many run
  // their part of the V-cycle as one cluster-resident kernel when that is
  // faster than one launch per pass (decided by timing at setup); 0 = never.
  int tail_rows = 65536;
  int tail = 1;  // 0 never, 1 when timed faster at setup, 2 always (if the levels qualify)
  // > 0 (with coarse == 1): the dense coarsest solve moves up to the first
  // level below the finest with at most this many rows, and the levels under
  // it are not used (their colour passes are latency-bound; a dense inverse
  // of a few thousand rows is one bandwidth-bound matvec). 0: the
  // hierarchy's own coarsest level.
  int coarse_rows = 0;
  // 2: V-cycle kernels carry programmatic stream serialization, in captured
  // graphs too (programmatic edges): each one's CTAs become resident while
  // its predecessor drains, load the matrix operands that a solve never
  // changes, and wait in-kernel for the predecessor's results; 1: only
  // kernels launched on the stream (graph captures use plain edges);
  // 0: plain order.
  int overlap_launch = 2;
  // Dense coarsest levels with more rows than this keep only the lower
  // triangle of their inverse, in tiles read once per solve for both halves
  // (half the bytes); smaller ones the full row-major inverse, which the
  // cluster-resident coarse tail can also read. The tail is off when packed.
  int packed_rows = 8192;
  // Multicolouring of every level: 0 the reference's greedy first-fit in row
  // order (GraphColoring::compute), 1 the same first-fit in smallest-last
  // order where that uses fewer colours (usually: fewer colour passes per
  // sweep), else the greedy colouring (kept at once on a level it colours
  // with two); 2 as 1 on the finest level and, on the coarser scalar
  // Gauss-Seidel levels, a colouring of the strong couplings only
  // (relaxed_coloring) whose passes read their own colour's neighbours from
  // the iterate the sweep started with. A value refresh keeps the colouring.
  int coloring = 0;
  // Symmetric Gauss-Seidel sweeps of a scalar level: 0 one launch per colour
  // pass (the reference's structure), 1 the whole smoothing step as one
  // cooperative launch with grid barriers between colours where that is
  // timed faster at setup, 2 cooperative on every such level. Colour passes
  // of a 3x3 block level in the BELL-1 layout: 1 with each slice's blocks
  // bulk-copied to shared memory where timed faster, 2 on every such level
  // whose widest slice fits, 0 never. The iterates are the same bit for bit.
  int sweep_launch = 1;
  // 1: pre-smoothing is `pre` forward colour sweeps and post-smoothing `post`
  // backward sweeps (the symmetric pair S, S^T of a textbook V-cycle: half the
  // colour passes of symmetric steps, the preconditioner stays symmetric
  // positive definite); 0: symmetric Gauss-Seidel steps on both sides (the
  // reference's SymmetricGaussSeidelSmoother / BlockGaussSeidelSmoother).
  int half_sweeps = 0;
  // 1 (FP32 V-cycle, packed dense coarsest level): the inverse's tiles are
  // stored in FP16, each with one FP32 scale (its largest magnitude / 16384),
  // halving the bytes of the coarse solve; products still in FP32, sums in
  // FP64. 0: tiles in the V-cycle's precision.
  int coarse_half = 0;
  double tol = 1e-6;       // stop when ||r||^2 / ||b||^2 < tol^2 (recurrence residual)
  int max_iter = 1000;
};

struct SolveStats {
  int iterations = 0;      // the reference's count: 0-based index of the converging iteration
  int status = 0;          // CgStatus
  int spmv = 0;            // outer SpMVs performed
  double ratio = 0.0;      // final ||r||^2 / ||b||^2 (recurrence)
  double bb = 0.0;
  double solve_ms = 0.0;   // device time of the solve (CUDA events)
};

// Per-(level, colour) relaxation weights, ordered level-major, colour-minor;
// empty means omega everywhere.
struct ColourWeights {
  std::vector<double> w;
  std::vector<int> level_offset;  // levels + 1
};

struct LevelInfo {
  int rows = 0, nnz = 0, colors = 0, slices = 0;
  long long stored = 0;  // stored (padded) entries of the level matrix
  int lanes = 1, p_lanes = 1, r_lanes = 1;  // threads per row: A, P (to this level's fine side), R
  int sliced = 1;                           // A's layout: 1 sliced (SELL / BELL), 0 CSR-vector
  int in_tail = 0;                          // 1: runs inside the cluster-resident coarse kernel
  int tail_ctas = 0;                        // CTAs of that kernel's cluster
  int launch = 0;                           // colour passes: 0 one launch each, 1 one cooperative
                                            // launch per smoothing step, 2 bulk-copy staged (BELL-1)
};

class Solver {
 public:
  // `o2n[k]`, `n2o[k]`: the caller's permutation of level k (nullptr for
  // identity), as the reference's MultigridSmoother takes them.
  static std::unique_ptr<Solver> create(const Hierarchy &h,
                                        const std::vector<const int *> &o2n,
                                        const std::vector<const int *> &n2o,
                                        const SolverOptions &opt, int device);
  virtual ~Solver() = default;

  // b and x are device arrays in the caller's (unpermuted) order; x holds the
  // initial guess on entry. All work is queued on `stream`; the call returns
  // once the solve has finished.
  virtual void solve_device(const double *b, double *x, cudaStream_t stream, SolveStats *st) = 0;
  // Host arrays: copies in, solves, copies out (the end-to-end path).
  virtual void solve_host(const double *b, double *x, SolveStats *st) = 0;
  // Applies the preconditioner once, z = M r, arrays in the caller's order
  // (device pointers).
  virtual void apply_preconditioner(const double *r, double *z, cudaStream_t stream) = 0;
  // Times `reps` launches of one kernel with CUDA events on `stream`: kind
  // 0 = SpMV of the outer CG (y = A p), 1 = one full forward Gauss-Seidel
  // sweep over all colours of the finest level, 2 = the finest V-cycle
  // residual, 3 = the dense coarsest solve (both launches when packed).
  // Returns the average milliseconds per launch (per sweep / solve).
  virtual double time_kernel(int kind, int reps, cudaStream_t stream) = 0;
  // One operation of `level` (which must have a coarser level): op 0 forward
  // Gauss-Seidel sweep over all colours, 1 residual, 2 restriction,
  // 3 prolongation, with `lanes` threads per row (0 = the solver's own
  // choice). Average device ms, CUDA events on `stream`.
  virtual double time_level(int level, int op, int lanes, int reps, cudaStream_t stream) = 0;
  virtual void set_weights(const ColourWeights &w) = 0;
  // New values of the finest-level matrix (the caller's CSR order, the
  // sparsity the solver was built with): every coarser level is recomputed as
  // R_k A_k P_k with the transfer operators kept, and every device copy of
  // the levels (all layouts, Jacobi and block inverses, the dense coarsest
  // inverse, the outer CG's matrix) is overwritten in place. Colouring,
  // layouts and autotuner decisions are kept.
  virtual void update_values(const double *a0_values) = 0;
  // Host wall-clock milliseconds of the setup phases: {levels (permutation,
  // colouring, layouts, uploads, coarsest inverse), autotuner, coarse-tail
  // decision, total}.
  virtual std::vector<double> setup_times() const = 0;
  virtual std::vector<LevelInfo> level_info() const = 0;
  virtual int device() const = 0;
  virtual int rows() const = 0;
  virtual const SolverOptions &options() const = 0;
  virtual void set_tolerance(double tol, int max_iter) = 0;
  // Kernels this solver has launched so far (graph replays included).
  virtual long long launches() const = 0;
  // Eight features per (level, colour), level-major and colour-minor, for
  // the learned relaxation weights: level depth, colour position, colour
  // size, mean and minimum diagonal dominance, diagonal contrast, row
  // length, colour fraction (all scaled to about [0, 1]).
  virtual std::vector<float> colour_features() const = 0;
  // Eight features per node (3x3 block row) of every level of a block
  // hierarchy, in the caller's node order: level depth, colour position,
  // block diagonal dominance, off-diagonal block contrast, blocks per row,
  // diagonal block norm against the level's mean, diagonal anisotropy,
  // colour share. Empty for scalar hierarchies.
  virtual std::vector<float> node_features() const = 0;
  // A relaxation weight in (0, 2) per node of every level (the order of
  // node_features), used by the 3x3 block Gauss-Seidel passes in place of
  // the colour weight; the same weight in every sweep, so the V-cycle stays
  // symmetric positive definite. Empty restores the colour weights / omega.
  virtual void set_node_weights(const std::vector<double> &w) = 0;
  // ||e1||_A / ||e0||_A for one preconditioner application used as a
  // stationary step, e1 = e0 - M A e0; e0 is a device array in the caller's
  // order (FP64).
  virtual double error_reduction(const double *e0, cudaStream_t stream) = 0;
};

}  // namespace gsb
