// Batched AMG-PCG: many independent SPD systems of uneven sizes, each with
// up to four right-hand sides, solved together on one GPU. No counterpart in
// the reference, which solves one system per CGSolver (src/CGSolver.cc:87-306);
// every (system, right-hand side) pair follows that solve's semantics
// (iteration count, stop test, zero right-hand side, early exits) with the
// multigrid preconditioner of src/Smoothers/MultigridSmoother.cc:337-420.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "setup.h"
#include "solver.h"

namespace gsb {

struct BatchLevelInfo {
  int rows = 0;          // rows of the batch level (all systems that reach it)
  long long nnz = 0;
  int systems = 0;       // systems with this level
  int smoothed = 0;      // systems for which it is not the coarsest level
  int max_colors = 0;    // colour passes per sweep
  int lanes = 1, p_lanes = 1, r_lanes = 1;  // threads per row (1 = SELL-32)
  long long sweep_items = 0;  // work-list items of one forward sweep
};

class BatchSolver {
 public:
  virtual ~BatchSolver() = default;
  // b, x: caller layout, system after system, right-hand side j of system s
  // at offset (sum_{t<s} n_t) * nrhs + j * n_s; x is the initial guess on
  // entry. stats: one entry per (system, right-hand side), system-major.
  virtual void solve_device(const double *b, double *x, cudaStream_t stream,
                            std::vector<SolveStats> &stats) = 0;
  virtual void solve_host(const double *b, double *x, std::vector<SolveStats> &stats) = 0;
  virtual void set_tolerance(double tol, int max_iter) = 0;
  virtual int num_systems() const = 0;
  virtual int nrhs() const = 0;
  virtual const std::vector<int> &system_rows() const = 0;
  virtual const std::vector<BatchLevelInfo> &level_info() const = 0;
  virtual long long launches() const = 0;
  // Average device milliseconds of one launch sequence, CUDA events on the
  // solver's stream after `stream`: kind 0 outer FP64 SpMV (+ p.Ap) over all
  // systems and right-hand sides, 1 one forward Gauss-Seidel sweep of level 0
  // (all colour passes), 2 one preconditioner application (V-cycle).
  virtual double time_kernel(int kind, int reps, cudaStream_t stream) = 0;
  // One operation of `level` (which must have a coarser level): op 0 forward
  // Gauss-Seidel sweep, 1 residual, 2 restriction, 3 prolongation, with
  // `lanes` threads per row (0 = the solver's own choice). Average ms.
  virtual double time_level(int level, int op, int lanes, int reps, cudaStream_t stream) = 0;
};

// Options honoured: pre, post, vcycles, omega, mixed, flexible, graph, tol,
// max_iter, autotune, lanes. Required: smoother 0 (scalar SGS), coarse 1
// (dense coarsest solve), reference_vcycle 0, at least two levels per system.
std::unique_ptr<BatchSolver> make_batch_solver(const std::vector<const Hierarchy *> &h, int nrhs,
                                               const SolverOptions &opt, int device);

// Host-only check of the batch plan (colouring, layout, work lists of every
// format): every colour of every system is covered exactly once by the
// forward and once by the backward passes, items never cross systems or
// colours. Throws on a violation.
struct BatchPlanStats {
  int levels = 0;
  int passes = 0;        // colour passes of one V-cycle sweep pair (forward + backward, all levels)
  long long items = 0;   // items of all passes, SELL-32 format
};
BatchPlanStats check_batch_plan(const std::vector<const Hierarchy *> &h);

}  // namespace gsb
