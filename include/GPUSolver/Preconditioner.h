// gpuSolver::Preconditioner and the multigrid preconditioners of the
// reference (include/GPUSolver/Preconditioners/Multigrid*Preconditioner.h).
// A preconditioner here carries its hierarchy, permutations and smoothing
// parameters; the device-side V-cycle is built when a CGSolver takes it.
#pragma once
#include <vector>

#include "Smoothers/MultigridSmoother.h"
#include "cuda/CudaBackend.h"
#include "detail/b200.h"

namespace gpuSolver {

class Preconditioner {
 public:
  virtual ~Preconditioner() = default;
  // a subclass written against the reference's interface (its own
  // initialize / apply): CGSolver runs the reference's CG loop on the
  // Backend for it instead of the fused device solve
  bool custom() const { return custom_; }
  // single-level preconditioners smooth the CG's own matrix (no hierarchy)
  bool singleLevel() const { return single_level_; }
  const AMGHierarchy &hierarchy() const { return hierarchy_; }
  const std::vector<Permutation> &permutations() const { return perms_; }
  const gs_solver_options &options() const { return opt_; }
  int blockSize() const { return block_; }
  void setB200Options(const B200Options &b) {
    opt_.precision = b.precision;
    opt_.flexible = b.flexible;
    opt_.use_graph = b.useGraph;
    opt_.coarse_solver = b.coarseSolver;
    opt_.reference_vcycle = b.referenceVCycle;
    opt_.coarse_rows = b.coarseRows;
    opt_.coloring = b.coloring;
    opt_.overlap_launch = b.overlapLaunch;
    opt_.packed_rows = b.packedRows;
    opt_.sweep_launch = b.sweepLaunch;
    opt_.half_sweeps = b.halfSweeps;
    opt_.coarse_half = b.coarseHalf;
  }

  // Preconditioner::initialize / apply (include/GPUSolver/Preconditioner.h:13-20,
  // src/Preconditioners/*.cc of the reference) on the objects of any Backend:
  // apply sets output = 0 and runs the smoother on it -- numberOfVCycles
  // V-cycles of a MultigridSmoother over the hierarchy (built on first use),
  // or the single-level smoother's steps on the matrix given to initialize;
  // IdentityPreconditioner copies. CGSolver does not use these: it runs the
  // same preconditioner fused on the device.
  virtual void initialize(Backend &backend, const HostCSRMatrix &hostMatrix, const DeviceCSRMatrix &deviceMatrix) {
    if (!single_level_) {
      multigrid(backend);
      return;
    }
    if (opt_.smoother == 4) return;
    smoother_.reset();
    switch (opt_.smoother) {
      case 0: smoother_.reset(new SymmetricGaussSeidelSmoother(opt_.omega)); break;
      case 1: smoother_.reset(new BlockGaussSeidelSmoother(opt_.omega)); break;
      case 2: smoother_.reset(new DampedJacobiSmoother(opt_.omega)); break;
      default: smoother_.reset(new BlockJacobiSmoother(opt_.omega)); break;
    }
    smoother_->initialize(backend, hostMatrix, deviceMatrix);
  }
  virtual void apply(Backend &backend, BackendEncoder &encoder, const DeviceVector &input, DeviceVector &output) {
    if (single_level_ && opt_.smoother == 4) {
      backend.encodeCopy(encoder, input, output);
      return;
    }
    if (!single_level_) multigrid(backend);
    if (!smoother_) throw std::runtime_error("Preconditioner: not initialized.");
    backend.encodeSetZero(encoder, output);
    smoother_->smooth(backend, encoder, input, output,
                      static_cast<std::size_t>(single_level_ ? opt_.coarse_steps : opt_.vcycles));
  }

 protected:
  // for preconditioners written by the caller: override initialize and apply
  Preconditioner() : block_(1), custom_(true) {}
  Preconditioner(Backend &backend, const AMGHierarchy &h, const std::vector<Permutation> &perms,
                 int smoother, std::size_t pre, std::size_t post, std::size_t coarse, float omega,
                 std::size_t vcycles)
      : backend_(&backend), hierarchy_(h), block_(smoother == 1 || smoother == 3 ? 3 : 1) {
    if (h.A.empty()) throw std::runtime_error("MultigridSmoother: empty hierarchy.");
    if (perms.size() != h.A.size()) throw std::runtime_error("MultigridSmoother: invalid number of permutations.");
    if (h.P.size() + 1 != h.A.size() || h.R.size() + 1 != h.A.size())
      throw std::runtime_error("MultigridSmoother: invalid number of transfers.");
    for (const Permutation &p : perms) perms_.emplace_back(p.size(), p.oldToNew(), p.newToOld());
    gs_solver_options_default(&opt_);
    opt_.smoother = smoother;
    opt_.pre_steps = static_cast<int>(pre);
    opt_.post_steps = static_cast<int>(post);
    opt_.coarse_steps = static_cast<int>(coarse);
    opt_.vcycles = static_cast<int>(vcycles);
    opt_.omega = omega;
    setB200Options(B200Options());
  }
  // A single-level preconditioner: `steps` smoothing steps of `kind` on the
  // CG's matrix from z = 0 (Jacobi: one damped Jacobi step, omega 1).
  Preconditioner(int kind, std::size_t steps, float omega) : block_(kind == 1 || kind == 3 ? 3 : 1) {
    single_level_ = true;
    gs_solver_options_default(&opt_);
    opt_.smoother = kind;
    opt_.coarse_solver = 0;
    opt_.coarse_steps = static_cast<int>(steps);
    opt_.omega = omega;
    opt_.reference_vcycle = 0;
  }
  void setCoarseSmoother(int kind) { opt_.coarse_smoother = kind; }
  Backend *backend_ = nullptr;

 private:
  static MultigridSmoother::SmootherType type_of(int kind) {
    switch (kind) {
      case 0: return MultigridSmoother::SmootherType::SymmetricGaussSeidel;
      case 1: return MultigridSmoother::SmootherType::BlockGaussSeidel;
      case 2: return MultigridSmoother::SmootherType::DampedJacobi;
      default: return MultigridSmoother::SmootherType::BlockJacobi;
    }
  }
  void multigrid(Backend &backend) {
    if (smoother_) return;
    const int coarse = opt_.coarse_smoother >= 0 ? opt_.coarse_smoother : opt_.smoother;
    smoother_.reset(new MultigridSmoother(backend, hierarchy_, perms_, type_of(opt_.smoother), type_of(coarse),
                                          static_cast<std::size_t>(opt_.pre_steps),
                                          static_cast<std::size_t>(opt_.post_steps),
                                          static_cast<std::size_t>(opt_.coarse_steps), opt_.omega));
  }
  std::unique_ptr<Smoother> smoother_;

  AMGHierarchy hierarchy_;
  std::vector<Permutation> perms_;
  gs_solver_options opt_{};
  int block_;
  bool single_level_ = false;
  bool custom_ = false;
};

// src/Preconditioners/MultigridGaussSeidelPreconditioner.cc:6-25: coarsest
// level smoothed pre + post times.
class MultigridGaussSeidelPreconditioner : public Preconditioner {
 public:
  MultigridGaussSeidelPreconditioner(Backend &backend, const AMGHierarchy &hierarchy,
                                     const std::vector<Permutation> &permutations,
                                     std::size_t preSmoothingSteps, std::size_t postSmoothingSteps,
                                     std::size_t numberOfVCycles, float omega)
      : Preconditioner(backend, hierarchy, permutations, 0, preSmoothingSteps, postSmoothingSteps,
                       preSmoothingSteps + postSmoothingSteps, omega, numberOfVCycles) {}
};

// src/Preconditioners/MultigridDampedJacobiPreconditioner.cc: damped Jacobi on
// every level, coarsest level smoothed pre + post times.
class MultigridDampedJacobiPreconditioner : public Preconditioner {
 public:
  MultigridDampedJacobiPreconditioner(Backend &backend, const AMGHierarchy &hierarchy,
                                      const std::vector<Permutation> &permutations,
                                      std::size_t preSmoothingSteps, std::size_t postSmoothingSteps,
                                      std::size_t numberOfVCycles, float omega)
      : Preconditioner(backend, hierarchy, permutations, 2, preSmoothingSteps, postSmoothingSteps,
                       preSmoothingSteps + postSmoothingSteps, omega, numberOfVCycles) {}
};

// src/Preconditioners/MultigridBlockJacobiPreconditioner.cc: 3x3 block Jacobi on every level.
class MultigridBlockJacobiPreconditioner : public Preconditioner {
 public:
  MultigridBlockJacobiPreconditioner(Backend &backend, const AMGHierarchy &hierarchy,
                                     const std::vector<Permutation> &permutations,
                                     std::size_t preSmoothingSteps, std::size_t postSmoothingSteps,
                                     std::size_t coarseSmoothingSteps, float omega,
                                     std::size_t numberOfVCycles = 1)
      : Preconditioner(backend, hierarchy, permutations, 3, preSmoothingSteps, postSmoothingSteps,
                       coarseSmoothingSteps, omega, numberOfVCycles) {}
};

// src/Preconditioners/MultigridHybridBlockPreconditioner.cc: 3x3 block GS on the
// finest level, 3x3 block Jacobi on every coarser one.
class MultigridHybridBlockPreconditioner : public Preconditioner {
 public:
  MultigridHybridBlockPreconditioner(Backend &backend, const AMGHierarchy &hierarchy,
                                     const std::vector<Permutation> &permutations,
                                     std::size_t preSmoothingSteps, std::size_t postSmoothingSteps,
                                     std::size_t coarseSmoothingSteps, float omega,
                                     std::size_t numberOfVCycles = 1)
      : Preconditioner(backend, hierarchy, permutations, 1, preSmoothingSteps, postSmoothingSteps,
                       coarseSmoothingSteps, omega, numberOfVCycles) {
    setCoarseSmoother(3);
  }
};

// Single-level preconditioners (src/Preconditioners/*.cc): z = 0, then the
// smoother's steps on the CG's matrix.
class JacobiPreconditioner : public Preconditioner {
 public:
  JacobiPreconditioner() : Preconditioner(2, 1, 1.0f) {}
};
class DampedJacobiPreconditioner : public Preconditioner {
 public:
  DampedJacobiPreconditioner(std::size_t nSmoother, float weight) : Preconditioner(2, nSmoother, weight) {}
};
class BlockJacobiPreconditioner : public Preconditioner {
 public:
  BlockJacobiPreconditioner(std::size_t nSmoother, float weight) : Preconditioner(3, nSmoother, weight) {}
};
class SymmetricGaussSeidelPreconditioner : public Preconditioner {
 public:
  explicit SymmetricGaussSeidelPreconditioner(float omega = 1.0f, std::size_t nbOfIters = 1)
      : Preconditioner(0, nbOfIters, omega) {}
};
class BlockGaussSeidelPreconditioner : public Preconditioner {
 public:
  explicit BlockGaussSeidelPreconditioner(float omega = 1.0f, std::size_t numberOfSweeps = 1)
      : Preconditioner(1, numberOfSweeps, omega) {}
};
class IdentityPreconditioner : public Preconditioner {
 public:
  IdentityPreconditioner() : Preconditioner(4, 1, 1.0f) {}
};

// src/Preconditioners/MultigridBlockGaussSeidelPreconditioner.cc:8-29
class MultigridBlockGaussSeidelPreconditioner : public Preconditioner {
 public:
  MultigridBlockGaussSeidelPreconditioner(Backend &backend, const AMGHierarchy &hierarchy,
                                          const std::vector<Permutation> &permutations,
                                          std::size_t preSmoothingSteps, std::size_t postSmoothingSteps,
                                          std::size_t coarseSmoothingSteps, float omega,
                                          std::size_t numberOfVCycles = 1)
      : Preconditioner(backend, hierarchy, permutations, 1, preSmoothingSteps, postSmoothingSteps,
                       coarseSmoothingSteps, omega, numberOfVCycles) {}
};

}  // namespace gpuSolver
