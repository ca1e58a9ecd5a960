// gpuSolver::MultigridSmoother (include/GPUSolver/Smoothers/MultigridSmoother.h,
// src/Smoothers/MultigridSmoother.cc:22-445 of the reference): the V-cycle
// composed of Backend operations on FP32 device objects. Level k holds
// A_k permuted by its permutation on both sides, P_k / R_k permuted by the
// permutations of the two levels they join, a single-level smoother (the
// fine type on level 0, the coarse type below) and four work vectors. One
// iteration of smooth() is one V-cycle on `solution`:
//   pre-smooth; r = b - A x; b_c = R r; e_c = 0; recurse on (b_c, e_c);
//   e = P e_c; x += e; post-smooth;  the coarsest level is smoothed
//   coarseSmoothingSteps times.
// On every level below the finest the V-cycle's solution vector is that
// level's correction vector, so P e_c is written over the solution before it
// is added to itself, exactly as the reference's buffers do; the product's
// fused solver reproduces the same V-cycle with its reference_vcycle option.
//
// This class runs on any Backend implementation; the B200 path for a full
// solve is CGSolver with a Multigrid*Preconditioner, which fuses the same
// V-cycle into CUDA-graph-replayed kernels.
#pragma once
#include <memory>
#include <vector>

#include "../AMGHierarchy.h"
#include "../Permutation.h"
#include "../SparseMatrixUtils.h"
#include "BlockGaussSeidelSmoother.h"
#include "BlockJacobiSmoother.h"
#include "DampedJacobiSmoother.h"
#include "SymmetricGaussSeidelSmoother.h"

namespace gpuSolver {

class MultigridSmoother : public Smoother {
 public:
  enum class SmootherType { DampedJacobi, SymmetricGaussSeidel, BlockJacobi, BlockGaussSeidel };

  MultigridSmoother(Backend &backend, const AMGHierarchy &hierarchy, const std::vector<Permutation> &permutations,
                    SmootherType smootherType, std::size_t preSmoothingSteps, std::size_t postSmoothingSteps,
                    std::size_t coarseSmoothingSteps, float omega)
      : MultigridSmoother(backend, hierarchy, permutations, smootherType, smootherType, preSmoothingSteps,
                          postSmoothingSteps, coarseSmoothingSteps, omega) {}

  MultigridSmoother(Backend &backend, const AMGHierarchy &hierarchy, const std::vector<Permutation> &permutations,
                    SmootherType fineSmootherType, SmootherType coarseSmootherType, std::size_t preSmoothingSteps,
                    std::size_t postSmoothingSteps, std::size_t coarseSmoothingSteps, float omega)
      : pre_(preSmoothingSteps), post_(postSmoothingSteps), coarse_(coarseSmoothingSteps) {
    const std::size_t L = hierarchy.A.size();
    if (L == 0) throw std::runtime_error("MultigridSmoother: empty hierarchy.");
    if (permutations.size() != L) throw std::runtime_error("MultigridSmoother: invalid number of permutations.");
    if (hierarchy.P.size() + 1 != L || hierarchy.R.size() + 1 != L)
      throw std::runtime_error("MultigridSmoother: invalid number of transfers.");
    levels_.resize(L);
    transfers_.resize(L - 1);
    for (std::size_t k = 0; k < L; ++k) {
      const int *pk = permutations[k].oldToNew();
      const HostCSRMatrix hostA(permuteMatrix(hierarchy.A[k], pk, pk));
      Level &lv = levels_[k];
      lv.matrix.reset(backend.createCSRMatrix(hostA));
      lv.smoother = make_smoother(k == 0 ? fineSmootherType : coarseSmootherType, omega);
      lv.smoother->initialize(backend, hostA, *lv.matrix);
      const std::size_t n = hostA.rows();
      lv.rhs.reset(backend.createVector(n));
      lv.residual.reset(backend.createVector(n));
      lv.correction.reset(backend.createVector(n));
      lv.Az.reset(backend.createVector(n));
      if (k > 0) {
        const int *pf = permutations[k - 1].oldToNew();
        const HostCSRMatrix hostP(permuteMatrix(hierarchy.P[k - 1], pf, pk));
        const HostCSRMatrix hostR(permuteMatrix(hierarchy.R[k - 1], pk, pf));
        transfers_[k - 1].prolongation.reset(backend.createCSRMatrix(hostP));
        transfers_[k - 1].restriction.reset(backend.createCSRMatrix(hostR));
      }
    }
  }
  MultigridSmoother(const MultigridSmoother &) = delete;
  MultigridSmoother &operator=(const MultigridSmoother &) = delete;

  // the levels are set up by the constructor (as in the reference)
  void initialize(Backend &, const HostCSRMatrix &, const DeviceCSRMatrix &) override {}

  void smooth(Backend &backend, BackendEncoder &encoder, const DeviceVector &rhs, DeviceVector &solution,
              std::size_t iterations) override {
    for (std::size_t i = 0; i < iterations; ++i) vcycle(backend, encoder, 0, rhs, solution);
  }

 private:
  struct Level {
    std::unique_ptr<DeviceCSRMatrix> matrix;
    std::unique_ptr<Smoother> smoother;
    std::unique_ptr<DeviceVector> rhs, residual, correction, Az;
  };
  struct Transfer {
    std::unique_ptr<DeviceCSRMatrix> restriction, prolongation;
  };

  static std::unique_ptr<Smoother> make_smoother(SmootherType t, float omega) {
    switch (t) {
      case SmootherType::DampedJacobi: return std::unique_ptr<Smoother>(new DampedJacobiSmoother(omega));
      case SmootherType::SymmetricGaussSeidel:
        return std::unique_ptr<Smoother>(new SymmetricGaussSeidelSmoother(omega));
      case SmootherType::BlockJacobi: return std::unique_ptr<Smoother>(new BlockJacobiSmoother(omega));
      case SmootherType::BlockGaussSeidel: return std::unique_ptr<Smoother>(new BlockGaussSeidelSmoother(omega));
    }
    throw std::runtime_error("MultigridSmoother: unsupported smoother type.");
  }

  void vcycle(Backend &backend, BackendEncoder &encoder, std::size_t k, const DeviceVector &rhs,
              DeviceVector &solution) {
    Level &lv = levels_[k];
    if (k + 1 == levels_.size()) {
      lv.smoother->smooth(backend, encoder, rhs, solution, coarse_);
      return;
    }
    lv.smoother->smooth(backend, encoder, rhs, solution, pre_);
    backend.encodeSpmv(encoder, *lv.matrix, solution, *lv.Az);
    backend.encodeCopy(encoder, rhs, *lv.residual);
    backend.encodeAxpy(encoder, -1.0f, *lv.Az, *lv.residual);
    Level &next = levels_[k + 1];
    backend.encodeSpmv(encoder, *transfers_[k].restriction, *lv.residual, *next.rhs);
    backend.encodeSetZero(encoder, *next.correction);
    vcycle(backend, encoder, k + 1, *next.rhs, *next.correction);
    backend.encodeSpmv(encoder, *transfers_[k].prolongation, *next.correction, *lv.correction);
    backend.encodeAxpy(encoder, 1.0f, *lv.correction, solution);
    lv.smoother->smooth(backend, encoder, rhs, solution, post_);
  }

  std::vector<Level> levels_;
  std::vector<Transfer> transfers_;
  std::size_t pre_, post_, coarse_;
};

// src/Smoothers/ of the reference: the three fixed choices of smoother types.
class MultigridGaussSeidelSmoother : public MultigridSmoother {
 public:
  MultigridGaussSeidelSmoother(Backend &backend, const AMGHierarchy &hierarchy,
                               const std::vector<Permutation> &permutations, std::size_t preSmoothingSteps,
                               std::size_t postSmoothingSteps, std::size_t coarseSmoothingSteps, float omega)
      : MultigridSmoother(backend, hierarchy, permutations, SmootherType::SymmetricGaussSeidel, preSmoothingSteps,
                          postSmoothingSteps, coarseSmoothingSteps, omega) {}
};

class MultigridDampedJacobiSmoother : public MultigridSmoother {
 public:
  MultigridDampedJacobiSmoother(Backend &backend, const AMGHierarchy &hierarchy,
                                const std::vector<Permutation> &permutations, std::size_t preSmoothingSteps,
                                std::size_t postSmoothingSteps, std::size_t coarseSmoothingSteps, float omega)
      : MultigridSmoother(backend, hierarchy, permutations, SmootherType::DampedJacobi, preSmoothingSteps,
                          postSmoothingSteps, coarseSmoothingSteps, omega) {}
};

class MultigridHybridBlockSmoother : public MultigridSmoother {
 public:
  MultigridHybridBlockSmoother(Backend &backend, const AMGHierarchy &hierarchy,
                               const std::vector<Permutation> &permutations, std::size_t preSmoothingSteps,
                               std::size_t postSmoothingSteps, std::size_t coarseSmoothingSteps, float omega)
      : MultigridSmoother(backend, hierarchy, permutations, SmootherType::BlockGaussSeidel, SmootherType::BlockJacobi,
                          preSmoothingSteps, postSmoothingSteps, coarseSmoothingSteps, omega) {}
};

}  // namespace gpuSolver
