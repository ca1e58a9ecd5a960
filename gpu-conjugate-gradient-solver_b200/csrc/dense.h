// Dense SPD inverse on the GPU (coarsest levels of thousands of rows).
#pragma once

#include <cuda_runtime.h>

#include "setup.h"

namespace gsb {

// A^-1 of the SPD matrix `m` (FP64, row-major n x n) into device memory
// d_out (n * n doubles): tiled Cholesky factorisation and inversion from the
// factor in the library's own kernels, on `s`. With `lower_only` only the
// 64 x 64 tiles on and below the diagonal are written (the diagonal tiles in
// full). Synchronises `s`; throws if the factorisation fails (matrix not SPD).
void spd_inverse_device(const Csr &m, double *d_out, cudaStream_t s, bool lower_only = false);

// Levels of a hierarchy the V-cycle uses when the dense coarsest solve may
// move up to the first level with at most `coarse_rows` rows (k >= 1):
// min(own depth, depth_limit) where depth_limit is that first level + 1
// (for a batch: the largest such over all systems). coarse_rows <= 0 keeps
// every level.
int dense_depth(const std::vector<int> &level_rows, int coarse_rows);

}  // namespace gsb
