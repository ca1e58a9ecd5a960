// Smoothed-aggregation setup on the GPU: the hierarchy that build_hierarchy
// (setup.cc) computes with SaOptions::aggregation == 1, built level by level
// on one device and returned as host CSR levels.
#pragma once

#include "setup.h"

namespace gsb {

struct DeviceSetupStats {
  double total_ms = 0.0;     // host wall clock of the whole build
  double upload_ms = 0.0;    // finest matrix to the device
  double build_ms = 0.0;     // all coarsening steps (device work, host-synchronised)
  double download_ms = 0.0;  // levels, transfers and aggregates back to the host
  int mis_rounds = 0;        // independent-set rounds summed over the levels
};

// `a` must hold sorted, duplicate-free column indices in every row (the
// host build walks the same entries in the same order). Throws
// std::runtime_error on invalid input or a CUDA error.
Hierarchy build_hierarchy_device(const Csr &a, const SaOptions &opt, int device, DeviceSetupStats *stats);

// Value refresh of a hierarchy on the GPU: level 0 is a0 (new values on the
// hierarchy's finest sparsity), A_{k+1} = R_k (A_k P_k) for k < levels - 1
// with the transfer operators kept -- the same sparse products as the setup,
// bit-identical to the host's spgemm. Throws (nothing computed) on a row of a
// product with more than 1024 columns or unsorted input rows.
std::vector<Csr> galerkin_device(const Csr &a0, const std::vector<Csr> &P, const std::vector<Csr> &R, int levels,
                                 int device);

// True when every row of `a` has strictly increasing column indices.
bool rows_sorted_unique(const Csr &a);

}  // namespace gsb
