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

// True when every row of `a` has strictly increasing column indices.
bool rows_sorted_unique(const Csr &a);

}  // namespace gsb
