// C ABI of gpusolver_b200 (declarations and reference citations in
// include/gpusolver_b200.h). Each entry point converts C++ exceptions into
// status codes and a thread-local message.
#include "gpusolver_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <string>
#include <vector>

#include "setup.h"
#include "solver.h"
#include "batch.h"
#include "dense.h"
#include "backend.h"
#include "mlp.h"
#include "amg_setup.h"

struct gs_host_csr {
  gsb::Csr a;
  std::vector<double> rhs;
};

struct gs_hierarchy {
  gsb::Hierarchy h;
};

struct gs_device_csr {
  std::unique_ptr<gsb::DeviceCsr> m;
};

struct gs_batch {
  std::unique_ptr<gsb::BatchSolver> b;
};

struct gs_solver {
  std::unique_ptr<gsb::Solver> s;
  std::vector<double> hb, hx;  // FP32 entry point staging
};

namespace {

thread_local std::string g_error;
thread_local std::string g_tune_cache;

template <typename F>
int guarded(F &&f) {
  try {
    return f();
  } catch (const gsb::CudaError &e) {
    g_error = e.what();
    return GS_ERR_CUDA;
  } catch (const std::exception &e) {
    g_error = e.what();
    const std::string m = e.what();
    if (m.find("NaN/Inf") != std::string::npos) return GS_ERR_NOT_FINITE;
    return GS_ERR_INVALID;
  }
}

int fail(const char *msg, int code = GS_ERR_INVALID) {
  g_error = msg;
  return code;
}

// Row pointers are checked before anything is read through them: they start
// at 0 and never decrease, so rp[rows] is the entry count.
void check_row_ptr(int rows, const int *rp, const char *what) {
  const std::string w(what);
  if (rows < 0) throw std::runtime_error(w + ": negative dimensions");
  if (rp == nullptr) throw std::runtime_error(w + ": input pointers must not be null.");
  if (rp[0] != 0) throw std::runtime_error(w + ": row pointer must start at 0");
  for (int i = 0; i < rows; ++i)
    if (rp[i + 1] < rp[i]) throw std::runtime_error(w + ": row pointer decreases");
}

// The graph entry points (colourings, RCM, node graph) read rp[0..n] and
// ci[0..rp[n]) and index arrays of size n with every ci.
void check_graph(int n, const int *rp, const int *ci, const char *what) {
  check_row_ptr(n, rp, what);
  if (rp[n] > 0 && ci == nullptr) throw std::runtime_error(std::string(what) + ": input pointers must not be null.");
  for (int k = 0; k < rp[n]; ++k)
    if (ci[k] < 0 || ci[k] >= n) throw std::runtime_error(std::string(what) + ": column index out of range");
}

void check_outputs(std::initializer_list<const void *> out, const char *what) {
  for (const void *p : out)
    if (p == nullptr) throw std::runtime_error(std::string(what) + ": output pointers must not be null.");
}

// permuteMatrix places entry (i, j) at (ro2n[i], co2n[j]); both maps must be
// permutations of their index range.
void check_map(int n, const int *o2n, const char *what) {
  if (o2n == nullptr) throw std::runtime_error(std::string(what) + ": input pointers must not be null.");
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; ++i) {
    const int j = o2n[i];
    if (j < 0 || j >= n || seen[j]) throw std::runtime_error(std::string(what) + ": map is not a permutation");
    seen[j] = 1;
  }
}

// Off-diagonal entries of a checked graph as sorted, unique (row, col) pairs.
std::vector<std::pair<int, int>> off_diagonal_pairs(int n, const int *rp, const int *ci) {
  std::vector<std::pair<int, int>> e;
  e.reserve(static_cast<size_t>(rp[n]));
  for (int r = 0; r < n; ++r)
    for (int k = rp[r]; k < rp[r + 1]; ++k)
      if (ci[k] != r) e.emplace_back(r, ci[k]);
  std::sort(e.begin(), e.end());
  e.erase(std::unique(e.begin(), e.end()), e.end());
  return e;
}

// Every off-diagonal entry (i, j) has its mirror (j, i).
bool structurally_symmetric(int n, const int *rp, const int *ci) {
  const std::vector<std::pair<int, int>> e = off_diagonal_pairs(n, rp, ci);
  for (const auto &p : e)
    if (!std::binary_search(e.begin(), e.end(), std::make_pair(p.second, p.first))) return false;
  return true;
}

// The pattern joined with its transpose (off-diagonal entries, columns sorted).
void symmetrised(int n, const int *rp, const int *ci, std::vector<int> &srp, std::vector<int> &sci) {
  std::vector<std::pair<int, int>> e = off_diagonal_pairs(n, rp, ci);
  const size_t m = e.size();
  for (size_t t = 0; t < m; ++t) e.emplace_back(e[t].second, e[t].first);
  std::sort(e.begin(), e.end());
  e.erase(std::unique(e.begin(), e.end()), e.end());
  srp.assign(static_cast<size_t>(n) + 1, 0);
  sci.resize(e.size());
  for (size_t t = 0; t < e.size(); ++t) {
    srp[e[t].first + 1]++;
    sci[t] = e[t].second;
  }
  for (int r = 0; r < n; ++r) srp[r + 1] += srp[r];
}

gsb::Csr make_csr(int rows, int cols, const int *rp, const int *ci, const double *v) {
  if (rows < 0 || cols < 0) throw std::runtime_error("CSR: negative dimensions");
  check_row_ptr(rows, rp, "CSR");
  if (rp[rows] > 0 && (ci == nullptr || v == nullptr))
    throw std::runtime_error("CSR: input pointers must not be null.");
  gsb::Csr a;
  a.rows = rows;
  a.cols = cols;
  a.rp.assign(rp, rp + rows + 1);
  a.ci.assign(ci, ci + rp[rows]);
  a.v.assign(v, v + rp[rows]);
  a.check("CSR");
  return a;
}

void copy_csr(const gsb::Csr &a, int *rp, int *ci, double *v) {
  std::memcpy(rp, a.rp.data(), sizeof(int) * (a.rows + 1));
  if (a.nnz() > 0) {
    std::memcpy(ci, a.ci.data(), sizeof(int) * a.nnz());
    std::memcpy(v, a.v.data(), sizeof(double) * a.nnz());
  }
}

int require_device(int device) {
  int count = 0;
  const cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail("no CUDA device is available (this library has no CPU fallback)", GS_ERR_NO_DEVICE);
  }
  if (device < 0 || device >= count) return fail("device index out of range");
  return GS_OK;
}

// The documented range of every option (include/gpusolver_b200.h), checked
// on the host before a device is touched. The solver and the batch re-check
// what depends on the hierarchy or on the path (the single-system solver
// takes lanes 1, 4, 8, 16 or 32; the batch also 2).
void check_options(const gs_solver_options &o) {
  const auto in = [](int v, int lo, int hi) { return v >= lo && v <= hi; };
  const auto bad = [](const char *what) { throw std::runtime_error(std::string("solver options: ") + what); };
  if (!in(o.smoother, 0, 4)) bad("smoother must be 0..4");
  if (!in(o.coarse_smoother, -1, 4)) bad("coarse_smoother must be -1..4");
  if (o.pre_steps < 1 || o.post_steps < 1 || o.vcycles < 1) bad("pre_steps, post_steps and vcycles must be >= 1");
  if (!in(o.coarse_solver, 0, 1)) bad("coarse_solver must be 0 or 1");
  if (o.coarse_solver == 0 && o.coarse_steps < 1) bad("coarse_steps must be >= 1 with coarse_solver 0");
  if (!(o.omega > 0.0 && o.omega < 2.0)) bad("omega must be in (0, 2)");
  if (!in(o.precision, 0, 1) || !in(o.flexible, 0, 1) || !in(o.use_graph, 0, 1) || !in(o.reference_vcycle, 0, 1) ||
      !in(o.autotune, 0, 1))
    bad("precision, flexible, use_graph, reference_vcycle and autotune must be 0 or 1");
  if (!in(o.coloring, 0, 2)) bad("coloring must be 0, 1 or 2");
  if (!(o.tol > 0.0 && std::isfinite(o.tol))) bad("tol must be a finite value > 0");
  if (o.max_iter < 1) bad("max_iter must be >= 1");
  if (!in(o.coarse_tail, 0, 2)) bad("coarse_tail must be 0, 1 or 2");
  if (!in(o.overlap_launch, 0, 2)) bad("overlap_launch must be 0, 1 or 2");
  if (o.lanes != 0 && o.lanes != 1 && o.lanes != 2 && o.lanes != 4 && o.lanes != 8 && o.lanes != 16 && o.lanes != 32)
    bad("lanes must be 0, 1, 2, 4, 8, 16 or 32");
  if (o.sliced_lanes != 0 && o.sliced_lanes != 1 && o.sliced_lanes != 2 && o.sliced_lanes != 4 && o.sliced_lanes != 8)
    bad("sliced_lanes must be 0, 1, 2, 4 or 8");
  if (o.coarse_rows < 0 || o.packed_rows < 0) bad("coarse_rows and packed_rows must be >= 0");
  if (!in(o.sweep_launch, 0, 2)) bad("sweep_launch must be 0, 1 or 2");
  if (!in(o.half_sweeps, 0, 1)) bad("half_sweeps must be 0 or 1");
  if (!in(o.coarse_half, 0, 1)) bad("coarse_half must be 0 or 1");
}

gsb::SolverOptions to_options(const gs_solver_options &opt) {
  gsb::SolverOptions o;
  o.smoother = opt.smoother;
  o.pre = opt.pre_steps;
  o.post = opt.post_steps;
  o.coarse_steps = opt.coarse_steps;
  o.vcycles = opt.vcycles;
  o.omega = opt.omega;
  o.coarse = opt.coarse_solver;
  o.mixed = opt.precision;
  o.flexible = opt.flexible;
  o.graph = opt.use_graph;
  o.check_every = opt.check_every;
  o.tol = opt.tol;
  o.max_iter = opt.max_iter;
  o.reference_vcycle = opt.reference_vcycle;
  o.autotune = opt.autotune;
  o.tune_cache = g_tune_cache;
  o.tail = opt.coarse_tail;
  o.lanes = opt.lanes;
  o.coarse_rows = opt.coarse_rows;
  o.sliced_lanes = opt.sliced_lanes;
  o.coarse_smoother = opt.coarse_smoother;
  o.overlap_launch = opt.overlap_launch;
  o.packed_rows = opt.packed_rows;
  o.coloring = opt.coloring;
  o.sweep_launch = opt.sweep_launch;
  o.half_sweeps = opt.half_sweeps;
  o.coarse_half = opt.coarse_half;
  return o;
}

}  // namespace

extern "C" {

const char *gs_last_error(void) { return g_error.c_str(); }
int gs_version(void) { return GS_VERSION; }

int gs_greedy_coloring(int n, const int *rp, const int *ci, int *colors, int *verts, int *offs,
                       int *ncolors) {
  return guarded([&] {
    if (n < 0 || rp == nullptr) return fail("gs_greedy_coloring: bad arguments");
    check_graph(n, rp, ci, "gs_greedy_coloring");
    check_outputs({colors, verts, offs, ncolors}, "gs_greedy_coloring");
    std::vector<int> c, v, o;
    const int nc = gsb::greedy_coloring(n, rp, ci, c, v, o);
    if (n > 0) {
      std::memcpy(colors, c.data(), sizeof(int) * n);
      std::memcpy(verts, v.data(), sizeof(int) * n);
    }
    std::memcpy(offs, o.data(), sizeof(int) * (nc + 1));
    *ncolors = nc;
    return GS_OK;
  });
}

int gs_smallest_last_coloring(int n, const int *rp, const int *ci, int *colors, int *verts, int *offs,
                              int *ncolors) {
  return guarded([&] {
    if (n < 0 || rp == nullptr) return fail("gs_smallest_last_coloring: bad arguments");
    check_graph(n, rp, ci, "gs_smallest_last_coloring");
    check_outputs({colors, verts, offs, ncolors}, "gs_smallest_last_coloring");
    // The ordering and first-fit look at the entries each row lists; a
    // pattern that is not structurally symmetric is coloured on its
    // symmetrised pattern, so that no entry joins two rows of one colour
    // (a symmetric pattern is coloured as given).
    std::vector<int> srp, sci;
    if (!structurally_symmetric(n, rp, ci)) {
      symmetrised(n, rp, ci, srp, sci);
      rp = srp.data();
      ci = sci.data();
    }
    std::vector<int> c, v, o;
    const int nc = gsb::smallest_last_coloring(n, rp, ci, c, v, o);
    if (n > 0) {
      std::memcpy(colors, c.data(), sizeof(int) * n);
      std::memcpy(verts, v.data(), sizeof(int) * n);
    }
    std::memcpy(offs, o.data(), sizeof(int) * (nc + 1));
    *ncolors = nc;
    return GS_OK;
  });
}

int gs_relaxed_coloring(int n, const int *rp, const int *ci, const double *v, double theta, double rho, int *colors,
                        int *verts, int *offs, int *ncolors) {
  return guarded([&] {
    if (n < 0 || rp == nullptr) return fail("gs_relaxed_coloring: bad arguments");
    check_graph(n, rp, ci, "gs_relaxed_coloring");
    check_outputs({colors, verts, offs, ncolors}, "gs_relaxed_coloring");
    if (v == nullptr && rp[n] > 0) return fail("gs_relaxed_coloring: null values");
    if (!(theta >= 0.0) || !std::isfinite(theta)) return fail("gs_relaxed_coloring: theta must be finite and >= 0");
    if (!(rho > 0.0 && rho < 1.0)) return fail("gs_relaxed_coloring: rho must be in (0, 1)");
    for (int k = 0; k < rp[n]; ++k)
      if (!std::isfinite(v[k])) return fail("gs_relaxed_coloring: values must be finite");
    if (!structurally_symmetric(n, rp, ci)) return fail("gs_relaxed_coloring: pattern must be structurally symmetric");
    std::vector<int> c, vv, o;
    const int nc = gsb::relaxed_coloring(n, rp, ci, v, theta, rho, c, vv, o);
    if (n > 0) {
      std::memcpy(colors, c.data(), sizeof(int) * n);
      std::memcpy(verts, vv.data(), sizeof(int) * n);
    }
    std::memcpy(offs, o.data(), sizeof(int) * (nc + 1));
    *ncolors = nc;
    return GS_OK;
  });
}

int gs_relaxed_block_coloring(int n, const int *rp, const int *ci, const double *v, double theta, double rho,
                              int *colors, int *verts, int *offs, int *ncolors) {
  return guarded([&] {
    if (n < 0 || rp == nullptr || n % 3 != 0) return fail("gs_relaxed_block_coloring: bad arguments");
    check_graph(n, rp, ci, "gs_relaxed_block_coloring");
    check_outputs({colors, verts, offs, ncolors}, "gs_relaxed_block_coloring");
    if (v == nullptr && rp[n] > 0) return fail("gs_relaxed_block_coloring: null values");
    if (!(theta >= 0.0) || !std::isfinite(theta)) return fail("gs_relaxed_block_coloring: theta must be finite and >= 0");
    if (!(rho > 0.0 && rho < 1.0)) return fail("gs_relaxed_block_coloring: rho must be in (0, 1)");
    for (int k = 0; k < rp[n]; ++k)
      if (!std::isfinite(v[k])) return fail("gs_relaxed_block_coloring: values must be finite");
    if (!structurally_symmetric(n, rp, ci))
      return fail("gs_relaxed_block_coloring: pattern must be structurally symmetric");
    gsb::Csr a;
    a.rows = a.cols = n;
    a.rp.assign(rp, rp + n + 1);
    a.ci.assign(ci, ci + rp[n]);
    a.v.assign(v, v + rp[n]);
    std::vector<int> c, vv, o;
    const int nc = gsb::relaxed_block_coloring(a, theta, rho, c, vv, o);
    if (n > 0) {
      std::memcpy(colors, c.data(), sizeof(int) * (n / 3));
      std::memcpy(verts, vv.data(), sizeof(int) * (n / 3));
    }
    std::memcpy(offs, o.data(), sizeof(int) * (nc + 1));
    *ncolors = nc;
    return GS_OK;
  });
}

int gs_rcm(int n, const int *rp, const int *ci, int *o2n, int *n2o) {
  return guarded([&] {
    if (n <= 0 || rp == nullptr) return fail("gs_rcm: bad arguments");
    check_graph(n, rp, ci, "gs_rcm");
    check_outputs({o2n, n2o}, "gs_rcm");
    gsb::rcm(n, rp, ci, o2n, n2o);
    return GS_OK;
  });
}

int gs_apply_permutation(int n, const int *rp, const int *ci, const double *v, const int *o2n,
                         const int *n2o, int *orp, int *oci, double *ov) {
  return guarded([&] {
    const gsb::Csr a = make_csr(n, n, rp, ci, v);
    check_outputs({orp, oci, ov}, "gs_apply_permutation");
    copy_csr(gsb::apply_permutation(a, o2n, n2o), orp, oci, ov);
    return GS_OK;
  });
}

int gs_permute_matrix(int rows, int cols, const int *rp, const int *ci, const double *v,
                      const int *ro2n, const int *co2n, int *orp, int *oci, double *ov) {
  return guarded([&] {
    const gsb::Csr a = make_csr(rows, cols, rp, ci, v);
    check_map(rows, ro2n, "permuteMatrix (rows)");
    check_map(cols, co2n, "permuteMatrix (columns)");
    check_outputs({orp, oci, ov}, "gs_permute_matrix");
    copy_csr(gsb::permute_matrix(a, ro2n, co2n), orp, oci, ov);
    return GS_OK;
  });
}

int gs_ell_build(int n, int cols, const int *rp, const int *ci, const double *v, int width,
                 int *ell_col, double *ell_val, int *ovf_rp, int *ovf_ci, double *ovf_v,
                 int *ovf_nnz) {
  return guarded([&] {
    const gsb::Csr a = make_csr(n, cols, rp, ci, v);
    check_outputs({ell_col, ell_val, ovf_rp, ovf_nnz}, "gs_ell_build");
    const gsb::HostEll e = gsb::build_ell(a, width);
    if (!e.ovf_ci.empty()) check_outputs({ovf_ci, ovf_v}, "gs_ell_build");
    std::memcpy(ell_col, e.col.data(), sizeof(int) * e.col.size());
    std::memcpy(ell_val, e.val.data(), sizeof(double) * e.val.size());
    std::memcpy(ovf_rp, e.ovf_rp.data(), sizeof(int) * e.ovf_rp.size());
    *ovf_nnz = static_cast<int>(e.ovf_ci.size());
    if (!e.ovf_ci.empty()) {
      std::memcpy(ovf_ci, e.ovf_ci.data(), sizeof(int) * e.ovf_ci.size());
      std::memcpy(ovf_v, e.ovf_v.data(), sizeof(double) * e.ovf_v.size());
    }
    return GS_OK;
  });
}

int gs_block_graph(int n, const int *rp, const int *ci, int block, int *grp, int *gci, int *gnnz) {
  return guarded([&] {
    if (block <= 0) return fail("buildBlockGraph: block size must be positive.");
    check_graph(n, rp, ci, "buildBlockGraph");
    check_outputs({grp, gnnz}, "gs_block_graph");
    if (rp[n] > 0) check_outputs({gci}, "gs_block_graph");
    gsb::Csr a;
    a.rows = a.cols = n;
    a.rp.assign(rp, rp + n + 1);
    a.ci.assign(ci, ci + rp[n]);
    a.v.assign(rp[n], 0.0);
    std::vector<int> g_rp, g_ci;
    gsb::block_graph(a, block, g_rp, g_ci);
    // g_col holds nnz entries: enough for any structurally symmetric pattern
    // (every node edge comes from an entry off the diagonal blocks); the
    // symmetrised graph of an unsymmetric pattern can need more
    if (g_ci.size() > static_cast<size_t>(rp[n]))
      return fail("buildBlockGraph: the node graph has more entries than the matrix (unsymmetric pattern)");
    std::memcpy(grp, g_rp.data(), sizeof(int) * g_rp.size());
    if (!g_ci.empty()) std::memcpy(gci, g_ci.data(), sizeof(int) * g_ci.size());
    *gnnz = static_cast<int>(g_ci.size());
    return GS_OK;
  });
}

int gs_block_inverses3x3(int n, const int *rp, const int *ci, const double *v, double *dinv) {
  return guarded([&] {
    const gsb::Csr a = make_csr(n, n, rp, ci, v);
    check_outputs({dinv}, "gs_block_inverses3x3");
    std::vector<double> d;
    if (gsb::block_inverses3x3(a, d) >= 0) return fail("Block diagonal is not SPD.");
    if (!d.empty()) std::memcpy(dinv, d.data(), sizeof(double) * d.size());
    return GS_OK;
  });
}

int gs_expand_block_permutation(int nodes, int block, const int *no2n, const int *nn2o, int *o2n,
                                int *n2o) {
  return guarded([&] {
    if (block <= 0) return fail("expandBlockPermutation: block size must be positive.");
    gsb::check_permutation(nodes, no2n, nn2o);
    check_outputs({o2n, n2o}, "gs_expand_block_permutation");
    gsb::expand_block_permutation(nodes, block, no2n, nn2o, o2n, n2o);
    return GS_OK;
  });
}

// ---- host CSR / problems ----------------------------------------------------
int gs_problem_create(int kind, const int *ip, const double *dp, unsigned long long seed,
                      gs_host_csr **out) {
  return guarded([&] {
    if (ip == nullptr || out == nullptr || (kind != GS_PROBLEM_POISSON7 && dp == nullptr))
      return fail("gs_problem_create: null argument");
    // Sizes are checked so that rows and entries stay within int: at most
    // 7 entries per row for the 7-point stencils, 15 for the P1 Laplacian and
    // 15 blocks of 9 per node for elasticity.
    const bool grid = kind == GS_PROBLEM_POISSON7 || kind == GS_PROBLEM_VARCOEF_GRF ||
                      kind == GS_PROBLEM_VARCOEF_LOGUNI;
    long long entries = 0;
    if (grid) {
      if (ip[0] <= 0 || ip[1] <= 0 || ip[2] <= 0) return fail("gs_problem_create: grid sides must be positive");
      entries = 7LL * ip[0] * ip[1] * ip[2];
    } else if (kind == GS_PROBLEM_KUHN_P1) {
      if (ip[0] < 2) return fail("gs_problem_create: need at least 2 cells per side");
      entries = 15LL * (ip[0] - 1) * (ip[0] - 1) * (ip[0] - 1);
    } else if (kind == GS_PROBLEM_ELASTICITY_P1) {
      if (ip[0] < 2) return fail("gs_problem_create: need at least 2 vertices per side");
      entries = 135LL * ip[0] * ip[0] * ip[0];
    }
    if (entries > 2147483647LL) return fail("gs_problem_create: problem too large for 32-bit indices");
    if (kind == GS_PROBLEM_VARCOEF_GRF && !(dp[0] > 0.0)) return fail("gs_problem_create: correlation length must be positive");
    if (kind == GS_PROBLEM_VARCOEF_LOGUNI && !(dp[0] > 0.0 && dp[1] >= dp[0]))
      return fail("gs_problem_create: need 0 < lo <= hi");
    if (kind == GS_PROBLEM_KUHN_P1 && !(dp[0] >= 0.0)) return fail("gs_problem_create: jitter must be >= 0");
    if (kind == GS_PROBLEM_ELASTICITY_P1 && !(dp[0] > -1.0 && dp[0] < 0.5))
      return fail("gs_problem_create: Poisson ratio must lie in (-1, 0.5)");
    std::unique_ptr<gs_host_csr> m(new gs_host_csr);
    switch (kind) {
      case GS_PROBLEM_POISSON7:
        m->a = gsb::poisson7(ip[0], ip[1], ip[2]);
        break;
      case GS_PROBLEM_VARCOEF_GRF:
        m->a = gsb::varcoef7(ip[0], ip[1], ip[2],
                             gsb::grf_coefficients(ip[0], ip[1], ip[2], dp[0], dp[1], seed));
        break;
      case GS_PROBLEM_VARCOEF_LOGUNI:
        m->a = gsb::varcoef7(ip[0], ip[1], ip[2],
                             gsb::loguniform_coefficients(ip[0] * ip[1] * ip[2], dp[0], dp[1], seed));
        break;
      case GS_PROBLEM_KUHN_P1:
        m->a = gsb::kuhn_laplacian(ip[0], dp[0], seed);
        break;
      case GS_PROBLEM_ELASTICITY_P1:
        m->a = gsb::elasticity_p1(ip[0], dp[0], seed, m->rhs);
        break;
      default:
        return fail("gs_problem_create: unknown problem kind");
    }
    *out = m.release();
    return GS_OK;
  });
}

int gs_host_csr_create(int rows, int cols, const int *rp, const int *ci, const double *v,
                       gs_host_csr **out) {
  return guarded([&] {
    std::unique_ptr<gs_host_csr> m(new gs_host_csr);
    if (out == nullptr) return fail("gs_host_csr_create: null argument");
    m->a = make_csr(rows, cols, rp, ci, v);
    *out = m.release();
    return GS_OK;
  });
}

int gs_host_csr_info(const gs_host_csr *m, int *rows, int *cols, int *nnz, int *has_rhs) {
  if (m == nullptr) return fail("null matrix");
  if (rows) *rows = m->a.rows;
  if (cols) *cols = m->a.cols;
  if (nnz) *nnz = m->a.nnz();
  if (has_rhs) *has_rhs = m->rhs.empty() ? 0 : 1;
  return GS_OK;
}

int gs_host_csr_copy(const gs_host_csr *m, int *rp, int *ci, double *v) {
  if (m == nullptr) return fail("null matrix");
  if (rp == nullptr || (m->a.nnz() > 0 && (ci == nullptr || v == nullptr))) return fail("null output array");
  copy_csr(m->a, rp, ci, v);
  return GS_OK;
}

int gs_host_csr_rhs(const gs_host_csr *m, double *rhs) {
  if (m == nullptr || m->rhs.empty()) return fail("matrix has no right-hand side");
  if (rhs == nullptr) return fail("null output array");
  std::memcpy(rhs, m->rhs.data(), sizeof(double) * m->rhs.size());
  return GS_OK;
}

void gs_host_csr_destroy(gs_host_csr *m) { delete m; }

int gs_uniform_rhs(int n, unsigned long long seed, double *out) {
  return guarded([&] {
    if (n < 0 || (n > 0 && out == nullptr)) return fail("gs_uniform_rhs: bad arguments");
    const std::vector<double> b = gsb::uniform_rhs(n, seed);
    if (n > 0) std::memcpy(out, b.data(), sizeof(double) * n);
    return GS_OK;
  });
}

// ---- hierarchy --------------------------------------------------------------
int gs_hierarchy_build(const gs_host_csr *a, int block, double eps, int max_levels, int min_dofs,
                       gs_hierarchy **out) {
  return guarded([&] {
    if (a == nullptr || out == nullptr) return fail("null argument");
    gsb::SaOptions o;
    o.block = block;
    o.eps_strong = eps;
    o.max_levels = max_levels;
    o.min_dofs = min_dofs;
    std::unique_ptr<gs_hierarchy> h(new gs_hierarchy);
    h->h = gsb::build_hierarchy(a->a, o);
    *out = h.release();
    return GS_OK;
  });
}

int gs_hierarchy_build_ex(const gs_host_csr *a, int block, double eps, int max_levels, int min_dofs,
                          int aggregation, int device, gs_setup_stats *stats, gs_hierarchy **out) {
  return guarded([&] {
    if (a == nullptr || out == nullptr) return fail("null argument");
    if (aggregation != 0 && aggregation != 1) return fail("aggregation must be 0 or 1");
    if (device >= 0 && aggregation != 1) return fail("the GPU build uses aggregation 1");
    gsb::SaOptions o;
    o.block = block;
    o.eps_strong = eps;
    o.max_levels = max_levels;
    o.min_dofs = min_dofs;
    o.aggregation = aggregation;
    std::unique_ptr<gs_hierarchy> h(new gs_hierarchy);
    gsb::DeviceSetupStats st;
    if (device >= 0) {
      h->h = gsb::build_hierarchy_device(a->a, o, device, &st);
    } else {
      const auto t0 = std::chrono::steady_clock::now();
      h->h = gsb::build_hierarchy(a->a, o);
      st.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    if (stats != nullptr) {
      stats->total_ms = st.total_ms;
      stats->upload_ms = st.upload_ms;
      stats->build_ms = st.build_ms;
      stats->download_ms = st.download_ms;
      stats->mis_rounds = st.mis_rounds;
    }
    *out = h.release();
    return GS_OK;
  });
}

int gs_hierarchy_refresh(const gs_hierarchy *h, const double *values, int device, gs_hierarchy **out) {
  return guarded([&] {
    if (h == nullptr || values == nullptr || out == nullptr) return fail("gs_hierarchy_refresh: null argument");
    if (h->h.A.empty()) return fail("MultigridSmoother: empty hierarchy.");
    const int L = static_cast<int>(h->h.A.size());
    gsb::Csr a0 = h->h.A[0];
    if (!a0.v.empty()) std::memcpy(a0.v.data(), values, sizeof(double) * a0.v.size());
    std::unique_ptr<gs_hierarchy> r(new gs_hierarchy);
    r->h.block = h->h.block;
    r->h.P = h->h.P;
    r->h.R = h->h.R;
    r->h.agg = h->h.agg;
    if (device >= 0) {
      const int rc = require_device(device);
      if (rc != GS_OK) return rc;
      r->h.A = gsb::galerkin_device(a0, h->h.P, h->h.R, L, device);
    } else {
      r->h.A.push_back(a0);
      for (int k = 0; k + 1 < L; ++k) r->h.A.push_back(gsb::spgemm(h->h.R[k], gsb::spgemm(r->h.A[k], h->h.P[k])));
    }
    *out = r.release();
    return GS_OK;
  });
}

int gs_hierarchy_from_levels(int L, const gs_csr *A, const gs_csr *P, const gs_csr *R, int block,
                             gs_hierarchy **out) {
  return guarded([&] {
    if (L <= 0) return fail("MultigridSmoother: empty hierarchy.");
    if (A == nullptr || out == nullptr || (L > 1 && (P == nullptr || R == nullptr)))
      return fail("gs_hierarchy_from_levels: null argument");
    std::unique_ptr<gs_hierarchy> h(new gs_hierarchy);
    h->h.block = block;
    for (int k = 0; k < L; ++k) {
      h->h.A.push_back(make_csr(A[k].rows, A[k].cols, A[k].row_ptr, A[k].col_idx, A[k].val));
      if (k + 1 < L) {
        h->h.P.push_back(make_csr(P[k].rows, P[k].cols, P[k].row_ptr, P[k].col_idx, P[k].val));
        h->h.R.push_back(make_csr(R[k].rows, R[k].cols, R[k].row_ptr, R[k].col_idx, R[k].val));
      }
    }
    *out = h.release();
    return GS_OK;
  });
}

int gs_hierarchy_num_levels(const gs_hierarchy *h) {
  return h == nullptr ? 0 : static_cast<int>(h->h.A.size());
}

static const gsb::Csr *pick(const gs_hierarchy *h, int level, int which) {
  if (h == nullptr || level < 0) return nullptr;
  const auto &v = which == 0 ? h->h.A : (which == 1 ? h->h.P : h->h.R);
  if (level >= static_cast<int>(v.size())) return nullptr;
  return &v[level];
}

int gs_hierarchy_matrix_info(const gs_hierarchy *h, int level, int which, int *rows, int *cols,
                             int *nnz) {
  const gsb::Csr *m = pick(h, level, which);
  if (m == nullptr) return fail("gs_hierarchy_matrix_info: no such matrix");
  if (rows == nullptr || cols == nullptr || nnz == nullptr) return fail("gs_hierarchy_matrix_info: null output");
  *rows = m->rows;
  *cols = m->cols;
  *nnz = m->nnz();
  return GS_OK;
}

int gs_hierarchy_matrix(const gs_hierarchy *h, int level, int which, int *rp, int *ci, double *v) {
  const gsb::Csr *m = pick(h, level, which);
  if (m == nullptr) return fail("gs_hierarchy_matrix: no such matrix");
  if (rp == nullptr || (m->nnz() > 0 && (ci == nullptr || v == nullptr))) return fail("gs_hierarchy_matrix: null output");
  copy_csr(*m, rp, ci, v);
  return GS_OK;
}

int gs_hierarchy_aggregates(const gs_hierarchy *h, int level, int *agg) {
  if (h == nullptr || level < 0 || level >= static_cast<int>(h->h.agg.size()))
    return fail("gs_hierarchy_aggregates: no such level");
  if (agg == nullptr) return fail("gs_hierarchy_aggregates: null output");
  const auto &a = h->h.agg[level];
  for (size_t i = 0; i < a.size(); ++i) agg[i] = a[i] < 0 ? -1 : a[i];
  return GS_OK;
}

int gs_hierarchical_reordering(const gs_hierarchy *h, int *const *old_to_new, int *const *new_to_old) {
  return guarded([&] {
    if (h == nullptr || old_to_new == nullptr || new_to_old == nullptr)
      return fail("gs_hierarchical_reordering: null argument");
    std::vector<std::vector<int>> o2n, n2o;
    gsb::hierarchical_reordering(h->h, o2n, n2o);
    for (size_t k = 0; k < o2n.size(); ++k) {
      if (old_to_new[k] == nullptr || new_to_old[k] == nullptr) return fail("gs_hierarchical_reordering: null level array");
      std::memcpy(old_to_new[k], o2n[k].data(), sizeof(int) * o2n[k].size());
      std::memcpy(new_to_old[k], n2o[k].data(), sizeof(int) * n2o[k].size());
    }
    return GS_OK;
  });
}

void gs_hierarchy_destroy(gs_hierarchy *h) { delete h; }

// ---- solver -----------------------------------------------------------------
void gs_solver_options_default(gs_solver_options *o) {
  const gsb::SolverOptions d;
  o->smoother = d.smoother;
  o->pre_steps = d.pre;
  o->post_steps = d.post;
  o->coarse_steps = d.coarse_steps;
  o->vcycles = d.vcycles;
  o->omega = d.omega;
  o->coarse_solver = d.coarse;
  o->precision = d.mixed;
  o->flexible = d.flexible;
  o->use_graph = d.graph;
  o->check_every = d.check_every;
  o->tol = d.tol;
  o->max_iter = d.max_iter;
  o->reference_vcycle = d.reference_vcycle;
  o->autotune = d.autotune;
  o->coarse_tail = d.tail;
  o->lanes = d.lanes;
  o->coarse_rows = d.coarse_rows;
  o->sliced_lanes = d.sliced_lanes;
  o->coarse_smoother = d.coarse_smoother;
  o->overlap_launch = d.overlap_launch;
  o->packed_rows = d.packed_rows;
  o->coloring = d.coloring;
  o->sweep_launch = d.sweep_launch;
  o->half_sweeps = d.half_sweeps;
  o->coarse_half = d.coarse_half;
}

int gs_set_tune_cache(const char *path) {
  g_tune_cache = path == nullptr ? "" : path;
  return GS_OK;
}

int gs_solver_create(const gs_hierarchy *h, const int *const *o2n, const int *const *n2o,
                     const gs_solver_options *opt, int device, gs_solver **out) {
  return guarded([&] {
    if (h == nullptr || opt == nullptr || out == nullptr || (o2n != nullptr && n2o == nullptr))
      return fail("gs_solver_create: null argument");
    check_options(*opt);
    const int rc = require_device(device);
    if (rc != GS_OK) return rc;
    gsb::SolverOptions o = to_options(*opt);
    const int L = static_cast<int>(h->h.A.size());
    std::vector<const int *> po(L, nullptr), pn(L, nullptr);
    if (o2n != nullptr)
      for (int k = 0; k < L; ++k) po[k] = o2n[k], pn[k] = n2o[k];
    std::unique_ptr<gs_solver> s(new gs_solver);
    s->s = gsb::Solver::create(h->h, po, pn, o, device);
    *out = s.release();
    return GS_OK;
  });
}

int gs_solver_solve(gs_solver *s, const double *b, double *x, gs_solve_stats *stats) {
  return guarded([&] {
    if (s == nullptr || b == nullptr || x == nullptr) return fail("gs_solver_solve: null argument");
    gsb::SolveStats st;
    s->s->solve_host(b, x, &st);
    if (stats) *stats = gs_solve_stats{st.iterations, st.status, st.spmv, st.ratio, st.bb, st.solve_ms};
    return GS_OK;
  });
}

int gs_solver_solve_f32(gs_solver *s, const float *b, float *x, gs_solve_stats *stats) {
  return guarded([&] {
    if (s == nullptr || b == nullptr || x == nullptr) return fail("gs_solver_solve_f32: null argument");
    const int n = s->s->rows();
    s->hb.assign(b, b + n);
    s->hx.assign(x, x + n);
    gsb::SolveStats st;
    s->s->solve_host(s->hb.data(), s->hx.data(), &st);
    for (int i = 0; i < n; ++i) x[i] = static_cast<float>(s->hx[i]);
    if (stats) *stats = gs_solve_stats{st.iterations, st.status, st.spmv, st.ratio, st.bb, st.solve_ms};
    return GS_OK;
  });
}

int gs_solver_solve_device(gs_solver *s, const double *b, double *x, void *stream,
                           gs_solve_stats *stats) {
  return guarded([&] {
    if (s == nullptr || b == nullptr || x == nullptr) return fail("gs_solver_solve_device: null argument");
    gsb::SolveStats st;
    s->s->solve_device(b, x, static_cast<cudaStream_t>(stream), &st);
    if (stats) *stats = gs_solve_stats{st.iterations, st.status, st.spmv, st.ratio, st.bb, st.solve_ms};
    return GS_OK;
  });
}

int gs_solver_apply_preconditioner(gs_solver *s, const double *r, double *z, void *stream) {
  return guarded([&] {
    if (s == nullptr || r == nullptr || z == nullptr) return fail("gs_solver_apply_preconditioner: null argument");
    s->s->apply_preconditioner(r, z, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_solver_set_tolerance(gs_solver *s, double tol, int max_iter) {
  if (s == nullptr) return fail("null solver");
  if (!(tol > 0.0) || max_iter < 1) return fail("gs_solver_set_tolerance: tol must be > 0 and max_iter >= 1");
  s->s->set_tolerance(tol, max_iter);
  return GS_OK;
}

int gs_solver_set_colour_weights(gs_solver *s, const double *w, const int *offs, int L) {
  return guarded([&] {
    if (s == nullptr) return fail("null solver");
    gsb::ColourWeights cw;
    if (w != nullptr) {
      // offs[k] is where level k's weights start in w: 0 first, never decreasing
      if (offs == nullptr || L < 0) return fail("colour weights: level offsets missing");
      if (offs[0] != 0) return fail("colour weights: level offsets must start at 0");
      for (int k = 0; k < L; ++k)
        if (offs[k + 1] < offs[k]) return fail("colour weights: level offsets decrease");
      cw.level_offset.assign(offs, offs + L + 1);
      cw.w.assign(w, w + offs[L]);
    }
    s->s->set_weights(cw);
    return GS_OK;
  });
}

int gs_solver_num_levels(const gs_solver *s) {
  return s == nullptr ? 0 : static_cast<int>(s->s->level_info().size());
}

int gs_solver_level_info(const gs_solver *s, int level, int *rows, int *nnz, int *colors,
                         int *slices, long long *stored) {
  if (s == nullptr) return fail("null solver");
  const auto info = s->s->level_info();
  if (level < 0 || level >= static_cast<int>(info.size())) return fail("no such level");
  if (rows) *rows = info[level].rows;
  if (nnz) *nnz = info[level].nnz;
  if (colors) *colors = info[level].colors;
  if (slices) *slices = info[level].slices;
  if (stored) *stored = info[level].stored;
  return GS_OK;
}

int gs_solver_level_format(const gs_solver *s, int level, int *lanes, int *p_lanes, int *r_lanes) {
  if (s == nullptr) return fail("null solver");
  const auto info = s->s->level_info();
  if (level < 0 || level >= static_cast<int>(info.size())) return fail("no such level");
  if (lanes) *lanes = info[level].lanes;
  if (p_lanes) *p_lanes = info[level].p_lanes;
  if (r_lanes) *r_lanes = info[level].r_lanes;
  return GS_OK;
}

int gs_solver_level_layout(const gs_solver *s, int level) {
  if (s == nullptr) return -1;
  const auto info = s->s->level_info();
  if (level < 0 || level >= static_cast<int>(info.size())) return -1;
  return info[level].sliced;
}

int gs_solver_level_launch(const gs_solver *s, int level) {
  if (s == nullptr) return -1;
  const auto info = s->s->level_info();
  if (level < 0 || level >= static_cast<int>(info.size())) return -1;
  return info[level].launch;
}

int gs_solver_level_in_tail(const gs_solver *s, int level) {
  if (s == nullptr) return 0;
  const auto info = s->s->level_info();
  if (level < 0 || level >= static_cast<int>(info.size())) return 0;
  return info[level].in_tail ? info[level].tail_ctas : 0;
}

int gs_solver_setup_phases(const gs_solver *s, double *ms, int count) {
  return guarded([&] {
    if (s == nullptr || (ms == nullptr && count > 0) || count < 0)
      return fail("gs_solver_setup_phases: bad arguments");
    const std::vector<double> t = s->s->setup_times();
    for (int i = 0; i < count; ++i) ms[i] = i < static_cast<int>(t.size()) ? t[i] : 0.0;
    return GS_OK;
  });
}

int gs_solver_setup_times(const gs_solver *s, double *ms4) {
  return guarded([&] {
    if (s == nullptr || ms4 == nullptr) return fail("gs_solver_setup_times: null argument");
    const std::vector<double> t = s->s->setup_times();
    for (int i = 0; i < 4; ++i) ms4[i] = t[i];
    return GS_OK;
  });
}

int gs_solver_time_level(gs_solver *s, int level, int op, int lanes, int reps, void *stream, double *ms) {
  return guarded([&] {
    if (s == nullptr || ms == nullptr) return fail("gs_solver_time_level: null argument");
    *ms = s->s->time_level(level, op, lanes, reps, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_solver_time_kernel(gs_solver *s, int kind, int reps, void *stream, double *ms) {
  return guarded([&] {
    if (s == nullptr || ms == nullptr) return fail("null argument");
    *ms = s->s->time_kernel(kind, reps, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_solver_launch_count(const gs_solver *s, long long *count) {
  if (s == nullptr || count == nullptr) return fail("null argument");
  *count = s->s->launches();
  return GS_OK;
}

void gs_solver_destroy(gs_solver *s) { delete s; }

int gs_solver_update_matrix(gs_solver *s, const double *values) {
  return guarded([&] {
    if (s == nullptr || values == nullptr) return fail("gs_solver_update_matrix: null argument");
    s->s->update_values(values);
    return GS_OK;
  });
}

int gs_dense_spd_inverse(int n, const int *rp, const int *ci, const double *v, double *inverse, int device) {
  return guarded([&] {
    if (inverse == nullptr || n < 0) return fail("gs_dense_spd_inverse: bad arguments");
    const gsb::Csr a = make_csr(n, n, rp, ci, v);
    const int rc = require_device(device);
    if (rc != GS_OK) return rc;
    gsb::cuda_check(cudaSetDevice(device), "cudaSetDevice");
    double *d = nullptr;
    gsb::cuda_check(cudaMalloc(&d, sizeof(double) * static_cast<size_t>(n) * n + 8), "cudaMalloc");
    try {
      gsb::spd_inverse_device(a, d, nullptr);
      gsb::cuda_check(cudaMemcpy(inverse, d, sizeof(double) * static_cast<size_t>(n) * n, cudaMemcpyDeviceToHost),
                      "cudaMemcpy");
    } catch (...) {
      cudaFree(d);
      throw;
    }
    cudaFree(d);
    return GS_OK;
  });
}

// ---- batched solves of many systems ----------------------------------------------
namespace {
gs_solve_stats to_c(const gsb::SolveStats &st) {
  return gs_solve_stats{st.iterations, st.status, st.spmv, st.ratio, st.bb, st.solve_ms};
}
std::vector<const gsb::Hierarchy *> hierarchies(int n, const gs_hierarchy *const *h) {
  if (n < 1 || h == nullptr) throw std::runtime_error("batched solver: no systems");
  std::vector<const gsb::Hierarchy *> v(n);
  for (int i = 0; i < n; ++i) {
    if (h[i] == nullptr) throw std::runtime_error("batched solver: null hierarchy");
    v[i] = &h[i]->h;
  }
  return v;
}
}  // namespace

int gs_batch_create(int num_systems, const gs_hierarchy *const *h, int nrhs, const gs_solver_options *opt,
                    int device, gs_batch **out) {
  return guarded([&] {
    if (opt == nullptr || out == nullptr) return fail("gs_batch_create: null argument");
    if (num_systems > 65535) return fail("gs_batch_create: at most 65535 systems");
    const std::vector<const gsb::Hierarchy *> v = hierarchies(num_systems, h);
    check_options(*opt);
    if (opt->half_sweeps != 0) return fail("gs_batch_create: half_sweeps is not supported by the batched solver");
    if (opt->coloring == 2) return fail("gs_batch_create: coloring 2 is not supported by the batched solver");
    const int rc = require_device(device);
    if (rc != GS_OK) return rc;
    std::unique_ptr<gs_batch> b(new gs_batch);
    b->b = gsb::make_batch_solver(v, nrhs, to_options(*opt), device);
    *out = b.release();
    return GS_OK;
  });
}

int gs_batch_solve(gs_batch *b, const double *rhs, double *x, gs_solve_stats *stats) {
  return guarded([&] {
    if (b == nullptr || rhs == nullptr || x == nullptr) return fail("gs_batch_solve: null argument");
    std::vector<gsb::SolveStats> st;
    b->b->solve_host(rhs, x, st);
    if (stats)
      for (size_t i = 0; i < st.size(); ++i) stats[i] = to_c(st[i]);
    return GS_OK;
  });
}

int gs_batch_solve_device(gs_batch *b, const double *rhs, double *x, void *stream, gs_solve_stats *stats) {
  return guarded([&] {
    if (b == nullptr || rhs == nullptr || x == nullptr) return fail("gs_batch_solve_device: null argument");
    std::vector<gsb::SolveStats> st;
    b->b->solve_device(rhs, x, static_cast<cudaStream_t>(stream), st);
    if (stats)
      for (size_t i = 0; i < st.size(); ++i) stats[i] = to_c(st[i]);
    return GS_OK;
  });
}

int gs_batch_set_tolerance(gs_batch *b, double tol, int max_iter) {
  return guarded([&] {
    if (b == nullptr) return fail("gs_batch_set_tolerance: null argument");
    b->b->set_tolerance(tol, max_iter);
    return GS_OK;
  });
}

int gs_batch_info(const gs_batch *b, int *num_systems, int *nrhs, long long *unknowns, int *levels) {
  if (b == nullptr) return fail("gs_batch_info: null argument");
  if (num_systems) *num_systems = b->b->num_systems();
  if (nrhs) *nrhs = b->b->nrhs();
  if (unknowns) {
    long long u = 0;
    for (int n : b->b->system_rows()) u += n;
    *unknowns = u;
  }
  if (levels) *levels = static_cast<int>(b->b->level_info().size());
  return GS_OK;
}

int gs_batch_system_rows(const gs_batch *b, int *rows) {
  if (b == nullptr || rows == nullptr) return fail("gs_batch_system_rows: null argument");
  const std::vector<int> &r = b->b->system_rows();
  std::memcpy(rows, r.data(), sizeof(int) * r.size());
  return GS_OK;
}

int gs_batch_level_info(const gs_batch *b, int level, int *rows, long long *nnz, int *systems, int *max_colors,
                        int *lanes, int *p_lanes, int *r_lanes) {
  if (b == nullptr) return fail("gs_batch_level_info: null argument");
  const auto &li = b->b->level_info();
  if (level < 0 || level >= static_cast<int>(li.size())) return fail("gs_batch_level_info: level out of range");
  const gsb::BatchLevelInfo &l = li[level];
  if (rows) *rows = l.rows;
  if (nnz) *nnz = l.nnz;
  if (systems) *systems = l.systems;
  if (max_colors) *max_colors = l.max_colors;
  if (lanes) *lanes = l.lanes;
  if (p_lanes) *p_lanes = l.p_lanes;
  if (r_lanes) *r_lanes = l.r_lanes;
  return GS_OK;
}

int gs_batch_launch_count(const gs_batch *b, long long *count) {
  if (b == nullptr || count == nullptr) return fail("null argument");
  *count = b->b->launches();
  return GS_OK;
}

int gs_batch_time_kernel(gs_batch *b, int kind, int reps, void *stream, double *ms) {
  return guarded([&] {
    if (b == nullptr || ms == nullptr) return fail("gs_batch_time_kernel: null argument");
    *ms = b->b->time_kernel(kind, reps, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_batch_time_level(gs_batch *b, int level, int op, int lanes, int reps, void *stream, double *ms) {
  return guarded([&] {
    if (b == nullptr || ms == nullptr) return fail("gs_batch_time_level: null argument");
    *ms = b->b->time_level(level, op, lanes, reps, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

void gs_batch_destroy(gs_batch *b) { delete b; }

int gs_batch_plan_check(int num_systems, const gs_hierarchy *const *h, int *levels, int *passes,
                        long long *items) {
  return guarded([&] {
    const gsb::BatchPlanStats st = gsb::check_batch_plan(hierarchies(num_systems, h));
    if (levels) *levels = st.levels;
    if (passes) *passes = st.passes;
    if (items) *items = st.items;
    return GS_OK;
  });
}

// ---- learned relaxation weights -------------------------------------------------
int gs_mlp_param_count(void) { return gsb::kMlpParams; }

int gs_mlp_forward(const float *params, const float *feats, int n, float *omega, float *cache,
                   void *stream) {
  return guarded([&] {
    if (params == nullptr || feats == nullptr || omega == nullptr || n < 0) return fail("gs_mlp_forward: bad arguments");
    gsb::mlp_forward(params, feats, n, omega, cache, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_mlp_backward(const float *params, const float *feats, int n, const float *cache,
                    const float *upstream, float *delta, float *grad, void *stream) {
  return guarded([&] {
    if (params == nullptr || feats == nullptr || cache == nullptr || upstream == nullptr ||
        delta == nullptr || grad == nullptr || n < 0)
      return fail("gs_mlp_backward: bad arguments");
    gsb::mlp_backward(params, feats, n, cache, upstream, delta, grad, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_mlp_adam(float *params, const float *grad, float *m, float *v, int np, double lr, double b1,
                double b2, double eps, int step, void *stream) {
  return guarded([&] {
    if (params == nullptr || grad == nullptr || m == nullptr || v == nullptr) return fail("gs_mlp_adam: null argument");
    if (np < 1) return fail("gs_mlp_adam: np must be >= 1");
    gsb::mlp_adam(params, grad, m, v, np, static_cast<float>(lr), static_cast<float>(b1),
                  static_cast<float>(b2), static_cast<float>(eps), step, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_solver_colour_features(const gs_solver *s, float *out, int capacity, int *count) {
  if (s == nullptr || count == nullptr) return fail("null argument");
  const std::vector<float> f = s->s->colour_features();
  const int n = static_cast<int>(f.size() / 8);
  *count = n;
  if (out != nullptr) {
    if (capacity < static_cast<int>(f.size())) return fail("gs_solver_colour_features: capacity too small");
    std::memcpy(out, f.data(), sizeof(float) * f.size());
  }
  return GS_OK;
}

int gs_solver_node_features(const gs_solver *s, float *out, long long capacity, long long *count) {
  return guarded([&] {
    if (s == nullptr || count == nullptr) return fail("null argument");
    const std::vector<float> f = s->s->node_features();
    *count = static_cast<long long>(f.size() / 8);
    if (out != nullptr) {
      if (capacity < static_cast<long long>(f.size())) return fail("gs_solver_node_features: capacity too small");
      if (!f.empty()) std::memcpy(out, f.data(), sizeof(float) * f.size());
    }
    return GS_OK;
  });
}

int gs_solver_set_node_weights(gs_solver *s, const double *w, long long n) {
  return guarded([&] {
    if (s == nullptr) return fail("null solver");
    if (n < 0 || (n > 0 && w == nullptr)) return fail("gs_solver_set_node_weights: bad arguments");
    s->s->set_node_weights(n == 0 ? std::vector<double>() : std::vector<double>(w, w + n));
    return GS_OK;
  });
}

int gs_solver_error_reduction(gs_solver *s, const double *e0, void *stream, double *ratio) {
  return guarded([&] {
    if (s == nullptr || e0 == nullptr || ratio == nullptr) return fail("null argument");
    *ratio = s->s->error_reduction(e0, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

// ---- kernel-level Backend operations -----------------------------------------
int gs_device_csr_create(int rows, int cols, const int *rp, const int *ci, const void *val,
                         int dtype, gs_device_csr **out) {
  return guarded([&] {
    if (rp == nullptr || out == nullptr) return fail("gs_device_csr_create: null argument");
    // the device kernels index x with every column and walk the row pointers
    // unchecked, so the arrays are validated on the host before upload
    if (rows <= 0 || cols <= 0) return fail("DeviceCSRMatrix: matrix dimensions must be nonzero.");
    check_row_ptr(rows, rp, "DeviceCSRMatrix");
    if (rp[rows] > 0 && (ci == nullptr || val == nullptr))
      return fail("DeviceCSRMatrix: input pointers must not be null.");
    for (int k = 0; k < rp[rows]; ++k)
      if (ci[k] < 0 || ci[k] >= cols) return fail("DeviceCSRMatrix: column index out of range");
    const int rc = require_device(0);
    if (rc != GS_OK) return rc;
    std::unique_ptr<gs_device_csr> m(new gs_device_csr);
    m->m.reset(gsb::device_csr_create(rows, cols, rp, ci, val, dtype));
    *out = m.release();
    return GS_OK;
  });
}

int gs_device_csr_update_values(gs_device_csr *m, const void *val, long long count) {
  return guarded([&] {
    if (m == nullptr || val == nullptr) return fail("null argument");
    gsb::device_csr_update_values(m->m.get(), val, count);
    return GS_OK;
  });
}

void gs_device_csr_destroy(gs_device_csr *m) { delete m; }

int gs_spmv(const gs_device_csr *A, const void *x, void *y, void *stream) {
  return guarded([&] {
    if (A == nullptr || x == nullptr || y == nullptr) return fail("gs_spmv: null argument");
    gsb::spmv(A->m.get(), x, y, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_gauss_seidel_color(const gs_device_csr *A, const int *order, long long start, long long count,
                          const void *rhs, void *x, double omega, void *stream) {
  return guarded([&] {
    if (A == nullptr || order == nullptr || rhs == nullptr || x == nullptr)
      return fail("gs_gauss_seidel_color: null argument");
    if (start < 0 || count < 0 || start + count > A->m->rows)
      return fail("gs_gauss_seidel_color: invalid color range");
    gsb::gauss_seidel_color(A->m.get(), order, start, count, rhs, x, omega, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_block_gauss_seidel_color3x3(const gs_device_csr *A, const int *order, long long start,
                                   long long count, const void *dinv, const void *rhs, void *x,
                                   double omega, void *stream) {
  return guarded([&] {
    if (A == nullptr || order == nullptr || dinv == nullptr || rhs == nullptr || x == nullptr)
      return fail("gs_block_gauss_seidel_color3x3: null argument");
    if (start < 0 || count < 0 || start + count > A->m->rows / 3)
      return fail("gs_block_gauss_seidel_color3x3: invalid color range");
    gsb::block_gauss_seidel_color3x3(A->m.get(), order, start, count, dinv, rhs, x, omega,
                                     static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_apply_block_inverses3x3(long long n, const void *dinv, const void *r, void *c, int dtype,
                               void *stream) {
  return guarded([&] {
    if (dinv == nullptr || r == nullptr || c == nullptr) return fail("null argument");
    if (n < 0 || n > 0x7fffffffLL) return fail("encodeApplyBlockInverses3x3: bad size");
    if (dtype != GS_F32 && dtype != GS_F64) return fail("dtype must be GS_F32 or GS_F64");
    gsb::apply_block_inverses3x3(n, dinv, r, c, dtype, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_dot(long long n, const void *x, const void *y, void *result, int dtype, void *stream) {
  return guarded([&] {
    if (x == nullptr || y == nullptr || result == nullptr) return fail("gs_dot: null argument");
    if (dtype != GS_F32 && dtype != GS_F64) return fail("dtype must be GS_F32 or GS_F64");
    gsb::dot(n, x, y, result, dtype, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_dot_noalloc(long long n, const void *x, const void *y, void *result, int dtype, void *stream) {
  return guarded([&] {
    if (x == nullptr || y == nullptr || result == nullptr) return fail("gs_dot_noalloc: null argument");
    if (dtype != GS_F32 && dtype != GS_F64) return fail("dtype must be GS_F32 or GS_F64");
    gsb::dot_noalloc(n, x, y, result, dtype, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_vector_op(int op, long long n, const void *x, void *y, double alpha, const void *alpha_dev,
                 int dtype, void *stream) {
  return guarded([&] {
    if (op < GS_VEC_AXPY || op > GS_VEC_SCALE_BY_VECTOR) return fail("gs_vector_op: unknown op");
    if (y == nullptr || (x == nullptr && op != GS_VEC_SCALE && op != GS_VEC_SET_ZERO))
      return fail("gs_vector_op: null argument");
    if (dtype != GS_F32 && dtype != GS_F64) return fail("dtype must be GS_F32 or GS_F64");
    gsb::vector_op(op, n, x, y, alpha, alpha_dev, dtype, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

int gs_scalar_op(int op, const void *a, const void *b, void *out, double value, int dtype,
                 void *stream) {
  return guarded([&] {
    if (op < GS_SCALAR_DIVIDE || op > GS_SCALAR_SQRT || out == nullptr) return fail("gs_scalar_op: bad arguments");
    // every op but SET reads a; DIVIDE and MULTIPLY read b as well
    if ((op != GS_SCALAR_SET && a == nullptr) ||
        ((op == GS_SCALAR_DIVIDE || op == GS_SCALAR_MULTIPLY) && b == nullptr))
      return fail("gs_scalar_op: null operand");
    if (dtype != GS_F32 && dtype != GS_F64) return fail("dtype must be GS_F32 or GS_F64");
    gsb::scalar_op(op, a, b, out, value, dtype, static_cast<cudaStream_t>(stream));
    return GS_OK;
  });
}

// ---- device memory, copies and streams ----------------------------------------
namespace {
// Makes `device` current for the scope and restores the caller's device.
struct DeviceScope {
  int saved = -1;
  explicit DeviceScope(int device) {
    gsb::cuda_check(cudaGetDevice(&saved), "cudaGetDevice");
    gsb::cuda_check(cudaSetDevice(device), "cudaSetDevice");
  }
  ~DeviceScope() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};
}  // namespace

int gs_device_malloc(int device, unsigned long long bytes, void **ptr) {
  return guarded([&] {
    if (ptr == nullptr) return fail("gs_device_malloc: null argument");
    *ptr = nullptr;
    const int rc = require_device(device);
    if (rc != GS_OK) return rc;
    if (bytes == 0) return GS_OK;
    DeviceScope scope(device);
    gsb::cuda_check(cudaMalloc(ptr, static_cast<size_t>(bytes)), "cudaMalloc");
    return GS_OK;
  });
}

int gs_device_free(void *ptr) {
  return guarded([&] {
    if (ptr != nullptr) gsb::cuda_check(cudaFree(ptr), "cudaFree");
    return GS_OK;
  });
}

int gs_memcpy(void *dst, const void *src, unsigned long long bytes, int kind, void *stream) {
  return guarded([&] {
    if (kind < GS_COPY_H2D || kind > GS_COPY_D2D) return fail("gs_memcpy: unknown copy kind");
    if (bytes == 0) return GS_OK;
    if (dst == nullptr || src == nullptr) return fail("gs_memcpy: null argument");
    const cudaMemcpyKind k = kind == GS_COPY_H2D   ? cudaMemcpyHostToDevice
                             : kind == GS_COPY_D2H ? cudaMemcpyDeviceToHost
                                                   : cudaMemcpyDeviceToDevice;
    const size_t n = static_cast<size_t>(bytes);
    if (stream == nullptr)
      gsb::cuda_check(cudaMemcpy(dst, src, n, k), "cudaMemcpy");
    else
      gsb::cuda_check(cudaMemcpyAsync(dst, src, n, k, static_cast<cudaStream_t>(stream)), "cudaMemcpyAsync");
    return GS_OK;
  });
}

int gs_memset(void *dst, int byte_value, unsigned long long bytes, void *stream) {
  return guarded([&] {
    if (bytes == 0) return GS_OK;
    if (dst == nullptr) return fail("gs_memset: null argument");
    if (stream == nullptr)
      gsb::cuda_check(cudaMemset(dst, byte_value, static_cast<size_t>(bytes)), "cudaMemset");
    else
      gsb::cuda_check(cudaMemsetAsync(dst, byte_value, static_cast<size_t>(bytes), static_cast<cudaStream_t>(stream)),
                      "cudaMemsetAsync");
    return GS_OK;
  });
}

int gs_stream_create(int device, void **stream) {
  return guarded([&] {
    if (stream == nullptr) return fail("gs_stream_create: null argument");
    *stream = nullptr;
    const int rc = require_device(device);
    if (rc != GS_OK) return rc;
    DeviceScope scope(device);
    cudaStream_t s = nullptr;
    gsb::cuda_check(cudaStreamCreate(&s), "cudaStreamCreate");
    *stream = s;
    return GS_OK;
  });
}

int gs_stream_destroy(void *stream) {
  return guarded([&] {
    if (stream != nullptr) gsb::cuda_check(cudaStreamDestroy(static_cast<cudaStream_t>(stream)), "cudaStreamDestroy");
    return GS_OK;
  });
}

int gs_stream_synchronize(void *stream) {
  return guarded([&] {
    gsb::cuda_check(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "cudaStreamSynchronize");
    return GS_OK;
  });
}

}  // extern "C"
