// Host-side setup for the AMG-PCG path: CSR containers and permutations,
// greedy multicolouring, reverse Cuthill-McKee, the reference's fixed-width
// ELL layout, smoothed-aggregation coarsening, and the synthetic problem
// generators. Everything here is integer or FP64 work that runs once per
// matrix; the per-iteration work lives in the CUDA kernels.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace gsb {

// Compressed sparse row matrix, FP64 values (the setup precision).
struct Csr {
  int rows = 0, cols = 0;
  std::vector<int> rp;   // rows + 1
  std::vector<int> ci;   // nnz
  std::vector<double> v; // nnz
  int nnz() const { return rows == 0 ? 0 : rp[rows]; }
  void check(const char *what) const;
};

// Splittable 64-bit generator (SplitMix64, Steele/Lea/Flood 2014): the one
// RNG used for every synthetic input so CPU tests and GPU runs see the same
// data. uniform() is (x >> 11) * 2^-53 in [0, 1).
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  double normal();  // Box-Muller on two uniforms
};

// Host threads the setup may use: hardware_concurrency, capped at 32 and by
// the environment variable GS_HOST_THREADS when it is set (read once).
int host_threads();

// Runs body(begin, end) over [0, n) cut into contiguous chunks, on up to
// host_threads() threads (serially below `grain` items per thread).
// Every index is visited exactly once; bodies write disjoint outputs, so the
// result does not depend on the thread count. The first exception thrown by
// a body is rethrown after all threads have joined.
void parallel_for(long long n, const std::function<void(long long, long long)> &body, long long grain = 32768);
// Grain for a parallel_for over the rows of a matrix: about 64K stored
// entries per chunk, whatever the row length.
inline long long row_grain(long long rows, long long nnz) {
  return nnz <= 0 ? 32768 : (rows * 65536 + nnz - 1) / nnz < 64 ? 64 : (rows * 65536 + nnz - 1) / nnz;
}

// --- permutations (same index conventions as the reference's Permutation:
//     old_to_new[old] = new, new_to_old[new] = old) -----------------------
void check_permutation(int n, const int *old_to_new, const int *new_to_old);

// A' = P A P^T as HostCSRMatrix::applyPermutation does it
// (src/HostSparseMatrix.cc:118-249): new row i is old row new_to_old[i],
// columns are mapped through old_to_new and keep their old in-row order.
Csr apply_permutation(const Csr &a, const int *old_to_new, const int *new_to_old);

// permuteMatrix (src/SparseMatrixUtils.cc:8-31): entry (i, j) moves to
// (row_old_to_new[i], col_old_to_new[j]); columns end up sorted within each
// row and duplicate positions are summed.
Csr permute_matrix(const Csr &a, const int *row_old_to_new, const int *col_old_to_new);

Csr transpose(const Csr &a);
// C = A B, Gustavson row-by-row in stored order; columns sorted per row.
Csr spgemm(const Csr &a, const Csr &b);

// --- greedy multicolouring (GraphColoring::compute, src/GraphColoring.cc:9-72)
// colours[v], vertices grouped by colour in increasing vertex order, offsets
// of size ncolours + 1. Returns the number of colours.
int greedy_coloring(int n, const int *rp, const int *ci, std::vector<int> &colors,
                    std::vector<int> &vertices, std::vector<int> &offsets);
// The same greedy first-fit, visiting the vertices in smallest-last order
// (Matula & Beck, J. ACM 30(3), 1983: repeatedly remove a vertex of minimum
// remaining degree, lowest index first; colour in reverse removal order).
// Same output layout as greedy_coloring; usually fewer colours on Galerkin
// coarse levels and unstructured meshes. No reference counterpart.
int smallest_last_coloring(int n, const int *rp, const int *ci, std::vector<int> &colors,
                           std::vector<int> &vertices, std::vector<int> &offsets);
// Colouring of the strong couplings only (no reference counterpart): the
// graph of the off-diagonal entries with |a_ij| >= theta sqrt(|a_ii a_jj|) is
// coloured first-fit (row order, or smallest-last order where that gives
// fewer colours), so rows joined by a weak entry may share a colour. A
// Gauss-Seidel pass over such a colouring reads its same-colour neighbours
// from the iterate the sweep started with (Jacobi within a colour). Then
// every row whose same-colour off-diagonal mass sum |a_ij| reaches
// rho |a_ii| moves, in row order, to the lowest colour that has no strong
// neighbour of the row and leaves that mass below rho |a_ii| (a new colour if
// none does), until no row is left (at most 64 passes; then the exact
// colouring of the whole graph is returned). With rho < 1 the same-colour
// part W keeps D - W strictly diagonally dominant, so the forward and
// backward sweeps stay a convergent symmetric pair. Same output layout as
// greedy_coloring.
int relaxed_coloring(int n, const int *rp, const int *ci, const double *v, double theta, double rho,
                     std::vector<int> &colors, std::vector<int> &vertices, std::vector<int> &offsets);
// The same for the nodes of a 3x3-blocked matrix (block Gauss-Seidel): a node
// pair is strong when ||A_IJ||_F >= theta sqrt(||A_II||_F ||A_JJ||_F), and a
// node keeps sum ||A_IJ||_F over its same-colour nodes below
// rho / ||A_II^-1||_F <= rho lambda_min(A_II): block diagonal dominance of
// D - W, so the block sweeps stay a convergent symmetric pair.
int relaxed_block_coloring(const Csr &a, double theta, double rho, std::vector<int> &colors,
                           std::vector<int> &vertices, std::vector<int> &offsets);

// --- reverse Cuthill-McKee (RCMReordering::compute,
//     src/ReorderingStrategies/RCMReordering.cc:11-110).
void rcm(int n, const int *rp, const int *ci, int *old_to_new, int *new_to_old);

// --- node graph of a 3x3-blocked matrix (buildBlockGraph,
//     src/BlockUtils.cc:126-216): sorted, de-duplicated off-diagonal blocks.
void block_graph(const Csr &a, int block, std::vector<int> &g_rp, std::vector<int> &g_ci);

// --- inverse 3x3 diagonal blocks, row-major 9 per node, via Cholesky
//     (extractInverseDiagonalBlocks3x3, src/BlockUtils.cc:218-277).
//     Returns the index of the first non-SPD block, or -1.
int block_inverses3x3(const Csr &a, std::vector<double> &dinv);

// --- node permutation expanded to dofs (expandBlockPermutation,
//     src/BlockUtils.cc:7-55).
void expand_block_permutation(int nodes, int block, const int *node_o2n, const int *node_n2o,
                              int *o2n, int *n2o);

// --- the reference's fixed-width ELL (HostELLMatrix, src/HostELLMatrix.cc):
//     slot-major (index = slot * rows + row), padding col 0 / value 0, and
//     the entries beyond `width` in an overflow CSR.
struct HostEll {
  int rows = 0, cols = 0, width = 0;
  std::vector<int> col;       // rows * width
  std::vector<double> val;    // rows * width
  std::vector<int> ovf_rp;    // rows + 1
  std::vector<int> ovf_ci;
  std::vector<double> ovf_v;
};
HostEll build_ell(const Csr &a, int width);

// --- smoothed aggregation (Vanek, Mandel & Brezina, Computing 56, 1996) --
struct SaOptions {
  int block = 1;           // dofs per node (1 scalar, 3 elasticity)
  double eps_strong = 0.1; // strength threshold on level 0, halved per level
  int max_levels = 10;     // maximum number of coarsenings
  int min_dofs = 1000;     // stop once a level has at most this many rows
  // 0: sequential greedy aggregation in node order (Vanek's three steps);
  // 1: aggregation from a distance-2 maximal independent set (the parallel
  // algorithm the GPU setup runs; see mis2_aggregate in setup.cc)
  int aggregation = 0;
};
struct Hierarchy {
  int block = 1;
  std::vector<Csr> A;                 // levels
  std::vector<Csr> P;                 // P[k]: level k+1 -> level k
  std::vector<Csr> R;                 // R[k] = P[k]^T
  std::vector<std::vector<int>> agg;  // agg[k][node of level k] (-1 = isolated)
};
// One coarsening step: aggregates, smoothed prolongator P, R = P^T,
// Ac = R A P.
void sa_coarsen(const Csr &a, int block, double eps, std::vector<int> &agg, Csr &p, Csr &r,
                Csr &ac, int aggregation = 0);
// Priority of a node in the distance-2 independent-set rounds.
uint32_t node_priority(uint32_t v);
// AMGHierarchyBuilder::build semantics
// (examples/amgSolver/src/AMGHierarchyBuilder.cc:59-150).
Hierarchy build_hierarchy(const Csr &a, const SaOptions &opt);

// HierarchicalReordering::compute
// (src/ReorderingStrategies/HierarchicalReordering.cc:217-278): RCM on the
// coarsest level; every finer level ordered by the rank of each row's
// strongest parent in the restriction (largest |R(c, f)| in FP32, the first
// coarse row winning ties; rows without a parent last), then by the row's
// own RCM rank. One (old_to_new, new_to_old) pair per level, finest first.
void hierarchical_reordering(const Hierarchy &h, std::vector<std::vector<int>> &old_to_new,
                             std::vector<std::vector<int>> &new_to_old);

// --- synthetic problems -------------------------------------------------
// 7-point finite-difference Laplacian, nx*ny*nz interior unknowns, Dirichlet
// zero boundary, diagonal 6 and off-diagonals -1, x fastest.
Csr poisson7(int nx, int ny, int nz);
// Cell-centred 7-point variable-coefficient operator: interior face
// transmissibility = harmonic mean 2 k_i k_j / (k_i + k_j); a boundary face
// contributes 2 k_i (Dirichlet zero half a cell away).
Csr varcoef7(int nx, int ny, int nz, const std::vector<double> &k);
// exp(sigma * G) with G a unit-variance Gaussian random field with Gaussian
// correlation of length `corr` cells (white noise from SplitMix64(seed),
// separable periodic Gaussian filter of standard deviation corr/sqrt(2),
// rescaled to unit sample variance).
std::vector<double> grf_coefficients(int nx, int ny, int nz, double corr, double sigma,
                                     uint64_t seed);
// Cell coefficients log-uniform in [lo, hi].
std::vector<double> loguniform_coefficients(int n, double lo, double hi, uint64_t seed);
// Unit cube cut into m^3 cubes of 6 Kuhn tetrahedra each, interior vertices
// jittered by U[-jitter*h, jitter*h] per coordinate, P1 stiffness Laplacian
// with Dirichlet on all boundary vertices (eliminated): (m-1)^3 unknowns.
Csr kuhn_laplacian(int m, double jitter, uint64_t seed);
// P1 linear elasticity on the unit cube with v^3 vertices and Kuhn
// tetrahedra; Young's modulus exp(N(0,1)) per element (seed), Poisson ratio
// nu, the x = 0 face clamped (eliminated), 3 dofs per vertex interleaved.
// `rhs` receives the consistent load of a unit body force in -z.
Csr elasticity_p1(int v, double nu, uint64_t seed, std::vector<double> &rhs);
// RHS uniform in [-1, 1].
std::vector<double> uniform_rhs(int n, uint64_t seed);

}  // namespace gsb
