// Host containers and helpers of the C++ API mirror (no GPU needed):
// HostCSRMatrix with and without a permutation (src/HostSparseMatrix.cc of
// the reference), HostELLMatrix (src/HostELLMatrix.cc), permuteMatrix
// (src/SparseMatrixUtils.cc), the block helpers (src/BlockUtils.cc) and the
// reordering strategies. Each property is checked here by direct loops and
// printed as "key value" lines; error messages are printed for comparison
// with the reference's.
#include <GPUSolver/BlockUtils.h>
#include <GPUSolver/HostELLMatrix.h>
#include <GPUSolver/HostSparseMatrix.h>
#include <GPUSolver/SparseMatrixUtils.h>
#include <GPUSolver/ReorderingStrategies/IdentityReordering.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>
#include <GPUSolver/cuda/CudaDeviceCSRMatrix.h>
#include <GPUSolver/cuda/CudaDeviceIndexVector.h>
#include <GPUSolver/cuda/CudaDeviceScalar.h>
#include <GPUSolver/cuda/CudaDeviceVector.h>
#include <GPUSolver/cuda/CudaEncoder.h>

#include <cmath>
#include <type_traits>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

using gpuSolver::CsrMatrix;

// the reference's CUDA class names name the B200 implementations of the interfaces
static_assert(std::is_base_of<gpuSolver::Backend, gpuSolver::CudaBackend>::value, "CudaBackend");
static_assert(std::is_base_of<gpuSolver::BackendEncoder, gpuSolver::CudaEncoder>::value, "CudaEncoder");
static_assert(std::is_base_of<gpuSolver::DeviceVector, gpuSolver::CudaDeviceVector>::value, "CudaDeviceVector");
static_assert(std::is_base_of<gpuSolver::DeviceIndexVector, gpuSolver::CudaDeviceIndexVector>::value,
              "CudaDeviceIndexVector");
static_assert(std::is_base_of<gpuSolver::DeviceScalar, gpuSolver::CudaDeviceScalar>::value, "CudaDeviceScalar");
static_assert(std::is_base_of<gpuSolver::DeviceCSRMatrix, gpuSolver::CudaDeviceCSRMatrix>::value,
              "CudaDeviceCSRMatrix");

// 7-point Laplacian on an m^3 grid with a varying diagonal, so that moved
// values are told apart
static CsrMatrix grid(int m) {
  std::vector<int> rp{0}, ci;
  std::vector<double> v;
  for (int z = 0; z < m; ++z)
    for (int y = 0; y < m; ++y)
      for (int x = 0; x < m; ++x) {
        const int i = (z * m + y) * m + x;
        auto add = [&](int j, double a) { ci.push_back(j), v.push_back(a); };
        if (z > 0) add(i - m * m, -1);
        if (y > 0) add(i - m, -1);
        if (x > 0) add(i - 1, -1);
        add(i, 6 + 0.25 * i);
        if (x + 1 < m) add(i + 1, -1);
        if (y + 1 < m) add(i + m, -1);
        if (z + 1 < m) add(i + m * m, -1);
        rp.push_back(static_cast<int>(ci.size()));
      }
  return CsrMatrix(m * m * m, m * m * m, rp, ci, v);
}

// 3x3 blocks: node graph of a path of `nodes` nodes, diagonal blocks SPD
static CsrMatrix block_path(int nodes) {
  std::vector<int> rp{0}, ci;
  std::vector<double> v;
  for (int node = 0; node < nodes; ++node)
    for (int r = 0; r < 3; ++r) {
      for (int nb = node - 1; nb <= node + 1; ++nb) {
        if (nb < 0 || nb >= nodes) continue;
        for (int c = 0; c < 3; ++c) {
          ci.push_back(3 * nb + c);
          if (nb == node) v.push_back(r == c ? 4.0 + node : 0.5);
          else v.push_back(-0.1);
        }
      }
      rp.push_back(static_cast<int>(ci.size()));
    }
  return CsrMatrix(3 * nodes, 3 * nodes, rp, ci, v);
}

static void expect_throw(const char *key, const std::function<void()> &f) {
  try {
    f();
    std::printf("%s no-throw\n", key);
  } catch (const std::runtime_error &e) {
    std::printf("%s throws: %s\n", key, e.what());
  }
}

static const char *ok(bool b) { return b ? "ok" : "FAIL"; }

int main() {
  using namespace gpuSolver;
  const CsrMatrix K = grid(4);
  const int n = K.rows();
  std::vector<float> kv(K.values.begin(), K.values.end());

  // ---- HostCSRMatrix ----
  expect_throw("csr_dims", [&] { HostCSRMatrix m(0, 3, 0, K.rowPtr.data(), K.colIdx.data(), kv.data()); });
  expect_throw("csr_null", [&] { HostCSRMatrix m(3, 3, 0, nullptr, K.colIdx.data(), kv.data()); });
  {
    HostCSRMatrix rect(2, 3, 2, std::vector<int>{0, 1, 2}.data(), std::vector<int>{0, 2}.data(),
                       std::vector<float>{1, 2}.data());
    std::vector<int> id{0, 1};
    Permutation p2(2, id.data(), id.data());
    expect_throw("csr_square", [&] { rect.applyPermutation(p2); });
  }
  RCMReordering rcm;
  std::vector<int> o2n(n), n2o(n);
  rcm.compute(n, K.rowPtr.data(), K.colIdx.data(), o2n.data(), n2o.data());
  const Permutation P(n, o2n.data(), n2o.data());
  {
    std::vector<int> id(8);
    for (int i = 0; i < 8; ++i) id[i] = i;
    Permutation small(8, id.data(), id.data());
    HostCSRMatrix m(n, n, K.nonZeros(), K.rowPtr.data(), K.colIdx.data(), kv.data());
    expect_throw("csr_perm_size", [&] { m.applyPermutation(small); });
  }
  HostCSRMatrix A(n, n, K.nonZeros(), K.rowPtr.data(), K.colIdx.data(), kv.data());
  std::printf("csr_unpermuted %s\n", ok(!A.isPermuted() && A.permutation() == nullptr &&
                                        A.activeRowPtr() == A.rowPtr() && A.activeValPtr() == A.values()));
  A.applyPermutation(P);
  // row r of A' is row n2o[r] of A, columns mapped by o2n, order kept
  bool same = A.isPermuted() && A.permutation() != &P && A.permutation()->size() == static_cast<std::size_t>(n);
  for (int r = 0; r < n && same; ++r) {
    const int old = n2o[r];
    const int len = K.rowPtr[old + 1] - K.rowPtr[old];
    same = A.activeRowPtr()[r + 1] - A.activeRowPtr()[r] == len;
    for (int t = 0; t < len && same; ++t) {
      const int kk = K.rowPtr[old] + t, kp = A.activeRowPtr()[r] + t;
      same = A.activeColPtr()[kp] == o2n[K.colIdx[kk]] && A.activeValPtr()[kp] == kv[kk];
    }
  }
  bool orig = true;
  for (int k = 0; k < K.nonZeros(); ++k) orig = orig && A.colIdx()[k] == K.colIdx[k] && A.values()[k] == kv[k];
  std::printf("csr_permuted %s originals_kept %s\n", ok(same), ok(orig));
  HostCSRMatrix B(K, P);  // from the container, FP64 values rounded once to FP32
  bool sameB = true;
  for (int k = 0; k < K.nonZeros(); ++k)
    sameB = sameB && B.activeColPtr()[k] == A.activeColPtr()[k] && B.activeValPtr()[k] == A.activeValPtr()[k];
  std::printf("csr_from_container %s\n", ok(sameB));

  // ---- HostELLMatrix: width 4 of rows with up to 7 entries ----
  expect_throw("ell_width0", [&] { HostELLMatrix e(A, 0); });
  HostELLMatrix E(A, 4);
  bool ell = E.rows() == A.rows() && E.ellWidth() == 4 && E.nnz() == A.nnz();
  std::size_t ovf = 0;
  for (std::size_t r = 0; r < E.rows() && ell; ++r) {
    const int b = A.activeRowPtr()[r], len = A.activeRowPtr()[r + 1] - b;
    for (int s = 0; s < 4; ++s) {
      const std::size_t cell = static_cast<std::size_t>(s) * E.rows() + r;
      if (s < len) ell = ell && E.ellColIdx()[cell] == A.activeColPtr()[b + s] && E.ellValues()[cell] == A.activeValPtr()[b + s];
      else ell = ell && E.ellColIdx()[cell] == 0 && E.ellValues()[cell] == 0.0f;
    }
    const int ob = E.overflowRowPtr()[r], olen = E.overflowRowPtr()[r + 1] - ob;
    ell = ell && olen == (len > 4 ? len - 4 : 0);
    for (int t = 0; t < olen && ell; ++t)
      ell = ell && E.overflowColIdx()[ob + t] == A.activeColPtr()[b + 4 + t] &&
            E.overflowValues()[ob + t] == A.activeValPtr()[b + 4 + t];
    ovf += static_cast<std::size_t>(olen);
  }
  std::printf("ell %s overflow %zu of %zu\n", ok(ell && ovf == E.overflowNnz()), E.overflowNnz(), E.nnz());

  // ---- permuteMatrix: rows reversed, columns by RCM; columns sorted per row ----
  std::vector<int> rev(n);
  for (int i = 0; i < n; ++i) rev[i] = n - 1 - i;
  const CsrMatrix M = permuteMatrix(K, rev.data(), o2n.data());
  bool pm = M.nonZeros() == K.nonZeros();
  for (int i = 0; i < n && pm; ++i) {
    const int r = rev[i];
    pm = M.rowPtr[r + 1] - M.rowPtr[r] == K.rowPtr[i + 1] - K.rowPtr[i];
    for (int k = M.rowPtr[r] + 1; k < M.rowPtr[r + 1] && pm; ++k) pm = M.colIdx[k - 1] < M.colIdx[k];
    for (int k = K.rowPtr[i]; k < K.rowPtr[i + 1] && pm; ++k) {
      bool found = false;
      for (int q = M.rowPtr[r]; q < M.rowPtr[r + 1]; ++q)
        found = found || (M.colIdx[q] == o2n[K.colIdx[k]] && M.values[q] == K.values[k]);
      pm = found;
    }
  }
  std::printf("permute_matrix %s\n", ok(pm));
  std::vector<int> dup(n, 0);
  expect_throw("permute_matrix_not_bijective", [&] { permuteMatrix(K, dup.data(), o2n.data()); });

  // ---- block helpers ----
  const CsrMatrix Bp = block_path(5);
  const BlockGraph g = buildBlockGraph(Bp, 3);
  std::string gs;
  for (std::size_t i = 0; i + 1 < g.rowPtr.size(); ++i) {
    gs += std::to_string(i) + ":";
    for (int k = g.rowPtr[i]; k < g.rowPtr[i + 1]; ++k) gs += std::to_string(g.colPtr[k]) + ",";
    gs += ";";
  }
  std::printf("block_graph %s\n", gs.c_str());
  const HostCSRMatrix Hb(Bp);
  const BlockGraph g2 = buildBlockGraph(Hb, 3);
  std::printf("block_graph_host %s\n", ok(g2.rowPtr == g.rowPtr && g2.colPtr == g.colPtr));
  expect_throw("block_graph_divisible", [&] { buildBlockGraph(K, 3); });
  {
    // unsymmetric pattern: 4 nodes of size 1, full upper triangle (10 entries, 12 graph edges)
    std::vector<int> rp{0}, ci;
    std::vector<double> v;
    for (int i = 0; i < 4; ++i) {
      for (int j = i; j < 4; ++j) ci.push_back(j), v.push_back(i == j ? 2.0 : 1.0);
      rp.push_back(static_cast<int>(ci.size()));
    }
    const CsrMatrix U(4, 4, rp, ci, v);
    expect_throw("block_graph_unsymmetric", [&] { buildBlockGraph(U, 1); });
  }
  const std::vector<float> dinv = extractInverseDiagonalBlocks3x3(Hb);
  double worst = 0;
  for (int node = 0; node < 5; ++node)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double s = 0;
        for (int t = 0; t < 3; ++t) s += (r == t ? 4.0 + node : 0.5) * dinv[9 * node + 3 * t + c];
        worst = std::fmax(worst, std::fabs(s - (r == c ? 1.0 : 0.0)));
      }
  std::printf("block_inverse_residual %.3g\n", worst);
  {
    CsrMatrix S = block_path(2);
    for (int k = 0; k < S.nonZeros(); ++k) S.values[k] = -S.values[k];
    const HostCSRMatrix Hs(S);
    expect_throw("block_inverse_not_spd", [&] { extractInverseDiagonalBlocks3x3(Hs); });
  }
  const int no2n[3] = {2, 0, 1}, nn2o[3] = {1, 2, 0};
  const Permutation nodes(3, no2n, nn2o);
  const Permutation dofs = expandBlockPermutation(nodes, 3, 3);
  bool ex = dofs.size() == 9;
  for (int v = 0; v < 3 && ex; ++v)
    for (int c = 0; c < 3; ++c)
      ex = ex && dofs.oldToNew()[3 * v + c] == 3 * no2n[v] + c && dofs.newToOld()[3 * no2n[v] + c] == 3 * v + c;
  std::printf("expand_block_permutation %s\n", ok(ex));

  // ---- reordering strategies through the base class ----
  IdentityReordering idr;
  const ReorderingStrategy &base = idr;
  std::vector<int> io2n(n, -1), in2o(n, -1);
  base.compute(n, K.rowPtr.data(), K.colIdx.data(), io2n.data(), in2o.data());
  bool ident = true;
  for (int i = 0; i < n; ++i) ident = ident && io2n[i] == i && in2o[i] == i;
  std::printf("identity_reordering %s\n", ok(ident));
  return 0;
}
