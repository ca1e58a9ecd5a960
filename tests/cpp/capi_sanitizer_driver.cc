// The host entry points of the C ABI (csrc/capi.cc with csrc/setup.cc) under
// AddressSanitizer and UndefinedBehaviorSanitizer, on random small graphs: half
// well formed (rows in any order), half malformed (row pointers that do not start
// at 0 or decrease, column indices out of range), with random maps and block
// sizes: colourings, RCM, permuteMatrix, HostELLMatrix, node graph, block inverses,
// host CSR and the SA hierarchy. Every call returns a status; none reads or writes
// outside the arrays the ABI contract sizes. Built and run by tests/test_sanitizers.py
// (only host code is reached; the CUDA parts of capi.cc are left unresolved).
#include <gpusolver_b200.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>
// SplitMix64 for the random cases
static uint64_t s = 12345;
static uint64_t next() { uint64_t z = (s += 0x9e3779b97f4a7c15ULL); z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL; z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL; return z ^ (z >> 31); }
static int rnd(int lo, int hi) { return lo + static_cast<int>(next() % static_cast<uint64_t>(hi - lo + 1)); }
int main() {
  long ok = 0, refused = 0;
  for (int trial = 0; trial < 4000; ++trial) {
    const int n = rnd(0, 9);
    int L = rnd(0, 24);
    std::vector<int> ci, rp(n + 1);
    if (trial % 2 == 0 && n > 0) {
      // well formed: rows of random length with in-range columns, in any order
      rp[0] = 0;
      for (int r = 0; r < n; ++r) {
        const int len = rnd(0, 5);
        for (int t = 0; t < len; ++t) ci.push_back(rnd(0, n - 1));
        rp[r + 1] = static_cast<int>(ci.size());
      }
      L = static_cast<int>(ci.size());
    } else {
      ci.resize(L);
      for (int &c : ci) c = rnd(-2, n + 2);
      const bool sorted = next() & 1;
      for (int &r : rp) r = rnd(-1, L);
      if (sorted) { std::sort(rp.begin(), rp.end()); rp[0] = 0; for (int &r : rp) if (r < 0) r = 0; }
    }
    ci.push_back(0);  // keeps data() valid for L == 0
    std::vector<double> v(L > 0 ? L : 1, 1.5);
    std::vector<int> colors(n + 1), verts(n + 1), offs(n + 2), o2n(n + 1), n2o(n + 1), grp(n + 2), gci(L + 1), orp(n + 2), oci(L + 1);
    std::vector<double> ov(L + 1), ev(static_cast<size_t>(n) * 4 + 1), dinv(3 * n + 3);
    std::vector<int> ec(static_cast<size_t>(n) * 4 + 1);
    int nc = 0, gn = 0, on = 0;
    const int *prp = n >= 0 ? rp.data() : nullptr;
    int rc[8];
    rc[0] = gs_greedy_coloring(n, prp, ci.data(), colors.data(), verts.data(), offs.data(), &nc);
    rc[1] = gs_smallest_last_coloring(n, prp, ci.data(), colors.data(), verts.data(), offs.data(), &nc);
    {
      // strong-coupling colourings with random (possibly invalid) theta and rho
      const double theta = 0.05 * rnd(-1, 3), rho = 0.3 * rnd(-1, 4);
      (gs_relaxed_coloring(n, prp, ci.data(), v.data(), theta, rho, colors.data(), verts.data(), offs.data(), &nc) ==
               GS_OK
           ? ok : refused)++;
      (gs_relaxed_block_coloring(n, prp, ci.data(), v.data(), theta, rho, colors.data(), verts.data(), offs.data(),
                                 &nc) == GS_OK
           ? ok : refused)++;
    }
    rc[2] = gs_rcm(n, prp, ci.data(), o2n.data(), n2o.data());
    std::vector<int> perm(n + 1);
    for (int i = 0; i < n; ++i) perm[i] = (next() & 3) ? (i + 1) % (n ? n : 1) : rnd(-1, n);
    rc[3] = gs_permute_matrix(n, n, prp, ci.data(), v.data(), perm.data(), perm.data(), orp.data(), oci.data(), ov.data());
    rc[4] = gs_ell_build(n, n, prp, ci.data(), v.data(), 4, ec.data(), ev.data(), orp.data(), oci.data(), ov.data(), &on);
    rc[5] = gs_block_graph(n, prp, ci.data(), rnd(0, 3), grp.data(), gci.data(), &gn);
    rc[6] = gs_block_inverses3x3(n, prp, ci.data(), v.data(), dinv.data());
    gs_host_csr *m = nullptr;
    rc[7] = gs_host_csr_create(n, n, prp, ci.data(), v.data(), &m);
    if (m) {
      gs_hierarchy *h = nullptr;
      if (gs_hierarchy_build(m, 1, 0.1, 4, 2, &h) == GS_OK) gs_hierarchy_destroy(h);
      gs_host_csr_destroy(m);
    }
    for (int r : rc) (r == GS_OK ? ok : refused)++;

    // applyPermutation with a random (possibly invalid) pair of maps
    std::vector<int> q(n + 1), qi(n + 1);
    for (int i = 0; i < n; ++i) q[i] = (i + 1) % n;
    for (int i = 0; i < n; ++i) qi[q[i]] = i;
    if (n > 0 && (next() & 1)) qi[rnd(0, n - 1)] = rnd(-1, n);
    (gs_apply_permutation(n, prp, ci.data(), v.data(), q.data(), qi.data(), orp.data(), oci.data(), ov.data()) == GS_OK
         ? ok : refused)++;
    // node permutation expanded to dofs, random block size
    const int block = rnd(-1, 3);
    std::vector<int> eo(static_cast<size_t>(n) * 4 + 1), en(static_cast<size_t>(n) * 4 + 1);
    (gs_expand_block_permutation(n, block, q.data(), qi.data(), eo.data(), en.data()) == GS_OK ? ok : refused)++;
    // generated problems with random (possibly invalid) parameters
    {
      const int kind = rnd(-1, 5);
      const int ip[3] = {rnd(-1, 6), rnd(-1, 6), rnd(-1, 6)};
      const double dp[2] = {rnd(-2, 9) * 0.1, rnd(-2, 20) * 0.1};
      gs_host_csr *pm = nullptr;
      if (gs_problem_create(kind, ip, dp, next(), &pm) == GS_OK) {
        ++ok;
        gs_hierarchy *h = nullptr;
        if (gs_hierarchy_build(pm, kind == GS_PROBLEM_ELASTICITY_P1 ? 3 : 1, 0.1, 5, 4, &h) == GS_OK) {
          // the levels back through gs_hierarchy_from_levels, then the reordering
          const int L = gs_hierarchy_num_levels(h);
          std::vector<std::vector<int>> lrp(3 * L), lci(3 * L);
          std::vector<std::vector<double>> lv(3 * L);
          std::vector<gs_csr> A(L), P(L), R(L);
          for (int k = 0; k < L; ++k)
            for (int which = 0; which < 3; ++which) {
              if (which > 0 && k + 1 == L) continue;
              int rows = 0, cols = 0, nnz = 0;
              gs_hierarchy_matrix_info(h, k, which, &rows, &cols, &nnz);
              const int t = 3 * k + which;
              lrp[t].resize(rows + 1);
              lci[t].resize(nnz + 1);
              lv[t].resize(nnz + 1);
              gs_hierarchy_matrix(h, k, which, lrp[t].data(), lci[t].data(), lv[t].data());
              gs_csr &m = which == 0 ? A[k] : which == 1 ? P[k] : R[k];
              m = gs_csr{rows, cols, lrp[t].data(), lci[t].data(), lv[t].data()};
            }
          if (L > 1 && (next() & 1)) A[1].cols += 1;  // a level that does not fit
          gs_hierarchy *h2 = nullptr;
          if (gs_hierarchy_from_levels(L, A.data(), P.data(), R.data(), 1, &h2) == GS_OK) {
            std::vector<std::vector<int>> ro(L), rn(L);
            std::vector<int *> po(L), pn(L);
            for (int k = 0; k < L; ++k) ro[k].resize(A[k].rows), rn[k].resize(A[k].rows), po[k] = ro[k].data(), pn[k] = rn[k].data();
            (gs_hierarchical_reordering(h2, po.data(), pn.data()) == GS_OK ? ok : refused)++;
            gs_hierarchy_destroy(h2);
          } else {
            ++refused;
          }
          gs_hierarchy_destroy(h);
        }
        gs_host_csr_destroy(pm);
      } else {
        ++refused;
      }
    }
  }
  std::printf("ok %ld refused %ld\n", ok, refused);
  return 0;
}
