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
  }
  std::printf("ok %ld refused %ld\n", ok, refused);
  return 0;
}
