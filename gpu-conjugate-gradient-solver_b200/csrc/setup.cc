// Host-side setup for the AMG-PCG path. See setup.h for the contract of each
// function and the reference routine whose observable behaviour it keeps.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <exception>
#include <numeric>
#include <queue>
#include <thread>
#include <stdexcept>
#include <string>

namespace gsb {

void Csr::check(const char *what) const {
  if (rows < 0 || cols < 0 || static_cast<int>(rp.size()) != rows + 1)
    throw std::runtime_error(std::string(what) + ": bad row pointer size");
  if (rp[0] != 0) throw std::runtime_error(std::string(what) + ": row pointer must start at 0");
  for (int i = 0; i < rows; ++i)
    if (rp[i + 1] < rp[i]) throw std::runtime_error(std::string(what) + ": row pointer decreases");
  if (static_cast<int>(ci.size()) != rp[rows] || static_cast<int>(v.size()) != rp[rows])
    throw std::runtime_error(std::string(what) + ": column/value arrays do not match nnz");
  for (int c : ci)
    if (c < 0 || c >= cols) throw std::runtime_error(std::string(what) + ": column index out of range");
}

double SplitMix64::normal() {
  double u1 = uniform();
  double u2 = uniform();
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// ---------------------------------------------------------------------------
// permutations
// ---------------------------------------------------------------------------
void check_permutation(int n, const int *o2n, const int *n2o) {
  if (n <= 0) throw std::runtime_error("Permutation: size must be nonzero.");
  if (o2n == nullptr || n2o == nullptr)
    throw std::runtime_error("Permutation: input pointers must not be null.");
  for (int i = 0; i < n; ++i) {
    const int j = o2n[i];
    if (j < 0 || j >= n) throw std::runtime_error("Permutation: oldToNew contains invalid index.");
    if (n2o[j] != i) throw std::runtime_error("Permutation: mappings are not inverses.");
  }
}

Csr apply_permutation(const Csr &a, const int *o2n, const int *n2o) {
  if (a.rows != a.cols) throw std::runtime_error("applyPermutation: matrix must be square.");
  check_permutation(a.rows, o2n, n2o);
  Csr out;
  out.rows = out.cols = a.rows;
  out.rp.assign(a.rows + 1, 0);
  for (int i = 0; i < a.rows; ++i) {
    const int old = n2o[i];
    out.rp[i + 1] = out.rp[i] + (a.rp[old + 1] - a.rp[old]);
  }
  out.ci.resize(a.nnz());
  out.v.resize(a.nnz());
  for (int i = 0; i < a.rows; ++i) {
    const int old = n2o[i];
    int dst = out.rp[i];
    for (int k = a.rp[old]; k < a.rp[old + 1]; ++k, ++dst) {
      out.ci[dst] = o2n[a.ci[k]];
      out.v[dst] = a.v[k];
    }
  }
  return out;
}

int host_threads() {
  static const int n = [] {
    int t = static_cast<int>(std::min(32u, std::max(1u, std::thread::hardware_concurrency())));
    if (const char *e = std::getenv("GS_HOST_THREADS")) {
      const int v = std::atoi(e);
      if (v > 0) t = std::min(t, v);
    }
    return t;
  }();
  return n;
}

void parallel_for(long long n, const std::function<void(long long, long long)> &body, long long grain) {
  if (n <= 0) return;
  const long long hw = host_threads();
  const long long threads = std::min<long long>({hw, 32, (n + grain - 1) / std::max(1LL, grain)});
  if (threads <= 1) {
    body(0, n);
    return;
  }
  std::vector<std::exception_ptr> errors(threads);
  std::vector<std::thread> pool;
  pool.reserve(threads - 1);
  const auto run = [&](long long t) {
    try {
      body(n * t / threads, n * (t + 1) / threads);
    } catch (...) {
      errors[t] = std::current_exception();
    }
  };
  for (long long t = 1; t < threads; ++t) pool.emplace_back(run, t);
  run(0);
  for (auto &th : pool) th.join();
  for (auto &e : errors)
    if (e) std::rethrow_exception(e);
}

Csr permute_matrix(const Csr &a, const int *ro2n, const int *co2n) {
  Csr out;
  out.rows = a.rows;
  out.cols = a.cols;
  out.rp.assign(a.rows + 1, 0);
  for (int i = 0; i < a.rows; ++i) out.rp[ro2n[i] + 1] = a.rp[i + 1] - a.rp[i];
  for (int i = 0; i < a.rows; ++i) out.rp[i + 1] += out.rp[i];
  out.ci.resize(a.nnz());
  out.v.resize(a.nnz());
  // Each old row lands in its own range of the new arrays, its entries in
  // increasing new column, equal columns in stored order (a stable sort:
  // insertion sort for short rows, (column, position) keys otherwise).
  parallel_for(a.rows, [&](long long i0, long long i1) {
    std::vector<std::pair<int, int>> key;  // (new column, stored position)
    for (long long i = i0; i < i1; ++i) {
      const int b = a.rp[i], e = a.rp[i + 1];
      key.clear();
      for (int k = b; k < e; ++k) key.emplace_back(co2n[a.ci[k]], k);
      if (key.size() <= 32) {
        for (size_t x = 1; x < key.size(); ++x) {
          const std::pair<int, int> kv = key[x];
          size_t y = x;
          while (y > 0 && key[y - 1].first > kv.first) key[y] = key[y - 1], --y;
          key[y] = kv;
        }
      } else {
        std::sort(key.begin(), key.end());
      }
      int dst = out.rp[ro2n[i]];
      for (const auto &kv : key) out.ci[dst] = kv.first, out.v[dst] = a.v[kv.second], ++dst;
    }
  }, row_grain(a.rows, a.nnz()));
  // Sum duplicate positions (none arise from a bijective relabelling of a
  // matrix without duplicates, but keep the documented semantics).
  bool dup = false;
  for (int i = 0; i < out.rows && !dup; ++i)
    for (int k = out.rp[i] + 1; k < out.rp[i + 1]; ++k)
      if (out.ci[k] == out.ci[k - 1]) { dup = true; break; }
  if (!dup) return out;
  Csr m;
  m.rows = out.rows;
  m.cols = out.cols;
  m.rp.assign(out.rows + 1, 0);
  for (int i = 0; i < out.rows; ++i) {
    for (int k = out.rp[i]; k < out.rp[i + 1]; ++k) {
      if (k > out.rp[i] && out.ci[k] == out.ci[k - 1]) {
        m.v.back() += out.v[k];
      } else {
        m.ci.push_back(out.ci[k]);
        m.v.push_back(out.v[k]);
      }
    }
    m.rp[i + 1] = static_cast<int>(m.ci.size());
  }
  return m;
}

Csr transpose(const Csr &a) {
  Csr t;
  t.rows = a.cols;
  t.cols = a.rows;
  // counting sort by column over chunks of consecutive rows: each column's
  // entries land chunk after chunk, rows in order -- the serial placement
  const long long hw = host_threads();
  const int chunks = a.nnz() < (1 << 20) ? 1 : static_cast<int>(std::min<long long>(hw, a.rows));
  std::vector<std::vector<int>> pos(chunks, std::vector<int>(a.cols, 0));
  parallel_for(chunks, [&](long long c0, long long c1) {
    for (long long c = c0; c < c1; ++c) {
      const int r0 = static_cast<int>(a.rows * c / chunks), r1 = static_cast<int>(a.rows * (c + 1) / chunks);
      for (int k = a.rp[r0]; k < a.rp[r1]; ++k) pos[c][a.ci[k]]++;
    }
  }, 1);
  t.rp.assign(a.cols + 1, 0);
  for (int col = 0; col < a.cols; ++col) {
    int off = t.rp[col];
    for (int c = 0; c < chunks; ++c) {
      const int n = pos[c][col];
      pos[c][col] = off;  // first slot of chunk c in this column
      off += n;
    }
    t.rp[col + 1] = off;
  }
  t.ci.resize(a.nnz());
  t.v.resize(a.nnz());
  parallel_for(chunks, [&](long long c0, long long c1) {
    for (long long c = c0; c < c1; ++c) {
      const int r0 = static_cast<int>(a.rows * c / chunks), r1 = static_cast<int>(a.rows * (c + 1) / chunks);
      std::vector<int> &next = pos[c];
      for (int i = r0; i < r1; ++i)
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
          const int d = next[a.ci[k]]++;
          t.ci[d] = i;
          t.v[d] = a.v[k];
        }
    }
  }, 1);
  return t;
}

namespace {

// Rows [0, n) of a CSR built in parallel: consecutive rows are grouped into
// chunks, each chunk appends its rows (row(i, scratch, ci, v)) to its own
// buffers with its own scratch (make_scratch()), and the chunks are joined in
// row order. Each row is produced by the same code as a serial loop would run,
// so the result does not depend on the number of threads.
template <typename MakeScratch, typename Row>
void chunked_rows(int n, MakeScratch make_scratch, Row row, std::vector<int> &rp, std::vector<int> &ci,
                  std::vector<double> &v) {
  const long long hw = host_threads();
  const int chunks = n < 8192 ? 1 : static_cast<int>(std::min<long long>(4 * hw, n / 2048));
  struct Part {
    std::vector<int> len, ci;
    std::vector<double> v;
  };
  std::vector<Part> parts(chunks);
  parallel_for(chunks, [&](long long c0, long long c1) {
    auto scratch = make_scratch();
    for (long long c = c0; c < c1; ++c) {
      const int r0 = static_cast<int>(n * c / chunks), r1 = static_cast<int>(n * (c + 1) / chunks);
      Part &pt = parts[c];
      pt.len.reserve(r1 - r0);
      for (int i = r0; i < r1; ++i) {
        const size_t before = pt.ci.size();
        row(i, scratch, pt.ci, pt.v);
        pt.len.push_back(static_cast<int>(pt.ci.size() - before));
      }
    }
  }, 1);
  rp.assign(static_cast<size_t>(n) + 1, 0);
  std::vector<long long> start(chunks + 1, 0);
  int r = 0;
  for (int c = 0; c < chunks; ++c) {
    for (int len : parts[c].len) {
      rp[r + 1] = rp[r] + len;
      ++r;
    }
    start[c + 1] = rp[r];
  }
  ci.resize(rp[n]);
  v.resize(rp[n]);
  parallel_for(chunks, [&](long long c0, long long c1) {
    for (long long c = c0; c < c1; ++c) {
      std::copy(parts[c].ci.begin(), parts[c].ci.end(), ci.begin() + start[c]);
      std::copy(parts[c].v.begin(), parts[c].v.end(), v.begin() + start[c]);
    }
  }, 1);
}

struct RowScratch {
  std::vector<double> acc;
  std::vector<int> mark, cols;
};

}  // namespace

Csr spgemm(const Csr &a, const Csr &b) {
  if (a.cols != b.rows) throw std::runtime_error("spgemm: inner dimensions differ");
  Csr c;
  c.rows = a.rows;
  c.cols = b.cols;
  chunked_rows(
      a.rows, [&] { return RowScratch{std::vector<double>(b.cols, 0.0), std::vector<int>(b.cols, -1), {}}; },
      [&](int i, RowScratch &sc, std::vector<int> &ci, std::vector<double> &v) {
        sc.cols.clear();
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
          const int j = a.ci[k];
          const double av = a.v[k];
          for (int q = b.rp[j]; q < b.rp[j + 1]; ++q) {
            const int col = b.ci[q];
            if (sc.mark[col] != i) {
              sc.mark[col] = i;
              sc.acc[col] = 0.0;
              sc.cols.push_back(col);
            }
            sc.acc[col] += av * b.v[q];
          }
        }
        std::sort(sc.cols.begin(), sc.cols.end());
        for (int col : sc.cols) {
          ci.push_back(col);
          v.push_back(sc.acc[col]);
        }
      },
      c.rp, c.ci, c.v);
  return c;
}

// ---------------------------------------------------------------------------
// colouring, RCM, block graph
// ---------------------------------------------------------------------------
int greedy_coloring(int n, const int *rp, const int *ci, std::vector<int> &colors,
                    std::vector<int> &vertices, std::vector<int> &offsets) {
  colors.assign(n, -1);
  // stamp[c] == v marks colour c as taken by an already coloured neighbour of v
  std::vector<int> stamp(static_cast<std::size_t>(n) + 1, -1);
  int ncolors = 0;
  for (int v = 0; v < n; ++v) {
    for (int k = rp[v]; k < rp[v + 1]; ++k) {
      const int u = ci[k];
      if (u != v && colors[u] >= 0) stamp[colors[u]] = v;
    }
    int c = 0;
    while (stamp[c] == v) ++c;
    colors[v] = c;
    ncolors = std::max(ncolors, c + 1);
  }
  offsets.assign(ncolors + 1, 0);
  for (int v = 0; v < n; ++v) offsets[colors[v] + 1]++;
  for (int c = 0; c < ncolors; ++c) offsets[c + 1] += offsets[c];
  vertices.assign(n, -1);
  std::vector<int> next(offsets.begin(), offsets.end() - 1);
  for (int v = 0; v < n; ++v) vertices[next[colors[v]]++] = v;
  return ncolors;
}

int smallest_last_coloring(int n, const int *rp, const int *ci, std::vector<int> &colors,
                           std::vector<int> &vertices, std::vector<int> &offsets) {
  // degree buckets as doubly linked lists; a bucket's head is its lowest
  // index among the vertices inserted last, so insert in decreasing index
  std::vector<int> deg(n, 0);
  int maxd = 0;
  for (int v = 0; v < n; ++v) {
    for (int k = rp[v]; k < rp[v + 1]; ++k)
      if (ci[k] != v) deg[v]++;
    maxd = std::max(maxd, deg[v]);
  }
  std::vector<int> head(maxd + 1, -1), nxt(n, -1), prv(n, -1);
  const auto insert = [&](int v) {
    const int d = deg[v];
    nxt[v] = head[d];
    prv[v] = -1;
    if (head[d] >= 0) prv[head[d]] = v;
    head[d] = v;
  };
  const auto remove = [&](int v) {
    const int d = deg[v];
    if (prv[v] >= 0) nxt[prv[v]] = nxt[v];
    else head[d] = nxt[v];
    if (nxt[v] >= 0) prv[nxt[v]] = prv[v];
  };
  for (int v = n - 1; v >= 0; --v) insert(v);
  std::vector<char> gone(n, 0);
  std::vector<int> order(n);
  int low = 0;
  for (int i = n - 1; i >= 0; --i) {
    while (head[low] < 0) ++low;
    const int v = head[low];
    remove(v);
    gone[v] = 1;
    order[i] = v;
    for (int k = rp[v]; k < rp[v + 1]; ++k) {
      const int u = ci[k];
      if (u == v || gone[u]) continue;
      remove(u);
      deg[u]--;
      insert(u);
      if (deg[u] < low) low = deg[u];
    }
  }
  colors.assign(n, -1);
  std::vector<int> stamp(static_cast<std::size_t>(n) + 1, -1);
  int ncolors = 0;
  for (int v : order) {
    for (int k = rp[v]; k < rp[v + 1]; ++k) {
      const int u = ci[k];
      if (u != v && colors[u] >= 0) stamp[colors[u]] = v;
    }
    int c = 0;
    while (stamp[c] == v) ++c;
    colors[v] = c;
    ncolors = std::max(ncolors, c + 1);
  }
  offsets.assign(ncolors + 1, 0);
  for (int v = 0; v < n; ++v) offsets[colors[v] + 1]++;
  for (int c = 0; c < ncolors; ++c) offsets[c + 1] += offsets[c];
  vertices.assign(n, -1);
  std::vector<int> next(offsets.begin(), offsets.end() - 1);
  for (int v = 0; v < n; ++v) vertices[next[colors[v]]++] = v;
  return ncolors;
}

namespace {

// The colouring behind relaxed_coloring on a graph with nonnegative edge
// weights w (one per stored entry; the diagonal's is ignored), a strength
// scale sd[i] and a dominance budget mu[i] per vertex: an edge is strong when
// w_ij >= theta sqrt(sd_i sd_j); a vertex must keep its same-colour weight
// below rho mu_i.
int relaxed_weighted(int n, const int *rp, const int *ci, const double *w, const std::vector<double> &sd,
                     const std::vector<double> &mu, double theta, double rho, std::vector<int> &colors,
                     std::vector<int> &vertices, std::vector<int> &offsets) {
  std::vector<int> srp(n + 1, 0), sci;
  sci.reserve(static_cast<size_t>(rp[n]));
  for (int i = 0; i < n; ++i) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = ci[k];
      if (j != i && w[k] >= theta * std::sqrt(sd[i] * sd[j])) sci.push_back(j);
    }
    srp[i + 1] = static_cast<int>(sci.size());
  }
  int nc = greedy_coloring(n, srp.data(), sci.data(), colors, vertices, offsets);
  if (nc > 2) {
    std::vector<int> c2, v2, o2;
    const int n2 = smallest_last_coloring(n, srp.data(), sci.data(), c2, v2, o2);
    if (n2 < nc) nc = n2, colors.swap(c2);
  }
  // repair: no vertex keeps rho mu_i or more of same-colour weight
  std::vector<double> mass;
  std::vector<int> forbid;
  bool clean = false;
  for (int pass = 0; pass < 64 && !clean; ++pass) {
    clean = true;
    for (int i = 0; i < n; ++i) {
      double own = 0.0;
      for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] != i && colors[ci[k]] == colors[i]) own += w[k];
      if (own == 0.0 || own < rho * mu[i]) continue;
      clean = false;
      mass.assign(static_cast<size_t>(nc) + 1, 0.0);
      forbid.assign(static_cast<size_t>(nc) + 1, 0);
      for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] != i) mass[colors[ci[k]]] += w[k];
      for (int k = srp[i]; k < srp[i + 1]; ++k) forbid[colors[sci[k]]] = 1;
      int c = 0;
      while (c < nc && (forbid[c] || (mass[c] > 0.0 && mass[c] >= rho * mu[i]))) ++c;
      colors[i] = c;
      if (c == nc) ++nc;
    }
  }
  if (!clean) return greedy_coloring(n, rp, ci, colors, vertices, offsets);
  // colours that the repair emptied are dropped (renumbered in order)
  std::vector<int> count(nc, 0), renum(nc, -1);
  for (int i = 0; i < n; ++i) count[colors[i]]++;
  int used = 0;
  for (int c = 0; c < nc; ++c)
    if (count[c] > 0) renum[c] = used++;
  for (int i = 0; i < n; ++i) colors[i] = renum[colors[i]];
  nc = used;
  offsets.assign(nc + 1, 0);
  for (int i = 0; i < n; ++i) offsets[colors[i] + 1]++;
  for (int c = 0; c < nc; ++c) offsets[c + 1] += offsets[c];
  vertices.assign(n, -1);
  std::vector<int> next(offsets.begin(), offsets.end() - 1);
  for (int i = 0; i < n; ++i) vertices[next[colors[i]]++] = i;
  return nc;
}

}  // namespace

int relaxed_coloring(int n, const int *rp, const int *ci, const double *v, double theta, double rho,
                     std::vector<int> &colors, std::vector<int> &vertices, std::vector<int> &offsets) {
  std::vector<double> diag(n, 0.0), w(static_cast<size_t>(rp[n]));
  for (int i = 0; i < n; ++i)
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      w[k] = std::fabs(v[k]);
      if (ci[k] == i) diag[i] += w[k];
    }
  return relaxed_weighted(n, rp, ci, w.data(), diag, diag, theta, rho, colors, vertices, offsets);
}

int relaxed_block_coloring(const Csr &a, double theta, double rho, std::vector<int> &colors,
                           std::vector<int> &vertices, std::vector<int> &offsets) {
  if (a.rows % 3 != 0 || a.rows != a.cols) throw std::runtime_error("relaxed_block_coloring: 3x3 blocks expected");
  const int nn = a.rows / 3;
  std::vector<int> grp, gci;
  block_graph(a, 3, grp, gci);
  // squared Frobenius norms of the off-diagonal blocks, in the node graph's
  // order, and the diagonal blocks themselves
  std::vector<double> w(gci.size(), 0.0), dblk(9 * static_cast<size_t>(nn), 0.0);
  for (int r = 0; r < a.rows; ++r) {
    const int I = r / 3;
    for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
      const int J = a.ci[k] / 3;
      if (J == I) {
        dblk[9 * static_cast<size_t>(I) + 3 * (r % 3) + a.ci[k] % 3] += a.v[k];
        continue;
      }
      const int *b = gci.data() + grp[I], *e = gci.data() + grp[I + 1];
      const int *p = std::lower_bound(b, e, J);
      if (p != e && *p == J) w[p - gci.data()] += a.v[k] * a.v[k];
    }
  }
  for (double &x : w) x = std::sqrt(x);
  // strength scale ||A_II||_F; budget 1 / ||A_II^-1||_F <= lambda_min(A_II)
  std::vector<double> sd(nn, 0.0), mu(nn, 0.0);
  for (int I = 0; I < nn; ++I) {
    const double *m = dblk.data() + 9 * static_cast<size_t>(I);
    double f = 0.0;
    for (int q = 0; q < 9; ++q) f += m[q] * m[q];
    sd[I] = std::sqrt(f);
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (!(std::fabs(det) > 0.0)) continue;  // budget 0: the node never shares its colour
    const double inv[9] = {c00, m[2] * m[7] - m[1] * m[8], m[1] * m[5] - m[2] * m[4],
                           c01, m[0] * m[8] - m[2] * m[6], m[2] * m[3] - m[0] * m[5],
                           c02, m[1] * m[6] - m[0] * m[7], m[0] * m[4] - m[1] * m[3]};
    double g = 0.0;
    for (double x : inv) g += (x / det) * (x / det);
    mu[I] = 1.0 / std::sqrt(g);
  }
  // the node graph has no diagonal entries: every entry is an edge
  return relaxed_weighted(nn, grp.data(), gci.data(), w.data(), sd, mu, theta, rho, colors, vertices, offsets);
}

void rcm(int n, const int *rp, const int *ci, int *o2n, int *n2o) {
  std::vector<int> degree(n, 0);
  for (int v = 0; v < n; ++v)
    for (int k = rp[v]; k < rp[v + 1]; ++k)
      if (ci[k] != v) degree[v]++;
  std::vector<char> seen(n, 0);
  std::vector<int> order;
  order.reserve(n);
  std::vector<int> nbr;
  std::queue<int> q;
  const int *deg = degree.data();
  while (static_cast<int>(order.size()) < n) {
    // Cuthill-McKee start: the lowest-numbered unvisited vertex of minimum degree.
    int start = -1, best = 0x7fffffff;
    for (int v = 0; v < n; ++v)
      if (!seen[v] && degree[v] < best) best = degree[v], start = v;
    seen[start] = 1;
    q.push(start);
    while (!q.empty()) {
      const int v = q.front();
      q.pop();
      order.push_back(v);
      nbr.clear();
      for (int k = rp[v]; k < rp[v + 1]; ++k)
        if (ci[k] != v) nbr.push_back(ci[k]);
      // Neighbours by ascending degree. std::sort is not stable: ties keep
      // the order libstdc++'s introsort leaves them in, which is what the
      // reference produces with the same call on the same input sequence.
      std::sort(nbr.begin(), nbr.end(), [deg](int a, int b) { return deg[a] < deg[b]; });
      for (int u : nbr)
        if (!seen[u]) seen[u] = 1, q.push(u);
    }
  }
  for (int i = 0; i < n; ++i) n2o[i] = order[n - 1 - i];
  for (int i = 0; i < n; ++i) o2n[n2o[i]] = i;
}

void block_graph(const Csr &a, int block, std::vector<int> &g_rp, std::vector<int> &g_ci) {
  if (a.rows != a.cols) throw std::runtime_error("buildBlockGraph: matrix must be square.");
  if (a.rows % block != 0)
    throw std::runtime_error("buildBlockGraph: matrix size is not divisible by block size.");
  const int nb = a.rows / block;
  // The node graph is the block pattern of A united with its transpose:
  // out[b] = block columns of block row b, in[b] = block rows that name b;
  // each node's neighbours are the sorted union without itself.
  std::vector<std::vector<int>> out(nb);
  parallel_for(nb, [&](long long b0, long long b1) {
    for (long long b = b0; b < b1; ++b) {
      auto &o = out[b];
      for (long long r = block * b; r < block * (b + 1); ++r)
        for (int k = a.rp[r]; k < a.rp[r + 1]; ++k)
          if (a.ci[k] / block != b) o.push_back(a.ci[k] / block);
      std::sort(o.begin(), o.end());
      o.erase(std::unique(o.begin(), o.end()), o.end());
    }
  }, row_grain(nb, a.nnz()));
  std::vector<int> in_rp(nb + 1, 0);
  for (int b = 0; b < nb; ++b)
    for (int c : out[b]) in_rp[c + 1]++;
  for (int b = 0; b < nb; ++b) in_rp[b + 1] += in_rp[b];
  std::vector<int> in_ci(in_rp[nb]), next(in_rp.begin(), in_rp.end() - 1);
  for (int b = 0; b < nb; ++b)  // rows in increasing order: each in-list comes out sorted
    for (int c : out[b]) in_ci[next[c]++] = b;
  std::vector<int> cnt(nb + 1, 0);
  const auto merge = [&](int b, int *dst) {
    const auto &o = out[b];
    size_t i = 0;
    int j = in_rp[b], m = 0, last = -1;
    while (i < o.size() || j < in_rp[b + 1]) {
      int v;
      if (j >= in_rp[b + 1] || (i < o.size() && o[i] <= in_ci[j])) v = o[i++];
      else v = in_ci[j++];
      if (v == last) continue;
      last = v;
      if (dst != nullptr) dst[m] = v;
      ++m;
    }
    return m;
  };
  parallel_for(nb, [&](long long b0, long long b1) {
    for (long long b = b0; b < b1; ++b) cnt[b + 1] = merge(static_cast<int>(b), nullptr);
  }, 8192);
  g_rp.assign(nb + 1, 0);
  for (int b = 0; b < nb; ++b) g_rp[b + 1] = g_rp[b] + cnt[b + 1];
  g_ci.assign(g_rp[nb], 0);
  parallel_for(nb, [&](long long b0, long long b1) {
    for (long long b = b0; b < b1; ++b) merge(static_cast<int>(b), g_ci.data() + g_rp[b]);
  }, 8192);
}

int block_inverses3x3(const Csr &a, std::vector<double> &dinv) {
  if (a.rows % 3 != 0)
    throw std::runtime_error("3x3 block smoother requires number of DOFs divisible by 3.");
  const int nb = a.rows / 3;
  dinv.assign(9 * static_cast<std::size_t>(nb), 0.0);
  for (int b = 0; b < nb; ++b) {
    double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int lr = 0; lr < 3; ++lr) {
      const int r = 3 * b + lr;
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
        const int c = a.ci[k] - 3 * b;
        if (c >= 0 && c < 3) m[lr][c] = a.v[k];
      }
    }
    // Cholesky of the lower triangle, then the inverse column by column.
    double l[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int j = 0; j < 3; ++j) {
      double d = m[j][j];
      for (int k = 0; k < j; ++k) d -= l[j][k] * l[j][k];
      if (!(d > 0.0)) return b;
      l[j][j] = std::sqrt(d);
      for (int i = j + 1; i < 3; ++i) {
        double s = m[i][j];
        for (int k = 0; k < j; ++k) s -= l[i][k] * l[j][k];
        l[i][j] = s / l[j][j];
      }
    }
    for (int col = 0; col < 3; ++col) {
      double y[3];
      for (int i = 0; i < 3; ++i) {
        double s = (i == col) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s -= l[i][k] * y[k];
        y[i] = s / l[i][i];
      }
      for (int i = 2; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < 3; ++k) s -= l[k][i] * y[k];
        y[i] = s / l[i][i];
      }
      for (int i = 0; i < 3; ++i) dinv[9 * static_cast<std::size_t>(b) + 3 * i + col] = y[i];
    }
  }
  return -1;
}

void expand_block_permutation(int nodes, int block, const int *no2n, const int *nn2o, int *o2n,
                              int *n2o) {
  for (int v = 0; v < nodes; ++v)
    for (int c = 0; c < block; ++c) {
      o2n[block * v + c] = block * no2n[v] + c;
      n2o[block * v + c] = block * nn2o[v] + c;
    }
}

HostEll build_ell(const Csr &a, int width) {
  if (a.rows == 0 || a.cols == 0)
    throw std::runtime_error("HostELLMatrix: matrix dimensions must be nonzero.");
  if (width <= 0) throw std::runtime_error("HostELLMatrix: ELL width must be nonzero.");
  HostEll e;
  e.rows = a.rows;
  e.cols = a.cols;
  e.width = width;
  const std::size_t cells = static_cast<std::size_t>(a.rows) * width;
  e.col.assign(cells, 0);
  e.val.assign(cells, 0.0);
  e.ovf_rp.assign(a.rows + 1, 0);
  for (int r = 0; r < a.rows; ++r) {
    const int len = a.rp[r + 1] - a.rp[r];
    const int in_ell = std::min(width, len);
    for (int s = 0; s < in_ell; ++s) {
      e.col[static_cast<std::size_t>(s) * a.rows + r] = a.ci[a.rp[r] + s];
      e.val[static_cast<std::size_t>(s) * a.rows + r] = a.v[a.rp[r] + s];
    }
    for (int k = a.rp[r] + in_ell; k < a.rp[r + 1]; ++k) {
      e.ovf_ci.push_back(a.ci[k]);
      e.ovf_v.push_back(a.v[k]);
    }
    e.ovf_rp[r + 1] = static_cast<int>(e.ovf_ci.size());
  }
  return e;
}

// ---------------------------------------------------------------------------
// smoothed aggregation
// ---------------------------------------------------------------------------
namespace {

// Node-level coupling strengths: for block size 1 the absolute entries, for
// block size b the Frobenius norm of each b x b block. Off-diagonal
// couplings are returned per node, sorted by neighbour; diag[i] is the
// strength of node i with itself.
void node_couplings(const Csr &a, int block, std::vector<int> &nrp, std::vector<int> &nci,
                    std::vector<double> &nw, std::vector<double> &diag) {
  const int nn = a.rows / block;
  diag.assign(nn, 0.0);
  // per node: (node column, stored position) keys sorted; the node's rows are
  // stored one after the other, so position order is the serial visiting
  // order and each column's squares are summed as a running sum would
  chunked_rows(
      nn, [] { return std::vector<std::pair<int, int>>(); },
      [&](int i, std::vector<std::pair<int, int>> &keys, std::vector<int> &ci, std::vector<double> &w) {
        keys.clear();
        double dsum = 0.0;
        for (int r = block * i; r < block * i + block; ++r)
          for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
            const int j = a.ci[k] / block;
            if (j == i) dsum += a.v[k] * a.v[k];
            else keys.emplace_back(j, k);
          }
        diag[i] = std::sqrt(dsum);
        std::sort(keys.begin(), keys.end());
        for (size_t q = 0; q < keys.size();) {
          const int j = keys[q].first;
          double acc = 0.0;
          for (; q < keys.size() && keys[q].first == j; ++q) acc += a.v[keys[q].second] * a.v[keys[q].second];
          ci.push_back(j);
          w.push_back(std::sqrt(acc));
        }
      },
      nrp, nci, nw);
}

}  // namespace

uint32_t node_priority(uint32_t v) {
  // MurmurHash3's 32-bit finaliser (a bijection, so no two nodes tie)
  v ^= v >> 16;
  v *= 0x85ebca6bu;
  v ^= v >> 13;
  v *= 0xc2b2ae35u;
  v ^= v >> 16;
  return v;
}

namespace {

// Aggregation from a distance-2 maximal independent set of the strength
// graph (Bell, Dalton & Olson, SIAM J. Sci. Comput. 34(4), 2012), the rounds
// a GPU runs, restated serially with the same synchronous updates:
//  * every node carries the key (state << 32 | priority), state 2 root,
//    1 undecided, 0 out (isolated nodes start out);
//  * a round takes, for every node, the largest key over itself and its
//    strong neighbours, twice; an undecided node whose result is its own key
//    becomes a root, one whose result carries state 2 is out;
//  * roots are numbered in index order; each non-root strong neighbour of a
//    root joins the lowest-numbered such root; every other node joins the
//    aggregate of its strongest strongly coupled aggregated neighbour (first
//    in column order on ties); nodes still left become singletons, numbered
//    after the roots in index order.
int mis2_aggregate(int nn, const std::vector<int> &nrp, const std::vector<int> &nci,
                   const std::vector<double> &nw, const std::vector<char> &strong,
                   const std::vector<int> &nstrong, std::vector<int> &agg) {
  std::vector<uint8_t> state(nn);
  for (int i = 0; i < nn; ++i) state[i] = nstrong[i] == 0 ? 0 : 1;
  auto key = [&](int i) { return (static_cast<uint64_t>(state[i]) << 32) | node_priority(static_cast<uint32_t>(i)); };
  std::vector<uint64_t> t1(nn), t2(nn);
  for (;;) {
    bool undecided = false;
    for (int i = 0; i < nn && !undecided; ++i) undecided = state[i] == 1;
    if (!undecided) break;
    // each pass reads only the previous pass's results: the same in parallel
    parallel_for(nn, [&](long long i0, long long i1) {
      for (long long i = i0; i < i1; ++i) {
        uint64_t m = key(static_cast<int>(i));
        for (int k = nrp[i]; k < nrp[i + 1]; ++k)
          if (strong[k]) m = std::max(m, key(nci[k]));
        t1[i] = m;
      }
    });
    parallel_for(nn, [&](long long i0, long long i1) {
      for (long long i = i0; i < i1; ++i) {
        uint64_t m = t1[i];
        for (int k = nrp[i]; k < nrp[i + 1]; ++k)
          if (strong[k]) m = std::max(m, t1[nci[k]]);
        t2[i] = m;
      }
    });
    parallel_for(nn, [&](long long i0, long long i1) {
      for (long long i = i0; i < i1; ++i) {
        if (state[i] != 1) continue;
        if (t2[i] == key(static_cast<int>(i))) state[i] = 2;
        else if ((t2[i] >> 32) == 2) state[i] = 0;
      }
    });
  }
  agg.assign(nn, -1);
  int nagg = 0;
  for (int i = 0; i < nn; ++i) {
    if (nstrong[i] == 0) agg[i] = -2;
    else if (state[i] == 2) agg[i] = nagg++;
  }
  for (int i = 0; i < nn; ++i) {  // roots in index order = in id order
    if (state[i] != 2) continue;
    for (int k = nrp[i]; k < nrp[i + 1]; ++k)
      if (strong[k] && agg[nci[k]] == -1) agg[nci[k]] = agg[i];
  }
  const std::vector<int> agg1 = agg;
  for (int i = 0; i < nn; ++i) {
    if (agg[i] != -1) continue;
    int best = -1;
    double bw = -1.0;
    for (int k = nrp[i]; k < nrp[i + 1]; ++k)
      if (strong[k] && agg1[nci[k]] >= 0 && nw[k] > bw) bw = nw[k], best = agg1[nci[k]];
    if (best >= 0) agg[i] = best;
  }
  for (int i = 0; i < nn; ++i)
    if (agg[i] == -1) agg[i] = nagg++;
  return nagg;
}

}  // namespace

void sa_coarsen(const Csr &a, int block, double eps, std::vector<int> &agg, Csr &p, Csr &r,
                Csr &ac, int aggregation) {
  if (a.rows != a.cols) throw std::runtime_error("sa_coarsen: matrix must be square.");
  if (a.rows % block != 0)
    throw std::runtime_error("SmoothedAggregationCoarsener: matrix size is not divisible by block size.");
  const int nn = a.rows / block;
  std::vector<int> nrp, nci;
  std::vector<double> nw, nd;
  node_couplings(a, block, nrp, nci, nw, nd);

  // Strong couplings: w_ij >= eps * sqrt(d_i d_j), tested squared.
  std::vector<char> strong(nci.size(), 0);
  std::vector<int> nstrong(nn, 0);
  const double eps2 = eps * eps;
  parallel_for(nn, [&](long long i0, long long i1) {
    for (long long i = i0; i < i1; ++i)
      for (int k = nrp[i]; k < nrp[i + 1]; ++k) {
        const int j = nci[k];
        if (nw[k] * nw[k] >= eps2 * nd[i] * nd[j]) strong[k] = 1, nstrong[i]++;
      }
  });

  // Aggregation. -1 unassigned, -2 isolated (no strong neighbour: left out
  // of every aggregate, its prolongator row stays empty).
  int nagg = 0;
  if (aggregation == 1) {
    nagg = mis2_aggregate(nn, nrp, nci, nw, strong, nstrong, agg);
  } else {
  agg.assign(nn, -1);
  for (int i = 0; i < nn; ++i)
    if (nstrong[i] == 0) agg[i] = -2;
  // Step 1: a node whose whole strong neighbourhood is free seeds an
  // aggregate made of itself and that neighbourhood.
  for (int i = 0; i < nn; ++i) {
    if (agg[i] != -1) continue;
    bool free_nbhd = true;
    for (int k = nrp[i]; k < nrp[i + 1] && free_nbhd; ++k)
      if (strong[k] && agg[nci[k]] != -1) free_nbhd = false;
    if (!free_nbhd) continue;
    agg[i] = nagg;
    for (int k = nrp[i]; k < nrp[i + 1]; ++k)
      if (strong[k]) agg[nci[k]] = nagg;
    ++nagg;
  }
  // Step 2: a remaining node joins the step-1 aggregate of its strongest
  // strongly coupled neighbour (first such neighbour on ties).
  const std::vector<int> agg1 = agg;
  for (int i = 0; i < nn; ++i) {
    if (agg[i] != -1) continue;
    int best = -1;
    double bw = -1.0;
    for (int k = nrp[i]; k < nrp[i + 1]; ++k)
      if (strong[k] && agg1[nci[k]] >= 0 && nw[k] > bw) bw = nw[k], best = agg1[nci[k]];
    if (best >= 0) agg[i] = best;
  }
  // Step 3: what is left forms aggregates from its still-free strong
  // neighbourhood.
  for (int i = 0; i < nn; ++i) {
    if (agg[i] != -1) continue;
    agg[i] = nagg;
    for (int k = nrp[i]; k < nrp[i + 1]; ++k)
      if (strong[k] && agg[nci[k]] == -1) agg[nci[k]] = nagg;
    ++nagg;
  }
  }

  // Tentative prolongator: piecewise constant per component, columns
  // normalised (the QR of the constant near-nullspace on each aggregate).
  std::vector<int> size(nagg, 0);
  for (int i = 0; i < nn; ++i)
    if (agg[i] >= 0) size[agg[i]]++;
  const int nc = nagg * block;
  std::vector<double> tval(a.rows, 0.0);  // the one nonzero of each Ptent row
  std::vector<int> tcol(a.rows, -1);
  for (int row = 0; row < a.rows; ++row) {
    const int i = row / block, comp = row % block;
    if (agg[i] >= 0) {
      tcol[row] = agg[i] * block + comp;
      tval[row] = 1.0 / std::sqrt(static_cast<double>(size[agg[i]]));
    }
  }

  // Filtered matrix: weak couplings are dropped and added to the diagonal
  // (row sums preserved). Damping omega = (4/3) / rho, rho bounded by the
  // largest row sum of |D^-1 A_F| (Gershgorin).
  std::vector<char> row_strong_entry(a.nnz(), 0);
  std::vector<double> fdiag(a.rows, 0.0), ratio(a.rows, 0.0);
  parallel_for(a.rows, [&](long long r0, long long r1) {
    for (long long row = r0; row < r1; ++row) {
      const int i = static_cast<int>(row / block);
      double lump = 0.0, d = 0.0;
      for (int k = a.rp[row]; k < a.rp[row + 1]; ++k) {
        const int j = a.ci[k] / block;
        bool keep = (j == i);
        if (!keep) {
          // neighbour j is in node i's sorted coupling list
          const int *b = nci.data() + nrp[i], *e = nci.data() + nrp[i + 1];
          const int *f = std::lower_bound(b, e, j);
          keep = (f != e && *f == j && strong[f - nci.data()]);
        }
        row_strong_entry[k] = keep ? 1 : 0;
        if (a.ci[k] == row) d += a.v[k];
        else if (!keep) lump += a.v[k];
      }
      fdiag[row] = d + lump;
      double s = std::fabs(fdiag[row]);
      for (int k = a.rp[row]; k < a.rp[row + 1]; ++k)
        if (row_strong_entry[k] && a.ci[k] != row) s += std::fabs(a.v[k]);
      if (fdiag[row] != 0.0) ratio[row] = s / std::fabs(fdiag[row]);
    }
  }, row_grain(a.rows, a.nnz()));
  double rho = 0.0;  // a maximum: the same whatever the order
  for (int row = 0; row < a.rows; ++row)
    if (fdiag[row] != 0.0) rho = std::max(rho, ratio[row]);
  const double omega = rho > 0.0 ? (4.0 / 3.0) / rho : 0.0;

  // P = (I - omega D_F^-1 A_F) Ptent, one row at a time, entries of the
  // filtered row in column order (the diagonal taking the lumped value).
  p = Csr();
  p.rows = a.rows;
  p.cols = nc;
  chunked_rows(
      a.rows, [&] { return RowScratch{std::vector<double>(nc, 0.0), std::vector<int>(nc, -1), {}}; },
      [&](int row, RowScratch &sc, std::vector<int> &ci, std::vector<double> &v) {
        sc.cols.clear();
        const double scale = fdiag[row] != 0.0 ? omega / fdiag[row] : 0.0;
        for (int k = a.rp[row]; k < a.rp[row + 1]; ++k) {
          if (!row_strong_entry[k]) continue;
          const int c = a.ci[k];
          if (tcol[c] < 0) continue;
          const double afv = (c == row) ? fdiag[row] : a.v[k];
          const double coef = ((c == row) ? 1.0 : 0.0) - scale * afv;
          const int pc = tcol[c];
          if (sc.mark[pc] != row) sc.mark[pc] = row, sc.acc[pc] = 0.0, sc.cols.push_back(pc);
          sc.acc[pc] += coef * tval[c];
        }
        std::sort(sc.cols.begin(), sc.cols.end());
        for (int c : sc.cols) ci.push_back(c), v.push_back(sc.acc[c]);
      },
      p.rp, p.ci, p.v);
  r = transpose(p);
  ac = spgemm(r, spgemm(a, p));
}

Hierarchy build_hierarchy(const Csr &a, const SaOptions &opt) {
  if (a.rows != a.cols) throw std::runtime_error("AMGHierarchyBuilder: matrix must be square.");
  if (opt.max_levels <= 0) throw std::runtime_error("AMGHierarchyBuilder: maxLevels must be positive.");
  if (opt.min_dofs <= 0) throw std::runtime_error("AMGHierarchyBuilder: minDofs must be positive.");
  if (opt.block <= 0) throw std::runtime_error("block size must be positive.");
  Hierarchy h;
  h.block = opt.block;
  h.A.push_back(a);
  for (int level = 0; level < opt.max_levels; ++level) {
    const Csr &cur = h.A.back();
    if (cur.rows <= opt.min_dofs) break;
    std::vector<int> agg;
    Csr p, r, ac;
    // Strength threshold halved on every coarser level, eps_k = eps_0 / 2^k
    // (Vanek, Mandel & Brezina 1996): Galerkin operators spread their
    // couplings over wider stencils.
    sa_coarsen(cur, opt.block, opt.eps_strong * std::ldexp(1.0, -level), agg, p, r, ac, opt.aggregation);
    // A coarsening that does not shrink the level (or empties it) ends the
    // hierarchy instead of looping.
    if (ac.rows == 0 || ac.rows >= cur.rows) break;
    h.agg.push_back(std::move(agg));
    h.P.push_back(std::move(p));
    h.R.push_back(std::move(r));
    h.A.push_back(std::move(ac));
  }
  return h;
}

// ---------------------------------------------------------------------------
// problem generators
// ---------------------------------------------------------------------------
Csr poisson7(int nx, int ny, int nz) {
  std::vector<double> k(static_cast<std::size_t>(nx) * ny * nz, 1.0);
  Csr a;
  a.rows = a.cols = nx * ny * nz;
  a.rp.assign(a.rows + 1, 0);
  a.ci.reserve(static_cast<std::size_t>(a.rows) * 7);
  a.v.reserve(static_cast<std::size_t>(a.rows) * 7);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const int i = (z * ny + y) * nx + x;
        auto add = [&](int j, double val) { a.ci.push_back(j), a.v.push_back(val); };
        if (z > 0) add(i - nx * ny, -1.0);
        if (y > 0) add(i - nx, -1.0);
        if (x > 0) add(i - 1, -1.0);
        add(i, 6.0);
        if (x + 1 < nx) add(i + 1, -1.0);
        if (y + 1 < ny) add(i + nx, -1.0);
        if (z + 1 < nz) add(i + nx * ny, -1.0);
        a.rp[i + 1] = static_cast<int>(a.ci.size());
      }
  return a;
}

Csr varcoef7(int nx, int ny, int nz, const std::vector<double> &k) {
  const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
  if (k.size() != n) throw std::runtime_error("varcoef7: coefficient array size mismatch");
  Csr a;
  a.rows = a.cols = static_cast<int>(n);
  a.rp.assign(n + 1, 0);
  a.ci.reserve(n * 7);
  a.v.reserve(n * 7);
  // 2 (p q) / (p + q): symmetric in p and q bit for bit
  auto harm = [](double p, double q) { return 2.0 * (p * q) / (p + q); };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const int i = (z * ny + y) * nx + x;
        const double ki = k[i];
        double diag = 0.0;
        double off[6];
        int offc[6];
        int m = 0;
        auto face = [&](bool inside, int j) {
          if (inside) {
            const double t = harm(ki, k[j]);
            diag += t;
            off[m] = -t;
            offc[m] = j;
            ++m;
          } else {
            diag += 2.0 * ki;
          }
        };
        face(z > 0, i - nx * ny);
        face(y > 0, i - nx);
        face(x > 0, i - 1);
        face(x + 1 < nx, i + 1);
        face(y + 1 < ny, i + nx);
        face(z + 1 < nz, i + nx * ny);
        // emit in ascending column order: the three lower neighbours, the
        // diagonal, then the three upper neighbours
        int q = 0;
        for (; q < m && offc[q] < i; ++q) a.ci.push_back(offc[q]), a.v.push_back(off[q]);
        a.ci.push_back(i), a.v.push_back(diag);
        for (; q < m; ++q) a.ci.push_back(offc[q]), a.v.push_back(off[q]);
        a.rp[i + 1] = static_cast<int>(a.ci.size());
      }
  return a;
}

std::vector<double> grf_coefficients(int nx, int ny, int nz, double corr, double sigma,
                                     uint64_t seed) {
  const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
  SplitMix64 rng(seed);
  std::vector<double> f(n), g(n);
  for (std::size_t i = 0; i < n; ++i) f[i] = rng.normal();
  const double s = corr / std::sqrt(2.0);
  const int rad = static_cast<int>(std::ceil(4.0 * s));
  std::vector<double> w(2 * rad + 1);
  for (int d = -rad; d <= rad; ++d) w[d + rad] = std::exp(-0.5 * d * d / (s * s));
  auto pass = [&](int axis) {
    const int dims[3] = {nx, ny, nz};
    const int len = dims[axis];
    const std::size_t stride = axis == 0 ? 1 : (axis == 1 ? static_cast<std::size_t>(nx)
                                                          : static_cast<std::size_t>(nx) * ny);
    for (std::size_t i = 0; i < n; ++i) {
      const int c = static_cast<int>((i / stride) % len);
      const std::size_t base = i - static_cast<std::size_t>(c) * stride;
      double acc = 0.0;
      for (int d = -rad; d <= rad; ++d) {
        int cc = (c + d) % len;
        if (cc < 0) cc += len;
        acc += w[d + rad] * f[base + static_cast<std::size_t>(cc) * stride];
      }
      g[i] = acc;
    }
    f.swap(g);
  };
  pass(0);
  pass(1);
  pass(2);
  double mean = 0.0, var = 0.0;
  for (double x : f) mean += x;
  mean /= static_cast<double>(n);
  for (double x : f) var += (x - mean) * (x - mean);
  const double sd = std::sqrt(var / static_cast<double>(n));
  std::vector<double> k(n);
  for (std::size_t i = 0; i < n; ++i) k[i] = std::exp(sigma * (f[i] - mean) / sd);
  return k;
}

std::vector<double> loguniform_coefficients(int n, double lo, double hi, uint64_t seed) {
  SplitMix64 rng(seed);
  std::vector<double> k(n);
  const double a = std::log(lo), b = std::log(hi);
  for (int i = 0; i < n; ++i) k[i] = std::exp(rng.uniform(a, b));
  return k;
}

std::vector<double> uniform_rhs(int n, uint64_t seed) {
  SplitMix64 rng(seed);
  std::vector<double> b(n);
  for (int i = 0; i < n; ++i) b[i] = rng.uniform(-1.0, 1.0);
  return b;
}

namespace {

// The six Kuhn tetrahedra of a unit cube share the diagonal 000-111; for
// each ordering (a, b, c) of the axes the tetrahedron is
// {0, e_a, e_a + e_b, e_a + e_b + e_c}. Returned as corner bit masks
// (bit 0 = x, bit 1 = y, bit 2 = z).
void kuhn_corners(int t, int corner[4]) {
  static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  corner[0] = 0;
  corner[1] = 1 << perm[t][0];
  corner[2] = corner[1] | (1 << perm[t][1]);
  corner[3] = 7;
}

// Gradients of the four P1 basis functions of tetrahedron p[4][3]; returns
// the volume.
double p1_gradients(const double p[4][3], double g[4][3]) {
  double j[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) j[r][c] = p[c + 1][r] - p[0][r];  // columns p_i - p_0
  const double det = j[0][0] * (j[1][1] * j[2][2] - j[1][2] * j[2][1]) -
                     j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
                     j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]);
  double inv[3][3];
  inv[0][0] = (j[1][1] * j[2][2] - j[1][2] * j[2][1]) / det;
  inv[0][1] = (j[0][2] * j[2][1] - j[0][1] * j[2][2]) / det;
  inv[0][2] = (j[0][1] * j[1][2] - j[0][2] * j[1][1]) / det;
  inv[1][0] = (j[1][2] * j[2][0] - j[1][0] * j[2][2]) / det;
  inv[1][1] = (j[0][0] * j[2][2] - j[0][2] * j[2][0]) / det;
  inv[1][2] = (j[0][2] * j[1][0] - j[0][0] * j[1][2]) / det;
  inv[2][0] = (j[1][0] * j[2][1] - j[1][1] * j[2][0]) / det;
  inv[2][1] = (j[0][1] * j[2][0] - j[0][0] * j[2][1]) / det;
  inv[2][2] = (j[0][0] * j[1][1] - j[0][1] * j[1][0]) / det;
  // grad lambda_{i+1} = row i of J^-1
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) g[i + 1][d] = inv[i][d];
  for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
  return std::fabs(det) / 6.0;
}

// Offsets between two vertices of a Kuhn mesh are (dx, dy, dz) with all
// nonzero components of one sign: 15 possibilities (including zero). The
// slot table is indexed by (dx+1) + 3 (dy+1) + 9 (dz+1).
struct KuhnStencil {
  int slot_of[27];
  int off[15][3];
  KuhnStencil() {
    int n = 0;
    for (int i = 0; i < 27; ++i) slot_of[i] = -1;
    // ascending linear offset dz * big + dy * mid + dx
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const bool neg = dx < 0 || dy < 0 || dz < 0;
          const bool pos = dx > 0 || dy > 0 || dz > 0;
          if (neg && pos) continue;
          slot_of[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] = n;
          off[n][0] = dx, off[n][1] = dy, off[n][2] = dz;
          ++n;
        }
  }
  int slot(int dx, int dy, int dz) const { return slot_of[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)]; }
};

}  // namespace

Csr kuhn_laplacian(int m, double jitter, uint64_t seed) {
  if (m < 2) throw std::runtime_error("kuhn_laplacian: need at least 2 cells per side");
  const int nv = m + 1, ni = m - 1;
  const double h = 1.0 / m;
  std::vector<double> xyz(3 * static_cast<std::size_t>(nv) * nv * nv);
  SplitMix64 rng(seed);
  for (int z = 0; z < nv; ++z)
    for (int y = 0; y < nv; ++y)
      for (int x = 0; x < nv; ++x) {
        const std::size_t v = (static_cast<std::size_t>(z) * nv + y) * nv + x;
        double p[3] = {x * h, y * h, z * h};
        const bool interior = x > 0 && x < m && y > 0 && y < m && z > 0 && z < m;
        if (interior)
          for (int d = 0; d < 3; ++d) p[d] += rng.uniform(-jitter * h, jitter * h);
        for (int d = 0; d < 3; ++d) xyz[3 * v + d] = p[d];
      }
  auto unknown = [&](int x, int y, int z) -> int {
    if (x <= 0 || x >= m || y <= 0 || y >= m || z <= 0 || z >= m) return -1;
    return ((z - 1) * ni + (y - 1)) * ni + (x - 1);
  };
  static const KuhnStencil st;
  const std::size_t n = static_cast<std::size_t>(ni) * ni * ni;
  std::vector<double> acc(n * 15, 0.0);
  std::vector<char> used(n * 15, 0);
  for (int cz = 0; cz < m; ++cz)
    for (int cy = 0; cy < m; ++cy)
      for (int cx = 0; cx < m; ++cx)
        for (int t = 0; t < 6; ++t) {
          int corner[4];
          kuhn_corners(t, corner);
          int vx[4], vy[4], vz[4];
          double p[4][3], g[4][3];
          for (int a = 0; a < 4; ++a) {
            vx[a] = cx + (corner[a] & 1);
            vy[a] = cy + ((corner[a] >> 1) & 1);
            vz[a] = cz + ((corner[a] >> 2) & 1);
            const std::size_t v = (static_cast<std::size_t>(vz[a]) * nv + vy[a]) * nv + vx[a];
            for (int d = 0; d < 3; ++d) p[a][d] = xyz[3 * v + d];
          }
          const double vol = p1_gradients(p, g);
          for (int a = 0; a < 4; ++a) {
            const int ia = unknown(vx[a], vy[a], vz[a]);
            if (ia < 0) continue;
            for (int b = 0; b < 4; ++b) {
              if (unknown(vx[b], vy[b], vz[b]) < 0) continue;
              const int s = st.slot(vx[b] - vx[a], vy[b] - vy[a], vz[b] - vz[a]);
              const double kab = vol * (g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2]);
              acc[static_cast<std::size_t>(ia) * 15 + s] += kab;
              used[static_cast<std::size_t>(ia) * 15 + s] = 1;
            }
          }
        }
  Csr a;
  a.rows = a.cols = static_cast<int>(n);
  a.rp.assign(n + 1, 0);
  for (int z = 1; z < m; ++z)
    for (int y = 1; y < m; ++y)
      for (int x = 1; x < m; ++x) {
        const int i = unknown(x, y, z);
        for (int s = 0; s < 15; ++s) {
          if (!used[static_cast<std::size_t>(i) * 15 + s]) continue;
          const int j = unknown(x + st.off[s][0], y + st.off[s][1], z + st.off[s][2]);
          a.ci.push_back(j);
          a.v.push_back(acc[static_cast<std::size_t>(i) * 15 + s]);
        }
        a.rp[i + 1] = static_cast<int>(a.ci.size());
      }
  return a;
}

Csr elasticity_p1(int v, double nu, uint64_t seed, std::vector<double> &rhs) {
  if (v < 2) throw std::runtime_error("elasticity_p1: need at least 2 vertices per side");
  const int m = v - 1;
  const double h = 1.0 / m;
  // unknown vertices: x index 1..m (the x = 0 face is clamped)
  auto unknown = [&](int x, int y, int z) -> int {
    if (x <= 0 || x > m || y < 0 || y > m || z < 0 || z > m) return -1;
    return (z * v + y) * m + (x - 1);
  };
  static const KuhnStencil st;
  const std::size_t nvu = static_cast<std::size_t>(m) * v * v;
  std::vector<double> acc(nvu * 15 * 9, 0.0);
  std::vector<char> used(nvu * 15, 0);
  rhs.assign(3 * nvu, 0.0);
  SplitMix64 rng(seed);
  for (int cz = 0; cz < m; ++cz)
    for (int cy = 0; cy < m; ++cy)
      for (int cx = 0; cx < m; ++cx)
        for (int t = 0; t < 6; ++t) {
          const double young = std::exp(rng.normal());
          const double lam = young * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
          const double mu = young / (2.0 * (1.0 + nu));
          int corner[4];
          kuhn_corners(t, corner);
          int vx[4], vy[4], vz[4];
          double p[4][3], g[4][3];
          for (int a = 0; a < 4; ++a) {
            vx[a] = cx + (corner[a] & 1);
            vy[a] = cy + ((corner[a] >> 1) & 1);
            vz[a] = cz + ((corner[a] >> 2) & 1);
            p[a][0] = vx[a] * h, p[a][1] = vy[a] * h, p[a][2] = vz[a] * h;
          }
          const double vol = p1_gradients(p, g);
          for (int a = 0; a < 4; ++a) {
            const int ia = unknown(vx[a], vy[a], vz[a]);
            if (ia < 0) continue;
            rhs[3 * static_cast<std::size_t>(ia) + 2] += -vol / 4.0;  // unit body force in -z
            for (int b = 0; b < 4; ++b) {
              if (unknown(vx[b], vy[b], vz[b]) < 0) continue;
              const int s = st.slot(vx[b] - vx[a], vy[b] - vy[a], vz[b] - vz[a]);
              const double gg = g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2];
              double *blk = &acc[(static_cast<std::size_t>(ia) * 15 + s) * 9];
              for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                  blk[3 * i + j] += vol * (lam * g[a][i] * g[b][j] + mu * g[b][i] * g[a][j] +
                                           (i == j ? mu * gg : 0.0));
              used[static_cast<std::size_t>(ia) * 15 + s] = 1;
            }
          }
        }
  Csr a;
  a.rows = a.cols = static_cast<int>(3 * nvu);
  a.rp.assign(a.rows + 1, 0);
  for (int z = 0; z <= m; ++z)
    for (int y = 0; y <= m; ++y)
      for (int x = 1; x <= m; ++x) {
        const int iv = unknown(x, y, z);
        for (int i = 0; i < 3; ++i) {
          const int row = 3 * iv + i;
          for (int s = 0; s < 15; ++s) {
            if (!used[static_cast<std::size_t>(iv) * 15 + s]) continue;
            const int jv = unknown(x + st.off[s][0], y + st.off[s][1], z + st.off[s][2]);
            const double *blk = &acc[(static_cast<std::size_t>(iv) * 15 + s) * 9];
            for (int j = 0; j < 3; ++j) {
              a.ci.push_back(3 * jv + j);
              a.v.push_back(blk[3 * i + j]);
            }
          }
          a.rp[row + 1] = static_cast<int>(a.ci.size());
        }
      }
  return a;
}

void hierarchical_reordering(const Hierarchy &h, std::vector<std::vector<int>> &o2n,
                             std::vector<std::vector<int>> &n2o) {
  const int L = static_cast<int>(h.A.size());
  if (L == 0) throw std::runtime_error("HierarchicalReordering: empty hierarchy.");
  if (static_cast<int>(h.R.size()) + 1 != L)
    throw std::runtime_error("HierarchicalReordering: expected one restriction matrix between consecutive levels.");
  o2n.assign(L, {});
  n2o.assign(L, {});
  auto own_rcm = [&](int k, std::vector<int> &a, std::vector<int> &b) {
    const Csr &m = h.A[k];
    a.resize(m.rows);
    b.resize(m.rows);
    rcm(m.rows, m.rp.data(), m.ci.data(), a.data(), b.data());
  };
  own_rcm(L - 1, o2n[L - 1], n2o[L - 1]);
  for (int f = L - 2; f >= 0; --f) {
    const Csr &A = h.A[f], &R = h.R[f];
    if (A.rows != A.cols) throw std::runtime_error("HierarchicalReordering: fine matrix must be square.");
    if (R.cols != A.rows)
      throw std::runtime_error("HierarchicalReordering: restriction dimensions do not match fine matrix.");
    const int nf = A.rows, nc = R.rows;
    // strongest parent of every fine row, weights compared in FP32
    std::vector<int> parent(nf, -1);
    std::vector<float> best(nf, -1.0f);
    for (int c = 0; c < nc; ++c)
      for (int e = R.rp[c]; e < R.rp[c + 1]; ++e) {
        const int fine = R.ci[e];
        const float w = std::fabs(static_cast<float>(R.v[e]));
        if (w > best[fine]) best[fine] = w, parent[fine] = c;
      }
    std::vector<int> frcm_o2n, frcm_n2o;
    own_rcm(f, frcm_o2n, frcm_n2o);
    const std::vector<int> &crank = o2n[f + 1];
    // keys (parent rank, own RCM rank) are unique, so the order is total
    std::vector<int> order(nf);
    for (int i = 0; i < nf; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
      const int pa = parent[a] >= 0 ? crank[parent[a]] : nc;
      const int pb = parent[b] >= 0 ? crank[parent[b]] : nc;
      if (pa != pb) return pa < pb;
      return frcm_o2n[a] < frcm_o2n[b];
    });
    n2o[f] = order;
    o2n[f].assign(nf, 0);
    for (int i = 0; i < nf; ++i) o2n[f][order[i]] = i;
  }
}

}  // namespace gsb
