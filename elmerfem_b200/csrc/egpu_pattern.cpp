// egpu_pattern.cpp -- CreateMatrix (ElementUtils.src:698-930) for meshes whose nodes
// are all active, and the element colouring used by the device assembly.
//
// Elmer builds the node graph as per-row linked lists kept sorted by column
// (List_GetMatrixIndex, ListMatrix.src:263-320), so the list of row i is exactly the
// ascending set of nodes sharing an element with i.  Here that set is held in CSR
// form; OptimizeBandwidth (BandwidthOptimize.src:108-355) walks it in the same order,
// which gives the same Perm, Rows, Cols and Diag.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/elmergpu.h"

namespace {

struct Graph {
  int n = 0;
  std::vector<long long> start;  // n+1
  std::vector<int> adj;          // 1-based node ids, ascending per row
};

// MakeListMatrix, ElementUtils.src:424-498 (node pairs of every element)
Graph node_graph(int nnodes, int nelem, int nen, const int *elem) {
  // node -> element incidence
  std::vector<int> cnt(nnodes + 1, 0);
  for (long long k = 0; k < (long long)nelem * nen; ++k) cnt[elem[k]]++;
  std::vector<long long> inc_start(nnodes + 1, 0);
  for (int i = 0; i < nnodes; ++i) inc_start[i + 1] = inc_start[i] + cnt[i + 1];
  std::vector<int> inc(inc_start[nnodes]);
  std::vector<long long> fill(inc_start.begin(), inc_start.end() - 1);
  for (int e = 0; e < nelem; ++e)
    for (int p = 0; p < nen; ++p) inc[fill[elem[(size_t)e * nen + p] - 1]++] = e;
  Graph g;
  g.n = nnodes;
  std::vector<std::vector<int>> rows_tmp(nnodes);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < nnodes; ++i) {
      buf.clear();
      for (long long k = inc_start[i]; k < inc_start[i + 1]; ++k) {
        const int *en = elem + (size_t)inc[k] * nen;
        for (int p = 0; p < nen; ++p) buf.push_back(en[p]);
      }
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
      rows_tmp[i] = buf;
    }
  }
  g.start.assign(nnodes + 1, 0);
  for (int i = 0; i < nnodes; ++i) g.start[i + 1] = g.start[i] + (long long)rows_tmp[i].size();
  g.adj.resize(g.start[nnodes]);
  for (int i = 0; i < nnodes; ++i) std::copy(rows_tmp[i].begin(), rows_tmp[i].end(), g.adj.begin() + g.start[i]);
  return g;
}

int bandwidth(const Graph &g, const int *reorder) {
  int hbw = 0;
  for (int i = 1; i <= g.n; ++i)
    for (long long p = g.start[i - 1]; p < g.start[i]; ++p) {
      const int k = g.adj[p];
      const int d = reorder ? std::abs(reorder[i - 1] - reorder[k - 1]) : std::abs(i - k);
      hbw = std::max(hbw, d);
    }
  return hbw;
}

struct Walker {
  const Graph &g;
  std::vector<int> level;
  std::vector<char> done;
  int max_level = 0;
  explicit Walker(const Graph &gg) : g(gg), level(gg.n, 0), done(gg.n, 0) {}
  int degree(int i) const { return (int)(g.start[i] - g.start[i - 1]); }

  // Levelize (BandwidthOptimize.src:290-350); a list position is (row, index into adj)
  void levelize(int nin, int lin) {
    struct Pos {
      int row;
      long long p;
    };
    std::vector<Pos> stack;
    stack.reserve(512);
    int n = nin, lev = lin;
    auto valid = [&](const Pos &q) { return q.p >= 0 && q.p < g.start[q.row]; };
    Pos p{n, g.start[n - 1]};
    if (!valid(p)) p.p = -1;
    while (p.p >= 0) {
      stack.push_back(p);
      level[n - 1] = lev;
      done[n - 1] = 1;
      max_level = std::max(max_level, lev);
      p = Pos{n, g.start[n - 1]};
      if (!valid(p)) p.p = -1;
      while (true) {
        if (p.p >= 0) {
          const int m = g.adj[p.p];
          if (m <= g.n && !done[m - 1]) {
            n = m;
            lev++;
            break;
          }
        } else if (!stack.empty()) {
          p = stack.back();
          lev--;
          stack.pop_back();
        } else {
          break;
        }
        p.p = (p.p + 1 < g.start[p.row]) ? p.p + 1 : -1;
      }
    }
  }
};

// OptimizeBandwidth, BandwidthOptimize.src:108-262
void optimize_bandwidth(const Graph &g, std::vector<int> &perm, bool optimize, bool use_always) {
  const int n = g.n;
  const int hbw_before = bandwidth(g, nullptr) + 1;
  if (!optimize) return;
  Walker w(g);
  int start = 1, min_degree = w.degree(1);
  for (int i = 1; i <= n; ++i) {
    if (w.degree(i) < min_degree) {
      start = i;
      min_degree = w.degree(i);
    }
    w.level[i - 1] = 0;
  }
  w.max_level = 0;
  std::fill(w.done.begin(), w.done.end(), 0);
  w.levelize(start, 0);
  bool new_root = true;
  while (new_root) {
    new_root = false;
    min_degree = w.degree(start);
    int k = start;
    for (int i = 1; i <= n; ++i)
      if (w.level[i - 1] == w.max_level && w.degree(i) < min_degree) {
        k = i;
        min_degree = w.degree(i);
      }
    if (k != start) {
      const int j = w.max_level;
      w.max_level = 0;
      std::fill(w.done.begin(), w.done.end(), 0);
      w.levelize(k, 0);
      if (j > w.max_level) {
        new_root = true;
        start = j;  // as written at BandwidthOptimize.src:190
      }
    }
  }
  // Cuthill-McKee numbering in list order, then reversed (:199-233)
  std::vector<int> order(n, 0), done_index(n, 0);
  int indx = 1;
  order[0] = start;
  done_index[start - 1] = indx++;
  for (int i = 1; i <= n; ++i) {
    if (order[i - 1] == 0) {
      for (int j = 1; j <= n; ++j)
        if (done_index[j - 1] == 0) {
          order[indx - 1] = j;
          done_index[j - 1] = indx++;
          break;
        }
    }
    const int r = order[i - 1];
    for (long long p = g.start[r - 1]; p < g.start[r]; ++p) {
      const int k = g.adj[p];
      if (k <= n && done_index[k - 1] == 0) {
        order[indx - 1] = k;
        done_index[k - 1] = indx++;
      }
    }
  }
  std::vector<int> rev(n);
  for (int i = 1; i <= n; ++i) rev[order[i - 1] - 1] = n - i + 1;
  std::vector<int> saved = perm;
  for (int i = 0; i < n; ++i) perm[i] = saved[i] > 0 ? rev[saved[i] - 1] : 0;
  const int hbw_after = bandwidth(g, perm.data()) + 1;
  if (hbw_before < hbw_after && !use_always) perm = saved;  // rejection rule (:251-257)
}

struct Cached {
  int nnodes = -1, nelem = -1, nen = -1, dofs = -1, opt = -1;
  const int *src = nullptr;
  uint64_t sig = 0;
  std::vector<int> perm, rows, cols, diag;
};
std::mutex g_mu;
Cached g_last;

uint64_t signature(const int *a, long long n) {
  uint64_t h = 1469598103934665603ull;
  const long long step = std::max(1LL, n / 4096);
  for (long long i = 0; i < n; i += step) h = (h ^ (uint64_t)(uint32_t)a[i]) * 1099511628211ull;
  return h ^ (uint64_t)n;
}

void build(int nnodes, int nelem, int nen, const int *elem, int dofs, int opt, Cached &out) {
  Graph g = node_graph(nnodes, nelem, nen, elem);
  std::vector<int> perm(nnodes);
  for (int i = 0; i < nnodes; ++i) perm[i] = i + 1;
  optimize_bandwidth(g, perm, opt != 0, false);
  const int n = dofs * nnodes;
  // CRS_CreateMatrix (CRSMatrix.src:816-875) + InitializeMatrix (ElementUtils.src:625-660)
  // + CRS_SortMatrix (CRSMatrix.src:168-232): row r of node i holds, for every neighbour
  // c, the DOF block of Perm(c), sorted ascending.
  std::vector<int> inv(nnodes);
  for (int i = 0; i < nnodes; ++i) inv[perm[i] - 1] = i;
  out.rows.assign(n + 1, 0);
  out.rows[0] = 1;
  for (int r = 0; r < n; ++r) {
    const int node = inv[r / dofs];
    out.rows[r + 1] = out.rows[r] + dofs * (int)(g.start[node + 1] - g.start[node]);
  }
  out.cols.assign((size_t)out.rows[n] - 1, 0);
  out.diag.assign(n, 0);
#pragma omp parallel
  {
    std::vector<int> nb;
#pragma omp for schedule(dynamic, 1024)
    for (int node = 0; node < nnodes; ++node) {
      nb.clear();
      for (long long p = g.start[node]; p < g.start[node + 1]; ++p) nb.push_back(perm[g.adj[p] - 1]);
      std::sort(nb.begin(), nb.end());
      for (int l = 1; l <= dofs; ++l) {
        const int row = dofs * (perm[node] - 1) + l;  // 1-based
        long long k = out.rows[row - 1] - 1;
        for (int c : nb)
          for (int m = 1; m <= dofs; ++m) {
            const int col = dofs * (c - 1) + m;
            out.cols[k] = col;
            if (col == row) out.diag[row - 1] = (int)k + 1;
            ++k;
          }
      }
    }
  }
  out.perm = std::move(perm);
}

}  // namespace

extern "C" int egpu_pattern_create(int nnodes, int nelem, int nen, const int *elem_nodes, int dofs,
                                   int optimize_bw, int *n_out, long long *nnz_out, int *perm, int *rows,
                                   int *cols, int *diag) {
  if (nnodes <= 0 || nelem <= 0 || nen <= 0 || nen > 27 || !elem_nodes || dofs < 1 || dofs > 8)
    return EGPU_ERR_ARG;
  for (long long k = 0; k < (long long)nelem * nen; ++k)
    if (elem_nodes[k] < 1 || elem_nodes[k] > nnodes) return EGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  const uint64_t sig = signature(elem_nodes, (long long)nelem * nen);
  Cached &c = g_last;
  if (!(c.nnodes == nnodes && c.nelem == nelem && c.nen == nen && c.dofs == dofs && c.opt == optimize_bw &&
        c.src == elem_nodes && c.sig == sig)) {
    Cached fresh;
    build(nnodes, nelem, nen, elem_nodes, dofs, optimize_bw, fresh);
    fresh.nnodes = nnodes;
    fresh.nelem = nelem;
    fresh.nen = nen;
    fresh.dofs = dofs;
    fresh.opt = optimize_bw;
    fresh.src = elem_nodes;
    fresh.sig = sig;
    c = std::move(fresh);
  }
  const int n = dofs * nnodes;
  if (n_out) *n_out = n;
  if (nnz_out) *nnz_out = (long long)c.cols.size();
  if (perm) std::memcpy(perm, c.perm.data(), nnodes * sizeof(int));
  if (rows) std::memcpy(rows, c.rows.data(), (n + 1) * sizeof(int));
  if (cols) std::memcpy(cols, c.cols.data(), c.cols.size() * sizeof(int));
  if (diag) std::memcpy(diag, c.diag.data(), n * sizeof(int));
  return EGPU_OK;
}

// Greedy first-fit colouring in element order: elements sharing a node get different
// colours.  Returns the number of colours; color_of[e] in [0, ncolors).
int egpu_color_elements(int nnodes, int nelem, int nen, const int *elem_nodes, std::vector<int> &color_of) {
  std::vector<uint64_t> used(nnodes, 0);
  std::vector<std::vector<uint64_t>> more;  // beyond 64 colours (unstructured meshes)
  color_of.assign(nelem, 0);
  int ncol = 0;
  for (int e = 0; e < nelem; ++e) {
    const int *en = elem_nodes + (size_t)e * nen;
    uint64_t forb = 0;
    for (int p = 0; p < nen; ++p) forb |= used[en[p] - 1];
    int c = 0;
    if (forb != ~0ull) {
      c = __builtin_ctzll(~forb);
    } else {
      // first colour >= 64 unused at all nodes
      int cc = 64;
      while (true) {
        const size_t w = cc / 64 - 1, b = cc % 64;
        bool clash = false;
        for (int p = 0; p < nen && !clash; ++p) {
          auto &m = more;
          if (m.size() > w && (m[w][en[p] - 1] >> b & 1ull)) clash = true;
        }
        if (!clash) break;
        ++cc;
      }
      c = cc;
    }
    color_of[e] = c;
    ncol = std::max(ncol, c + 1);
    if (c < 64) {
      for (int p = 0; p < nen; ++p) used[en[p] - 1] |= 1ull << c;
    } else {
      const size_t w = c / 64 - 1;
      while (more.size() <= w) more.emplace_back(nnodes, 0ull);
      for (int p = 0; p < nen; ++p) more[w][en[p] - 1] |= 1ull << (c % 64);
    }
  }
  return ncol;
}

// ---------------------------------------------------------------------------------------
// ILU(n) structure.  CRS_IncompleteLU(A, n > 0) (CRSMatrix.src:2196-2218) applies
// InitializeILU1 (:2391-2497) n times: row i of the next structure holds row i's entries
// plus, for every entry k < i that row i had before this step, the entries of row k to the
// right of its diagonal.  Each step here: a per-row union over those upper parts (rows in
// parallel), counted first and then written, columns ascending.
namespace {

void ilu_fill_step(int n, const std::vector<int> &rows, const std::vector<int> &cols, const std::vector<int> &diag,
                   std::vector<int> &orows, std::vector<int> &ocols, std::vector<int> &odiag) {
  std::vector<int> cnt(n + 1, 0);
  auto row_union = [&](int i, std::vector<int> &mark, std::vector<int> &out) {
    out.clear();
    for (int e = rows[i]; e < rows[i + 1]; ++e) {
      mark[cols[e]] = i + 1;
      out.push_back(cols[e]);
    }
    for (int e = rows[i]; e < diag[i]; ++e) {  // entries k < i of the input structure
      const int k = cols[e];
      for (int l = diag[k] + 1; l < rows[k + 1]; ++l) {
        const int j = cols[l];
        if (mark[j] != i + 1) {
          mark[j] = i + 1;
          out.push_back(j);
        }
      }
    }
    std::sort(out.begin(), out.end());
  };
#pragma omp parallel
  {
    std::vector<int> mark(n, 0), out;
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      row_union(i, mark, out);
      cnt[i + 1] = (int)out.size();
    }
  }
  orows.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) orows[i + 1] = orows[i] + cnt[i + 1];
  ocols.assign(orows[n], 0);
  odiag.assign(n, -1);
#pragma omp parallel
  {
    std::vector<int> mark(n, 0), out;
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      row_union(i, mark, out);
      for (size_t t = 0; t < out.size(); ++t) {
        ocols[orows[i] + t] = out[t];
        if (out[t] == i) odiag[i] = orows[i] + (int)t;
      }
    }
  }
}

}  // namespace

// 0-based input and output; order 0 returns the input structure
void egpu_ilu_structure(int n, const std::vector<int> &rows, const std::vector<int> &cols,
                        const std::vector<int> &diag, int order, std::vector<int> &orows, std::vector<int> &ocols,
                        std::vector<int> &odiag) {
  orows = rows;
  ocols = cols;
  odiag = diag;
  for (int step = 0; step < order; ++step) {
    std::vector<int> r, c, d;
    ilu_fill_step(n, orows, ocols, odiag, r, c, d);
    orows.swap(r);
    ocols.swap(c);
    odiag.swap(d);
  }
}

// Threshold ILU (CRS_ILUT, CRSMatrix.src:2849-3044), 0-based, on the host: the factor's
// pattern depends on its values, so it is computed row after row as the reference does and
// the device then runs the triangular solves on the result.  Row i: the matrix row is
// scattered into the dense row w; its flagged columns left of the diagonal are eliminated in
// ascending order (a min-heap holds them, fill included), w_k /= u_kk (U diagonals are
// still un-inverted here), then w_j -= w_k * U_kj over ILU row k's U part, flagging new fill
// whether or not w_k is zero, as the reference does.  The finished row keeps the entries
// with |w_k| >= tol * ||A(i,:)||_2, and the diagonal, in ascending column order.  Finally the
// U diagonal is inverted (1 where |u_ii| < AEPS).  Each entry sees the reference's updates
// in the reference's order with separately rounded products (built with
// -ffp-contract=off), so the factor is bit-identical.  False if a row's diagonal is absent.
bool egpu_ilut_host(int n, const std::vector<int> &rows, const std::vector<int> &cols,
                    const std::vector<double> &vals, double tol, std::vector<int> &ir, std::vector<int> &ic,
                    std::vector<int> &id, std::vector<double> &iv) {
  constexpr double AEPS = 10.0 * 2.220446049250313e-16;  // the reference's AEPS (EGPU_AEPS)
  std::vector<double> w(n, 0.0);
  std::vector<char> flag(n, 0);
  std::vector<int> touched, heap;
  ir.assign(n + 1, 0);
  id.assign(n, -1);
  ic.clear();
  iv.clear();
  ic.reserve((size_t)rows[n] * 2);
  iv.reserve((size_t)rows[n] * 2);
  auto push = [&](int k) {
    heap.push_back(k);
    std::push_heap(heap.begin(), heap.end(), std::greater<int>());
  };
  for (int i = 0; i < n; ++i) {
    touched.clear();
    for (int e = rows[i]; e < rows[i + 1]; ++e) {
      const int c = cols[e];
      flag[c] = 1;
      w[c] = vals[e];
      touched.push_back(c);
      if (c < i) push(c);
    }
    while (!heap.empty()) {
      std::pop_heap(heap.begin(), heap.end(), std::greater<int>());
      const int k = heap.back();
      heap.pop_back();
      const double ukk = iv[id[k]];
      if (std::fabs(ukk) > AEPS) w[k] = w[k] / ukk;
      const double mk = w[k];
      for (int l = id[k] + 1; l < ir[k + 1]; ++l) {
        const int j = ic[l];
        if (!flag[j]) {
          flag[j] = 1;
          touched.push_back(j);
          if (j < i) push(j);
        }
        const double prod = mk * iv[l];
        w[j] = w[j] - prod;
      }
    }
    double sq = 0.0;
    for (int e = rows[i]; e < rows[i + 1]; ++e) {
      const double a = std::fabs(vals[e]);
      const double a2 = a * a;
      sq = sq + a2;
    }
    const double drop = tol * std::sqrt(sq);
    std::sort(touched.begin(), touched.end());
    for (int k : touched) {
      if (std::fabs(w[k]) >= drop || k == i) {
        if (k == i) id[i] = (int)ic.size();
        ic.push_back(k);
        iv.push_back(w[k]);
      }
      w[k] = 0.0;
      flag[k] = 0;
    }
    if (id[i] < 0) return false;
    ir[i + 1] = (int)ic.size();
  }
  for (int i = 0; i < n; ++i) {
    double &d = iv[id[i]];
    d = std::fabs(d) < AEPS ? 1.0 : 1.0 / d;
  }
  return true;
}

extern "C" long long egpu_ilu_pattern(int n, const int *rows, const int *cols, const int *diag, int order,
                                      long long cap, int *ilu_rows, int *ilu_cols, int *ilu_diag) {
  if (n < 1 || !rows || !cols || !diag || order < 0 || order > 9) return EGPU_ERR_ARG;
  const int base = rows[0];
  const long long nnz = (long long)rows[n] - base;
  std::vector<int> r(n + 1), c(nnz), d(n);
  for (int i = 0; i <= n; ++i) r[i] = rows[i] - base;
  for (long long e = 0; e < nnz; ++e) {
    c[e] = cols[e] - base;
    if (c[e] < 0 || c[e] >= n) return EGPU_ERR_ARG;
  }
  for (int i = 0; i < n; ++i) {
    d[i] = diag[i] - base;
    if (d[i] < r[i] || d[i] >= r[i + 1] || c[d[i]] != i) return EGPU_ERR_ARG;
  }
  std::vector<int> orows, ocols, odiag;
  egpu_ilu_structure(n, r, c, d, order, orows, ocols, odiag);
  const long long onnz = orows[n];
  if (cap >= onnz && ilu_rows && ilu_cols && ilu_diag) {
    for (int i = 0; i <= n; ++i) ilu_rows[i] = orows[i] + base;
    for (long long e = 0; e < onnz; ++e) ilu_cols[e] = ocols[e] + base;
    for (int i = 0; i < n; ++i) ilu_diag[i] = odiag[i] + base;
  }
  return onnz;
}
