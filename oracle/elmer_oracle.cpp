// elmer_oracle.cpp -- CPU restatement of ElmerSolver's linear-system path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the GPU library, used by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg.  Never linked by the
// product.  Built with -ffp-contract=off so every a*b+c rounds twice, as the
// reference's gfortran -O2 x86-64 build does.
//
// Every routine names the Fortran it restates (paths relative to the Elmer tree).
// Pinned to the reference's regression targets (heateq / linearsolvers NRM values on their
// committed mesh) and to independent transcriptions; not to a built ElmerSolver (Fortran).
// Indices are 1-based like Matrix_t; arrays below are addressed with a -1 shift.

#include "elmer_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double AEPS = 10.0 * 2.220446049250313e-16;  // Types.src:64, 10*EPSILON(1.0_dp)
constexpr double TINY_DP = 2.2250738585072014e-308;     // TINY(1.0_dp)
constexpr double HUTI_EPSILON = 1.17549435E-38;         // hutiter/src/huti_defs.h:23

// HUTI status codes, hutiter/src/huti_fdefs.h:18-52
constexpr int HUTI_CONVERGENCE = 1;
constexpr int HUTI_MAXITER = 2;
constexpr int HUTI_DIVERGENCE = 3;
constexpr int HUTI_CG_RHO = 20;
constexpr int HUTI_BICGSTAB_RHO = 35;
constexpr int HUTI_BICGSTAB_SNORM = 36;
constexpr int HUTI_BICGSTAB_OMEGA = 37;

// ---------------------------------------------------------------------------
// List matrix: ListMatrix_t / ListMatrixEntry_t (Types.src) and
// List_GetMatrixIndex (ListMatrix.src:263-320): a per-row singly linked list kept
// sorted by column index; a new index is inserted before the first entry >= it.
struct Entry {
  int index;
  Entry *next;
};
struct ListRow {
  Entry *head = nullptr;
  int degree = 0;
  int level = 0;
};

struct EntryPool {
  std::vector<Entry *> blocks;
  size_t used = 0, cap = 0;
  Entry *get() {
    if (used == cap) {
      cap = 1 << 20;
      blocks.push_back(static_cast<Entry *>(std::malloc(sizeof(Entry) * cap)));
      used = 0;
    }
    return &blocks.back()[used++];
  }
  ~EntryPool() {
    for (auto *b : blocks) std::free(b);
  }
};

void list_get_matrix_index(std::vector<ListRow> &L, EntryPool &pool, int k1, int k2) {
  ListRow &row = L[k1 - 1];
  Entry *c = row.head;
  if (!c) {
    Entry *e = pool.get();
    e->index = k2;
    e->next = nullptr;
    row.degree = 1;
    row.head = e;
    return;
  }
  Entry *prev = nullptr;
  while (c) {
    if (c->index >= k2) break;
    prev = c;
    c = c->next;
  }
  if (c && c->index == k2) return;
  Entry *e = pool.get();
  e->index = k2;
  e->next = c;
  if (prev)
    prev->next = e;
  else
    row.head = e;
  row.degree++;
}

// ComputeBandwidth, BandwidthOptimize.src:70-97
int compute_bandwidth(int n, const std::vector<ListRow> &L, const int *reorder) {
  int hbw = 0;
  for (int i = 1; i <= n; ++i) {
    for (Entry *c = L[i - 1].head; c; c = c->next) {
      int k = c->index;
      int d = reorder ? std::abs(reorder[i - 1] - reorder[k - 1]) : std::abs(i - k);
      hbw = std::max(hbw, d);
    }
  }
  return hbw;
}

// OptimizeBandwidth, BandwidthOptimize.src:108-355 (Levelize :290-350, Renumber :266-286).
struct BandwidthOptimizer {
  std::vector<ListRow> &L;
  int n;
  std::vector<char> done_already;
  int max_level = 0;
  std::vector<int> perm_local, done_index;
  int indx = 1;

  BandwidthOptimizer(std::vector<ListRow> &l, int nn) : L(l), n(nn) {}

  // Levelize: depth-first walk from nin with an explicit stack of list positions.
  void levelize(int nin, int level_in) {
    int nn = nin, level = level_in;
    std::vector<Entry *> stack;
    stack.reserve(512);
    Entry *p = L[nn - 1].head;
    while (p) {
      stack.push_back(p);
      L[nn - 1].level = level;
      done_already[nn - 1] = 1;
      max_level = std::max(max_level, level);
      p = L[nn - 1].head;
      while (true) {
        if (p) {
          nn = p->index;
          if (nn <= n && !done_already[nn - 1]) {
            level++;
            break;
          }
        } else if (!stack.empty()) {
          p = stack.back();
          level--;
          stack.pop_back();
        } else {
          break;
        }
        p = p->next;
      }
    }
  }

  // Renumber: append the not-yet-numbered neighbours of a row in list order.
  void renumber(Entry *current) {
    for (Entry *p = current; p; p = p->next) {
      int k = p->index;
      if (k <= n && done_index[k - 1] == 0) {
        perm_local[indx - 1] = k;
        done_index[k - 1] = indx;
        indx++;
      }
    }
  }

  // Returns HalfBandWidth; perm (size n, entries 1..n) is updated in place.
  int run(int *perm, bool optimize, bool use_optimized, int *hbw_before_out, int *start_out,
          int *rejected_out) {
    int hbw = compute_bandwidth(n, L, nullptr) + 1;
    *hbw_before_out = hbw;
    *rejected_out = 0;
    *start_out = 0;
    if (!optimize) return hbw;
    int hbw_before = hbw;

    int start = 1;
    int min_degree = L[start - 1].degree;
    for (int i = 1; i <= n; ++i) {
      if (L[i - 1].degree < min_degree) {
        start = i;
        min_degree = L[i - 1].degree;
      }
      L[i - 1].level = 0;
    }
    done_already.assign(n, 0);
    max_level = 0;
    levelize(start, 0);

    bool new_root = true;
    while (new_root) {
      new_root = false;
      min_degree = L[start - 1].degree;
      int k = start;
      for (int i = 1; i <= n; ++i) {
        if (L[i - 1].level == max_level && L[i - 1].degree < min_degree) {
          k = i;
          min_degree = L[i - 1].degree;
        }
      }
      if (k != start) {
        int j = max_level;
        max_level = 0;
        std::fill(done_already.begin(), done_already.end(), 0);
        levelize(k, 0);
        if (j > max_level) {
          new_root = true;
          start = j;  // BandwidthOptimize.src:190 assigns the old level, kept as written
        }
      }
    }
    *start_out = start;

    perm_local.assign(n, 0);
    done_index.assign(n, 0);
    indx = 1;
    perm_local[indx - 1] = start;
    done_index[start - 1] = indx;
    indx++;
    for (int i = 1; i <= n; ++i) {
      if (perm_local[i - 1] == 0) {
        for (int j = 1; j <= n; ++j) {
          if (done_index[j - 1] == 0) {
            perm_local[indx - 1] = j;
            done_index[j - 1] = indx;
            indx++;
            break;
          }
        }
      }
      renumber(L[perm_local[i - 1] - 1].head);
    }
    // reverse order (profile optimisation)
    std::fill(done_index.begin(), done_index.end(), 0);
    for (int i = 1; i <= n; ++i) done_index[perm_local[i - 1] - 1] = n - i + 1;
    std::vector<int> saved(perm, perm + n);
    for (int i = 1; i <= n; ++i) {
      int k = saved[i - 1];
      perm[i - 1] = k > 0 ? done_index[k - 1] : 0;
    }
    int hbw_after = compute_bandwidth(n, L, perm) + 1;
    hbw = hbw_after;
    if (hbw_before < hbw && !use_optimized) {
      hbw = hbw_before;
      std::copy(saved.begin(), saved.end(), perm);
      *rejected_out = 1;
    }
    return hbw;
  }
};

inline double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// ===========================================================================
// Pattern
struct orc_pattern {
  int nnodes = 0, dofs = 1, n = 0;
  long long nnz = 0;
  int hbw_before = 0, hbw_after = 0, start_node = 0, rejected = 0;
  std::vector<int> perm, rows, cols, diag;
};

extern "C" orc_pattern *orc_pattern_create(int nnodes, int nelem, int nen, const int *elem_nodes,
                                           int dofs, int optimize_bw, int use_optimized_always) {
  auto *P = new orc_pattern;
  P->nnodes = nnodes;
  P->dofs = dofs;
  // CreateMatrix, ElementUtils.src:753-771: every node is active -> identity initial Perm.
  std::vector<int> perm(nnodes);
  for (int i = 0; i < nnodes; ++i) perm[i] = i + 1;

  // MakeListMatrix, ElementUtils.src:424-498: all node pairs of each element, element order.
  std::vector<ListRow> L(nnodes);
  EntryPool pool;
  for (int t = 0; t < nelem; ++t) {
    const int *ix = elem_nodes + (size_t)t * nen;
    for (int i = 0; i < nen; ++i) {
      int k1 = perm[ix[i] - 1];
      if (k1 <= 0) continue;
      for (int j = 0; j < nen; ++j) {
        int k2 = perm[ix[j] - 1];
        if (k2 <= 0) continue;
        list_get_matrix_index(L, pool, k1, k2);
      }
    }
  }
  // RowNonzeros / TotalMatrixElements, ElementUtils.src:603-614
  std::vector<int> row_nonzeros(nnodes);
  long long total = 0;
  for (int i = 0; i < nnodes; ++i) {
    row_nonzeros[i] = L[i].degree;
    total += L[i].degree;
  }

  BandwidthOptimizer bo(L, nnodes);
  P->hbw_after = bo.run(perm.data(), optimize_bw != 0, use_optimized_always != 0, &P->hbw_before,
                        &P->start_node, &P->rejected);

  // CRS_CreateMatrix, CRSMatrix.src:816-875
  const int n = dofs * nnodes;
  P->n = n;
  std::vector<int> inv_perm(nnodes, 0);
  {
    int j = 0;
    for (int i = 0; i < nnodes; ++i)
      if (perm[i] > 0) inv_perm[perm[i] - 1] = ++j;
  }
  P->rows.assign(n + 1, 0);
  P->rows[0] = 1;
  for (int i = 2; i <= n; ++i) {
    int j = inv_perm[(i - 2) / dofs];
    P->rows[i - 1] = P->rows[i - 2] + dofs * row_nonzeros[j - 1];
  }
  {
    int j = inv_perm[(n - 1) / dofs];
    P->rows[n] = P->rows[n - 1] + dofs * row_nonzeros[j - 1];
  }
  P->nnz = (long long)dofs * dofs * total;
  P->cols.assign(P->nnz, 0);
  P->diag.assign(n, 0);

  // InitializeMatrix, ElementUtils.src:625-660 (InvInitialReorder = identity)
  for (int i = 1; i <= nnodes; ++i) {
    for (int l = 1; l <= dofs; ++l) {
      int jn = perm[i - 1];
      int k1 = dofs * (jn - 1) + l;
      long long k2 = P->rows[k1 - 1] - 1;
      for (Entry *c = L[i - 1].head; c; c = c->next) {
        int k = perm[c->index - 1];
        k = dofs * (k - 1);
        for (int m = k + 1; m <= k + dofs; ++m) {
          k2++;
          P->cols[k2 - 1] = m;
        }
      }
    }
  }
  // CRS_SortMatrix, CRSMatrix.src:168-232
  for (int i = 1; i <= n; ++i)
    std::sort(P->cols.begin() + (P->rows[i - 1] - 1), P->cols.begin() + (P->rows[i] - 1));
  for (int i = 1; i <= n; ++i) {
    for (int j = P->rows[i - 1]; j <= P->rows[i] - 1; ++j) {
      if (P->cols[j - 1] == i) {
        P->diag[i - 1] = j;
        break;
      }
    }
  }
  P->perm = std::move(perm);
  return P;
}

extern "C" void orc_pattern_info(const orc_pattern *p, int *n, long long *nnz, int *hbw_before,
                                 int *hbw_after, int *start_node, int *rejected) {
  if (n) *n = p->n;
  if (nnz) *nnz = p->nnz;
  if (hbw_before) *hbw_before = p->hbw_before;
  if (hbw_after) *hbw_after = p->hbw_after;
  if (start_node) *start_node = p->start_node;
  if (rejected) *rejected = p->rejected;
}

extern "C" void orc_pattern_copy(const orc_pattern *p, int *perm, int *rows, int *cols, int *diag) {
  if (perm) std::copy(p->perm.begin(), p->perm.end(), perm);
  if (rows) std::copy(p->rows.begin(), p->rows.end(), rows);
  if (cols) std::copy(p->cols.begin(), p->cols.end(), cols);
  if (diag) std::copy(p->diag.begin(), p->diag.end(), diag);
}

extern "C" void orc_pattern_free(orc_pattern *p) { delete p; }

// ===========================================================================
// Reference elements and quadrature

namespace {

struct Quad {
  int n;
  double u[8], v[8], w[8], s[8];
};

// GaussPointsBrick, Integration.src:1446-1486 with the 2-point Gauss-Legendre rule
// (points +-1/sqrt(3), weights 1; ComputeGaussPoints1D, Integration.src:406-525).
Quad gauss_brick8() {
  Quad q{};
  const double P[2] = {-1.0 / std::sqrt(3.0), 1.0 / std::sqrt(3.0)};
  const double W[2] = {1.0, 1.0};
  int t = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) {
        q.u[t] = P[k];
        q.v[t] = P[j];
        q.w[t] = P[i];
        q.s[t] = W[i] * W[j] * W[k];
        ++t;
      }
  q.n = t;
  return q;
}

// GaussPointsTetra 4-point rule, Integration.src:281-295, 924-931 (weights / 6).
Quad gauss_tetra4() {
  Quad q{};
  const double U[4] = {0.1757281246520584, 0.2445310270213291, 0.5556470949048655, 0.0240937534217468};
  const double V[4] = {0.5656137776620919, 0.0501800797762026, 0.1487681308666864, 0.2354380116950194};
  const double Wt[4] = {0.2180665126782654, 0.5635595064952189, 0.0350112499848832, 0.1833627308416330};
  for (int i = 0; i < 4; ++i) {
    q.u[i] = U[i];
    q.v[i] = V[i];
    q.w[i] = Wt[i];
    q.s[i] = 0.25 / 6.0;
  }
  q.n = 4;
  return q;
}

// GaussPointsTriangle 3-point rule, Integration.src:84-91, 776-780 (weights / 2).
Quad gauss_triangle3() {
  Quad q{};
  const double U[3] = {0.16666666666666667, 0.66666666666666667, 0.16666666666666667};
  const double V[3] = {0.16666666666666667, 0.16666666666666667, 0.66666666666666667};
  for (int i = 0; i < 3; ++i) {
    q.u[i] = U[i];
    q.v[i] = V[i];
    q.w[i] = 0.0;
    q.s[i] = 0.33333333333333333 / 2.0;
  }
  q.n = 3;
  return q;
}

// Nodal basis and local derivatives (NodalBasisFunctions/NodalFirstDerivatives,
// ElementDescription.src:2012-2152) for the element types of this path
// (elements.def 303 :155-185, 504 :365-404, 808 :606-643).
int basis(int code, double u, double v, double w, double *N, double dN[][3]) {
  switch (code) {
    case 808: {
      static const double nu[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
      static const double nv[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
      static const double nw[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
      for (int p = 0; p < 8; ++p) {
        double a = 1.0 + nu[p] * u, b = 1.0 + nv[p] * v, c = 1.0 + nw[p] * w;
        N[p] = 0.125 * a * b * c;
        dN[p][0] = 0.125 * nu[p] * b * c;
        dN[p][1] = 0.125 * nv[p] * a * c;
        dN[p][2] = 0.125 * nw[p] * a * b;
      }
      return 8;
    }
    case 504:
      N[0] = 1.0 - u - v - w;
      N[1] = u;
      N[2] = v;
      N[3] = w;
      dN[0][0] = -1; dN[0][1] = -1; dN[0][2] = -1;
      dN[1][0] = 1;  dN[1][1] = 0;  dN[1][2] = 0;
      dN[2][0] = 0;  dN[2][1] = 1;  dN[2][2] = 0;
      dN[3][0] = 0;  dN[3][1] = 0;  dN[3][2] = 1;
      return 4;
    case 303:
      N[0] = 1.0 - u - v;
      N[1] = u;
      N[2] = v;
      dN[0][0] = -1; dN[0][1] = -1; dN[0][2] = 0;
      dN[1][0] = 1;  dN[1][1] = 0;  dN[1][2] = 0;
      dN[2][0] = 0;  dN[2][1] = 1;  dN[2][2] = 0;
      return 3;
  }
  return 0;
}

int elem_dim(int code) { return code / 100 >= 5 ? 3 : 2; }

// ElementInfo geometry part: ElementMetric (ElementDescription.src:6757-6884),
// InvertMatrix3x3 (:8536-8555) and the dBasisdx contraction (:3303-3312).
// Returns detJ = sqrt(det(G)), G = dx^T dx.
bool element_info(int nen, int dim, int cdim, const double (*X)[3], const double dN[][3],
                  double dBdx[][3], double *detJ) {
  double dx[3][3] = {{0}};
  for (int i = 0; i < dim; ++i)
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (int p = 0; p < nen; ++p) s = s + X[p][c] * dN[p][i];
      dx[c][i] = s;
    }
  double G[3][3] = {{0}}, GI[3][3] = {{0}};
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) {
      double s = 0.0;
      for (int k = 0; k < cdim; ++k) s = s + dx[k][i] * dx[k][j];
      G[i][j] = s;
    }
  double detG;
  if (dim == 2) {
    detG = G[0][0] * G[1][1] - G[0][1] * G[1][0];
    if (detG <= TINY_DP) return false;
    GI[0][0] = G[1][1] / detG;
    GI[0][1] = -G[0][1] / detG;
    GI[1][0] = -G[1][0] / detG;
    GI[1][1] = G[0][0] / detG;
  } else {
    detG = G[0][0] * (G[1][1] * G[2][2] - G[1][2] * G[2][1]) +
           G[0][1] * (G[1][2] * G[2][0] - G[1][0] * G[2][2]) +
           G[0][2] * (G[1][0] * G[2][1] - G[1][1] * G[2][0]);
    if (detG <= TINY_DP) return false;
    double s = 1.0 / detG;
    GI[0][0] = s * (G[1][1] * G[2][2] - G[2][1] * G[1][2]);
    GI[1][0] = -s * (G[1][0] * G[2][2] - G[2][0] * G[1][2]);
    GI[2][0] = s * (G[1][0] * G[2][1] - G[2][0] * G[1][1]);
    GI[0][1] = -s * (G[0][1] * G[2][2] - G[2][1] * G[0][2]);
    GI[1][1] = s * (G[0][0] * G[2][2] - G[2][0] * G[0][2]);
    GI[2][1] = -s * (G[0][0] * G[2][1] - G[2][0] * G[0][1]);
    GI[0][2] = s * (G[0][1] * G[1][2] - G[1][1] * G[0][2]);
    GI[1][2] = -s * (G[0][0] * G[1][2] - G[1][0] * G[0][2]);
    GI[2][2] = s * (G[0][0] * G[1][1] - G[1][0] * G[0][1]);
  }
  *detJ = std::sqrt(detG);
  double LtoG[3][3] = {{0}};
  for (int i = 0; i < cdim; ++i)
    for (int j = 0; j < dim; ++j) {
      double s = 0.0;
      for (int k = 0; k < dim; ++k) s = s + dx[i][k] * GI[k][j];
      LtoG[i][j] = s;
    }
  for (int p = 0; p < nen; ++p)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      if (j < cdim)
        for (int k = 0; k < dim; ++k) s = s + dN[p][k] * LtoG[j][k];
      dBdx[p][j] = s;
    }
  return true;
}

// CRS_GlueLocalMatrix, CRSMatrix.src:507-590: linear search in the row, split at Diag.
inline void glue_add(const int *rows, const int *cols, const int *diag, double *values, int row,
                     int col, double val) {
  if (col >= row) {
    for (int c = diag[row - 1]; c <= rows[row] - 1; ++c)
      if (cols[c - 1] == col) {
        values[c - 1] = values[c - 1] + val;
        return;
      }
  } else {
    for (int c = rows[row - 1]; c <= diag[row - 1] - 1; ++c)
      if (cols[c - 1] == col) {
        values[c - 1] = values[c - 1] + val;
        return;
      }
  }
}

}  // namespace

// HeatSolver bulk loop (modules/HeatSolve.src:655-985) with the diffusion-only branch
// of DiffuseConvectiveCompose (DiffuseConvectiveAnisotropic.src:289-612) and the
// scatter DefaultUpdateEquations -> UpdateGlobalEquations -> CRS_GlueLocalMatrix
// (SolverUtils.src:984-1054).  Conductivity is isotropic: C2 = k*I
// (HeatSolve.src:716-723); the load is nodal rho*q (HeatSolve.src:884) interpolated
// at the integration point.
extern "C" void orc_assemble_poisson(int nnodes, const double *xyz, int cdim, int nelem, int code,
                                     const int *elem_nodes, const double *elem_k,
                                     const double *nodal_k, const double *load, const int *perm,
                                     int n, const int *rows, const int *cols, const int *diag,
                                     double *values, double *rhs) {
  (void)nnodes;
  (void)n;
  const int dim = elem_dim(code);
  Quad q = code == 808 ? gauss_brick8() : code == 504 ? gauss_tetra4() : gauss_triangle3();
  const int nen = code % 100;
  for (int e = 0; e < nelem; ++e) {
    const int *ix = elem_nodes + (size_t)e * nen;
    double X[8][3];
    double nk[8], nl[8];
    for (int p = 0; p < nen; ++p) {
      for (int c = 0; c < 3; ++c) X[p][c] = xyz[(size_t)(ix[p] - 1) * 3 + c];
      nk[p] = elem_k ? elem_k[e] : (nodal_k ? nodal_k[ix[p] - 1] : 1.0);
      nl[p] = load ? load[ix[p] - 1] : 0.0;
    }
    double K[8][8] = {{0}}, F[8] = {0};
    for (int t = 0; t < q.n; ++t) {
      double N[8], dN[8][3], dB[8][3], detJ;
      basis(code, q.u[t], q.v[t], q.w[t], N, dN);
      if (!element_info(nen, dim, cdim, X, dN, dB, &detJ)) continue;
      double s = detJ * q.s[t];
      double kk = 0.0;
      for (int p = 0; p < nen; ++p) kk = kk + nk[p] * N[p];
      for (int p = 0; p < nen; ++p)
        for (int qq = 0; qq < nen; ++qq) {
          double A = 0.0;
          for (int i = 0; i < dim; ++i) A = A + kk * dB[qq][i] * dB[p][i];
          K[p][qq] = K[p][qq] + s * A;
        }
      double force = 0.0;
      for (int p = 0; p < nen; ++p) force = force + nl[p] * N[p];
      for (int p = 0; p < nen; ++p) F[p] = F[p] + s * (force * N[p]);
    }
    int gi[8];
    for (int p = 0; p < nen; ++p) gi[p] = perm[ix[p] - 1];
    for (int i = 0; i < nen; ++i) {
      if (gi[i] <= 0) continue;
      for (int j = 0; j < nen; ++j) {
        if (gi[j] <= 0) continue;
        glue_add(rows, cols, diag, values, gi[i], gi[j], K[i][j]);
      }
    }
    for (int i = 0; i < nen; ++i)
      if (gi[i] > 0) rhs[gi[i] - 1] = rhs[gi[i] - 1] + F[i];
  }
}

// StressSolver BulkAssembly (modules/StressSolve.src:815-1072) with StressCompose
// (Stress.src:59-521), isotropic 3D: C (Stress.src:260-273), G/B strain maps
// (:366-426), STIFF += s*G*C*B (:433-439), nodal body force load (:476-510) and the
// final symmetrisation STIFF = (STIFF+STIFF^T)/2 (:513-515).
extern "C" void orc_assemble_elastic(int nnodes, const double *xyz, int nelem, int code,
                                     const int *elem_nodes, double young, double poisson,
                                     const double *bf, const int *perm, int n, const int *rows,
                                     const int *cols, const int *diag, double *values,
                                     double *rhs) {
  (void)nnodes;
  (void)n;
  const int dim = 3, cdim = 3, dofs = 3;
  Quad q = code == 808 ? gauss_brick8() : gauss_tetra4();
  const int nen = code % 100;
  double C[6][6] = {{0}};
  C[0][0] = 1.0 - poisson; C[0][1] = poisson; C[0][2] = poisson;
  C[1][0] = poisson; C[1][1] = 1.0 - poisson; C[1][2] = poisson;
  C[2][0] = poisson; C[2][1] = poisson; C[2][2] = 1.0 - poisson;
  C[3][3] = 0.5 - poisson; C[4][4] = 0.5 - poisson; C[5][5] = 0.5 - poisson;
  const double cs = young / ((1 + poisson) * (1 - 2 * poisson));
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) C[i][j] = C[i][j] * cs;

  std::vector<double> K(24 * 24), F(24);
  for (int e = 0; e < nelem; ++e) {
    const int *ix = elem_nodes + (size_t)e * nen;
    double X[8][3];
    for (int p = 0; p < nen; ++p)
      for (int c = 0; c < 3; ++c) X[p][c] = xyz[(size_t)(ix[p] - 1) * 3 + c];
    std::fill(K.begin(), K.end(), 0.0);
    std::fill(F.begin(), F.end(), 0.0);
    const int nd = dofs * nen;
    for (int t = 0; t < q.n; ++t) {
      double N[8], dN[8][3], dB[8][3], detJ;
      basis(code, q.u[t], q.v[t], q.w[t], N, dN);
      if (!element_info(nen, dim, cdim, X, dN, dB, &detJ)) continue;
      double s = detJ * q.s[t];
      for (int p = 0; p < nen; ++p) {
        double G[3][6] = {{0}};
        G[0][0] = dB[p][0];
        G[1][1] = dB[p][1];
        G[2][2] = dB[p][2];
        G[0][3] = dB[p][1];
        G[1][3] = dB[p][0];
        G[1][4] = dB[p][2];
        G[2][4] = dB[p][1];
        G[0][5] = dB[p][2];
        G[2][5] = dB[p][0];
        double GC[3][6];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 6; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc = acc + G[i][k] * C[k][j];
            GC[i][j] = acc;
          }
        for (int qq = 0; qq < nen; ++qq) {
          double B[6][3] = {{0}};
          B[0][0] = dB[qq][0];
          B[1][1] = dB[qq][1];
          B[2][2] = dB[qq][2];
          B[3][0] = dB[qq][1];
          B[3][1] = dB[qq][0];
          B[4][1] = dB[qq][2];
          B[4][2] = dB[qq][1];
          B[5][0] = dB[qq][2];
          B[5][2] = dB[qq][0];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              double a = 0.0;
              for (int k = 0; k < 6; ++k) a = a + GC[i][k] * B[k][j];
              K[(size_t)(dim * p + i) * nd + dim * qq + j] += s * a;
            }
        }
        for (int i = 0; i < 3; ++i) {
          double lb = 0.0;
          for (int m = 0; m < nen; ++m) lb = lb + bf[i] * N[m];
          double load_ip = 0.0 + lb * N[p];
          F[dim * p + i] = F[dim * p + i] + s * load_ip;
        }
      }
    }
    for (int i = 0; i < nd; ++i)
      for (int j = i + 1; j < nd; ++j) {
        double a = (K[(size_t)i * nd + j] + K[(size_t)j * nd + i]) / 2.0;
        K[(size_t)i * nd + j] = a;
        K[(size_t)j * nd + i] = a;
      }
    int gi[8];
    for (int p = 0; p < nen; ++p) gi[p] = perm[ix[p] - 1];
    // CRS_GlueLocalMatrix DOF>1 branch, CRSMatrix.src:547-585
    for (int i = 1; i <= nen; ++i)
      for (int k = 0; k <= dofs - 1; ++k) {
        if (gi[i - 1] <= 0) continue;
        int row = dofs * gi[i - 1] - k;
        for (int j = 1; j <= nen; ++j)
          for (int l = 0; l <= dofs - 1; ++l) {
            if (gi[j - 1] <= 0) continue;
            int col = dofs * gi[j - 1] - l;
            glue_add(rows, cols, diag, values, row, col,
                     K[(size_t)(dofs * i - k - 1) * nd + (dofs * j - l - 1)]);
          }
      }
    for (int i = 0; i < nen; ++i)
      if (gi[i] > 0)
        for (int j = 1; j <= dofs; ++j) {
          int k = dofs * (gi[i] - 1) + j;
          rhs[k - 1] = rhs[k - 1] + F[dofs * i + j - 1];
        }
  }
}

// ===========================================================================
// Scaling: ScaleLinearSystem (SolverUtils.src:6470-6640)
extern "C" void orc_scale(int n, const int *rows, const int *cols, const int *diag, double *values,
                          double *b, double *x, double *D, double *rhs_scaling, int rhs_scale) {
  for (int i = 0; i < n; ++i) D[i] = 0.0;
  for (int i = 1; i <= n; ++i) {
    int j = diag[i - 1];
    if (j > 0) D[i - 1] = values[j - 1];
  }
  bool any_tiny = false;
  for (int i = 0; i < n; ++i)
    if (std::fabs(D[i]) <= TINY_DP) any_tiny = true;
  if (any_tiny) {
    for (int i = 1; i <= n; ++i) {
      if (std::fabs(D[i - 1]) <= TINY_DP) {
        double s = 0.0;
        for (int j = rows[i - 1]; j <= rows[i] - 1; ++j) s += std::fabs(values[j - 1]);
        D[i - 1] = s;
      } else {
        int j = diag[i - 1];
        if (j > 0) D[i - 1] = values[j - 1];
      }
    }
  }
  for (int i = 0; i < n; ++i) D[i] = std::fabs(D[i]) > TINY_DP ? 1.0 / std::sqrt(std::fabs(D[i])) : 1.0;
  for (int i = 1; i <= n; ++i)
    for (int j = rows[i - 1]; j <= rows[i] - 1; ++j)
      values[j - 1] = values[j - 1] * (D[i - 1] * D[cols[j - 1] - 1]);
  *rhs_scaling = 1.0;
  if (b) {
    for (int i = 0; i < n; ++i) b[i] = b[i] * D[i];
    double bnorm = 1.0;
    if (rhs_scale) {
      double s = 0.0;
      for (int i = 0; i < n; ++i) s = s + b[i] * b[i];
      bnorm = std::sqrt(s);
    }
    *rhs_scaling = bnorm;
    for (int i = 0; i < n; ++i) D[i] = D[i] * bnorm;
    for (int i = 0; i < n; ++i) b[i] = b[i] / bnorm;
    if (x)
      for (int i = 0; i < n; ++i) x[i] = x[i] / D[i];
  }
}

// BackScaleLinearSystem (SolverUtils.src:6754-6868)
static void backscale(int n, const int *rows, const int *cols, double *values, double *b,
                      double *x, double *D, double bnorm) {
  if (b) {
    if (x)
      for (int i = 0; i < n; ++i) x[i] = x[i] * D[i];
    for (int i = 0; i < n; ++i) D[i] = D[i] / bnorm;
    for (int i = 0; i < n; ++i) b[i] = b[i] / D[i] * bnorm;
  }
  for (int i = 1; i <= n; ++i)
    for (int j = rows[i - 1]; j <= rows[i] - 1; ++j)
      values[j - 1] = values[j - 1] / (D[i - 1] * D[cols[j - 1] - 1]);
}

// CRS_SetSymmDirichlet, CRSMatrix.src:674-740
static void set_symm_dirichlet(const int *rows, const int *cols, const int *diag, double *values,
                               double *b, int nrow, double val) {
  for (int l = rows[nrow - 1]; l <= rows[nrow] - 1; ++l) {
    int i = cols[l - 1];
    if (i == nrow) continue;
    int k1, k2;
    if (nrow > i) {
      k1 = diag[i - 1] + 1;
      k2 = rows[i] - 1;
    } else {
      k1 = rows[i - 1];
      k2 = diag[i - 1] - 1;
    }
    for (int j = k1; j <= k2; ++j) {  // the CRS_Search branch finds the same entry
      if (cols[j - 1] == nrow) {
        b[i - 1] = b[i - 1] - values[j - 1] * val;
        values[j - 1] = 0.0;
        break;
      } else if (cols[j - 1] > nrow) {
        break;
      }
    }
  }
  for (int j = rows[nrow - 1]; j <= rows[nrow] - 1; ++j) values[j - 1] = 0.0;  // CRS_ZeroRow
  b[nrow - 1] = val;
  values[diag[nrow - 1] - 1] = 1.0;
}

// DefaultDirichletBCs (DefUtils.src:3530-4031): ScaleLinearSystem(RHSscaling=.FALSE.),
// per constrained DOF SetElementValues (SolverUtils.src:2460-2476), BackScaleLinearSystem.
extern "C" void orc_dirichlet(int n, const int *rows, const int *cols, const int *diag,
                              double *values, double *rhs, int ncon, const int *con_rows,
                              const double *con_vals, int symmetric, int scale) {
  std::vector<double> D(n, 1.0);
  double rs = 1.0;
  if (scale) orc_scale(n, rows, cols, diag, values, rhs, nullptr, D.data(), &rs, 0);
  for (int c = 0; c < ncon; ++c) {
    int k = con_rows[c];
    double val = con_vals ? con_vals[c] : 0.0;
    if (symmetric) {
      set_symm_dirichlet(rows, cols, diag, values, rhs, k, val / D[k - 1]);
    } else {
      for (int j = rows[k - 1]; j <= rows[k] - 1; ++j) values[j - 1] = 0.0;  // ZeroRow
      values[diag[k - 1] - 1] = 1.0;                                          // SetMatrixElement
      rhs[k - 1] = val / D[k - 1];
    }
  }
  if (scale) backscale(n, rows, cols, values, rhs, nullptr, D.data(), 1.0);
}

// ===========================================================================
// Krylov path

// CRS_MatrixVectorProd, CRSMatrix.src:3565-3573 (OpenMP over rows)
extern "C" void orc_spmv(int n, const int *rows, const int *cols, const double *values,
                         const double *u, double *v, int omp_threads) {
#ifdef _OPENMP
  int nt = omp_threads > 0 ? omp_threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nt) schedule(static)
#endif
  for (int i = 1; i <= n; ++i) {
    double s = 0.0;
    for (int j = rows[i - 1]; j <= rows[i] - 1; ++j) s = s + values[j - 1] * u[cols[j - 1] - 1];
    v[i - 1] = s;
  }
  (void)omp_threads;
}

// CRS_IncompleteLU(A,0), CRSMatrix.src:2157-2388 (LU branch :2312-2366)
extern "C" void orc_ilu0(int n, const int *rows, const int *cols, const int *diag,
                         const double *values, double *ilu) {
  std::vector<double> S(n + 1, 0.0);
  std::vector<char> C(n + 1, 0);
  for (int i = 1; i <= n; ++i) {
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) S[cols[k - 1]] = values[k - 1];
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) C[cols[k - 1]] = 1;
    for (int m = rows[i - 1]; m <= diag[i - 1] - 1; ++m) {
      int k = cols[m - 1];
      if (S[k] == 0.0) continue;
      if (std::fabs(ilu[diag[k - 1] - 1]) > AEPS) S[k] = S[k] / ilu[diag[k - 1] - 1];
      for (int l = diag[k - 1] + 1; l <= rows[k] - 1; ++l) {
        int j = cols[l - 1];
        if (C[j]) S[j] = S[j] - S[k] * ilu[l - 1];
      }
    }
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) {
      if (C[cols[k - 1]]) {
        ilu[k - 1] = S[cols[k - 1]];
        S[cols[k - 1]] = 0.0;
        C[cols[k - 1]] = 0;
      }
    }
  }
  for (int i = 1; i <= n; ++i) {
    double &d = ilu[diag[i - 1] - 1];
    d = std::fabs(d) < AEPS ? 1.0 : 1.0 / d;
  }
}

// CRS_LUSolve non-Cholesky branch, CRSMatrix.src:3346-3364
extern "C" void orc_lusolve(int n, const int *rows, const int *cols, const int *diag,
                            const double *ilu, double *b) {
  for (int i = 1; i <= n; ++i) {
    double s = b[i - 1];
    for (int j = rows[i - 1]; j <= diag[i - 1] - 1; ++j) s = s - ilu[j - 1] * b[cols[j - 1] - 1];
    b[i - 1] = s;
  }
  for (int i = n; i >= 1; --i) {
    double s = b[i - 1];
    for (int j = diag[i - 1] + 1; j <= rows[i] - 1; ++j) s = s - ilu[j - 1] * b[cols[j - 1] - 1];
    b[i - 1] = ilu[diag[i - 1] - 1] * s;
  }
}

// InitializeILU1, CRSMatrix.src:2391-2497: row i keeps its own entries plus, for every
// original entry k < i of row i, the upper part of row k (the structure one elimination
// step fills); RowMin/RowMax bound the column scan as in the reference.
static void ilu1_step(int n, const std::vector<int> &rows, const std::vector<int> &cols,
                      const std::vector<int> &diag, std::vector<int> &irows, std::vector<int> &icols,
                      std::vector<int> &idiag) {
  std::vector<int> C(n + 1, 0);
  irows.assign(n + 1, 0);
  idiag.assign(n, 0);
  icols.clear();
  irows[0] = 1;
  for (int i = 1; i <= n; ++i) {
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) C[cols[k - 1]] = 1;
    const int rowmin = cols[rows[i - 1] - 1];
    int rowmax = cols[rows[i] - 2];
    for (int k = rowmin; k <= i - 1; ++k) {
      if (C[k] == 1) {
        for (int l = diag[k - 1] + 1; l <= rows[k] - 1; ++l) {
          const int j = cols[l - 1];
          if (C[j] == 0) {
            C[j] = 2;
            rowmax = std::max(rowmax, j);
          }
        }
      }
    }
    int j = irows[i - 1] - 1;
    for (int k = rowmin; k <= rowmax; ++k) {
      if (C[k] > 0) {
        j = j + 1;
        C[k] = 0;
        icols.push_back(k);
        if (k == i) idiag[i - 1] = j;
      }
    }
    irows[i] = j + 1;
  }
}

extern "C" long long orc_ilu_pattern(int n, const int *rows, const int *cols, const int *diag, int order,
                                     long long cap, int *ilu_rows, int *ilu_cols, int *ilu_diag) {
  std::vector<int> r(rows, rows + n + 1), c(cols, cols + (rows[n] - 1)), d(diag, diag + n);
  for (int round = 0; round < order; ++round) {  // CRS_IncompleteLU :2200-2218
    std::vector<int> ir, ic, id;
    ilu1_step(n, r, c, d, ir, ic, id);
    r.swap(ir);
    c.swap(ic);
    d.swap(id);
  }
  const long long nnz = (long long)r[n] - 1;
  if (cap >= nnz && ilu_rows && ilu_cols && ilu_diag) {
    std::copy(r.begin(), r.end(), ilu_rows);
    std::copy(c.begin(), c.end(), ilu_cols);
    std::copy(d.begin(), d.end(), ilu_diag);
  }
  return nnz;
}

// CRS_IncompleteLU LU branch, CRSMatrix.src:2312-2366, on the ILU structure
extern "C" void orc_iluk(int n, const int *rows, const int *cols, const double *values, const int *ilu_rows,
                         const int *ilu_cols, const int *ilu_diag, double *ilu) {
  std::vector<double> S(n + 1, 0.0);
  std::vector<char> C(n + 1, 0);
  for (int i = 1; i <= n; ++i) {
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) S[cols[k - 1]] = values[k - 1];
    for (int k = ilu_rows[i - 1]; k <= ilu_rows[i] - 1; ++k) C[ilu_cols[k - 1]] = 1;
    for (int m = ilu_rows[i - 1]; m <= ilu_diag[i - 1] - 1; ++m) {
      const int k = ilu_cols[m - 1];
      if (S[k] == 0.0) continue;
      if (std::fabs(ilu[ilu_diag[k - 1] - 1]) > AEPS) S[k] = S[k] / ilu[ilu_diag[k - 1] - 1];
      for (int l = ilu_diag[k - 1] + 1; l <= ilu_rows[k] - 1; ++l) {
        const int j = ilu_cols[l - 1];
        if (C[j]) S[j] = S[j] - S[k] * ilu[l - 1];
      }
    }
    for (int k = ilu_rows[i - 1]; k <= ilu_rows[i] - 1; ++k) {
      if (C[ilu_cols[k - 1]]) {
        ilu[k - 1] = S[ilu_cols[k - 1]];
        S[ilu_cols[k - 1]] = 0.0;
        C[ilu_cols[k - 1]] = 0;
      }
    }
  }
  for (int i = 1; i <= n; ++i) {
    double &dv = ilu[ilu_diag[i - 1] - 1];
    dv = std::fabs(dv) < AEPS ? 1.0 : 1.0 / dv;
  }
}

// CRS_ILUT / ComputeILUT, CRSMatrix.src:2849-3044.  Row i: the matrix row enters the dense
// row S with its flags C; k runs from the row's first column RowMin to i-1 over the flagged
// entries (fill included): S(k) /= u_kk (the U diagonal is still un-inverted while rows are
// factored), then every U entry j of ILU row k is flagged and S(j) -= S(k) * U(k,j)
// (:2944-2959: flags and updates do not test S(k) for zero).  The finished row keeps, in
// ascending column order, the entries with |S(k)| >= TOL * ||A(i,:)||_2 and the diagonal
// (:2961-2979).  Afterwards every U diagonal is inverted (1 if |u_ii| < AEPS, :3023-3030).
// Output 1-based; returns false if a row's diagonal never enters the factor.
static bool ilut_rows(int n, const int *rows, const int *cols, const double *values, double tol,
                      std::vector<int> &ir, std::vector<int> &ic, std::vector<int> &id, std::vector<double> &iv) {
  std::vector<double> S(n + 1, 0.0);
  std::vector<char> C(n + 1, 0);
  ir.assign(n + 1, 0);
  id.assign(n, 0);
  ic.clear();
  iv.clear();
  ir[0] = 1;
  for (int i = 1; i <= n; ++i) {
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) {
      C[cols[k - 1]] = 1;
      S[cols[k - 1]] = values[k - 1];
    }
    const int rowmin = cols[rows[i - 1] - 1];
    int rowmax = cols[rows[i] - 2];
    for (int k = rowmin; k <= i - 1; ++k) {
      if (!C[k]) continue;
      const double ukk = iv[id[k - 1] - 1];
      if (std::fabs(ukk) > AEPS) S[k] = S[k] / ukk;
      for (int l = id[k - 1] + 1; l <= ir[k] - 1; ++l) {
        const int j = ic[l - 1];
        if (!C[j]) {
          C[j] = 1;
          rowmax = std::max(rowmax, j);
        }
        S[j] = S[j] - S[k] * iv[l - 1];
      }
    }
    double sq = 0.0;
    for (int k = rows[i - 1]; k <= rows[i] - 1; ++k) sq = sq + std::fabs(values[k - 1]) * std::fabs(values[k - 1]);
    const double norma = std::sqrt(sq);
    bool has_diag = false;
    for (int k = rowmin; k <= rowmax; ++k) {
      if (!C[k]) continue;
      if (std::fabs(S[k]) >= tol * norma || k == i) {
        ic.push_back(k);
        iv.push_back(S[k]);
        if (k == i) {
          id[i - 1] = (int)ic.size();
          has_diag = true;
        }
      }
      S[k] = 0.0;
      C[k] = 0;
    }
    if (!has_diag) return false;
    ir[i] = (int)ic.size() + 1;
  }
  for (int i = 1; i <= n; ++i) {
    double &dv = iv[id[i - 1] - 1];
    dv = std::fabs(dv) < AEPS ? 1.0 : 1.0 / dv;
  }
  return true;
}

extern "C" long long orc_ilut(int n, const int *rows, const int *cols, const double *values, double tol,
                              long long cap, int *ilu_rows, int *ilu_cols, int *ilu_diag, double *ilu_values) {
  std::vector<int> ir, ic, id;
  std::vector<double> iv;
  if (!ilut_rows(n, rows, cols, values, tol, ir, ic, id, iv)) return -1;
  const long long nz = (long long)ic.size();
  if (cap >= nz && ilu_rows) {
    std::copy(ir.begin(), ir.end(), ilu_rows);
    std::copy(ic.begin(), ic.end(), ilu_cols);
    std::copy(id.begin(), id.end(), ilu_diag);
    std::copy(iv.begin(), iv.end(), ilu_values);
  }
  return nz;
}

extern "C" int orc_lower_levels(int n, const int *rows, const int *cols, const int *diag, int *level) {
  int maxl = 0;
  for (int i = 1; i <= n; ++i) {
    int l = 0;
    for (int j = rows[i - 1]; j <= diag[i - 1] - 1; ++j) l = std::max(l, level[cols[j - 1] - 1] + 1);
    level[i - 1] = l;
    maxl = std::max(maxl, l);
  }
  return maxl + 1;
}

// ComputeNorm default branch, SolverUtils.src:4983-4988: sqrt(sum(x^2)/n)
extern "C" double orc_compute_norm(int n, const double *x) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + x[i] * x[i];
  return std::sqrt(s / n);
}

namespace {

struct Ctx {
  int n;
  const int *rows, *cols, *diag;
  const double *values;
  const double *ilu;
  int precond;
  int threads;
  const int *irows, *icols, *idiag;  // ILU structure (the matrix's for ILU0)
};

// Threads for the vector operations (BLAS-1 and the elementwise updates) of the solve in
// flight: 0 runs them serially, as the vendored netlib BLAS does (the checker's setting);
// t > 0 splits every loop into t static chunks, as a threaded BLAS would (the timed CPU
// baseline's setting).  Dot products then sum each chunk serially and the chunk sums in chunk
// order, so the result is deterministic for a given t.
thread_local int t_blas_threads = 0;

double dot(int n, const double *x, const double *y) {  // ddot, restated as a plain sum
  const int t = t_blas_threads;
  if (t <= 1) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = s + x[i] * y[i];
    return s;
  }
  std::vector<double> part(t, 0.0);
#pragma omp parallel for num_threads(t) schedule(static, 1)
  for (int c = 0; c < t; ++c) {
    const long long lo = (long long)n * c / t, hi = (long long)n * (c + 1) / t;
    double s = 0.0;
    for (long long i = lo; i < hi; ++i) s = s + x[i] * y[i];
    part[c] = s;
  }
  double s = 0.0;
  for (int c = 0; c < t; ++c) s = s + part[c];
  return s;
}
double nrm2(int n, const double *x) {  // dnrm2, restated as sqrt of the plain sum of squares
  return std::sqrt(dot(n, x, x));
}

// an elementwise vector update f(i) for i in [0, n), on t_blas_threads threads
template <typename F>
void vec_loop(int n, F &&f) {
  const int t = t_blas_threads;
#pragma omp parallel for num_threads(t > 1 ? t : 1) schedule(static) if (t > 1)
  for (int i = 0; i < n; ++i) f(i);
}

void matvec(const Ctx &c, const double *u, double *v) {
  orc_spmv(c.n, c.rows, c.cols, c.values, u, v, c.threads);
}

// pcondlsubr: CRS_LUPrecondition (CRSMatrix.src:3259-3270) = copy + CRS_LUSolve;
// CRS_DiagPrecondition (:1467-1510); pcond_dummy = copy.
void pcond(const Ctx &c, double *u, const double *v) {
  const int n = c.n;
  if (c.precond == ORC_PREC_ILU0) {
    vec_loop(n, [&](int i) { u[i] = v[i]; });
    orc_lusolve(n, c.irows, c.icols, c.idiag, c.ilu, u);
  } else if (c.precond == ORC_PREC_DIAGONAL) {
    vec_loop(n, [&](int i) {
      double d = c.values[c.diag[i] - 1];
      u[i] = std::fabs(d) > AEPS ? v[i] / d : v[i];
    });
  } else {
    vec_loop(n, [&](int i) { u[i] = v[i]; });
  }
}

// huti_dcgsolv, hutiter/src/huti_cg_D.F90:84-257 (stop test HUTI_TRESID_SCALED_BYB)
int huti_cg(const Ctx &c, double *X, const double *B, int maxit, double tol, int *iters,
            double *resid) {
  const int n = c.n;
  std::vector<double> R(n), Z(n), P(n), Q(n);
  int iter_count = 1;
  double rhsnorm = nrm2(n, B);
  double rho = 0, oldrho = 1, alpha, beta, residual = 0;
  int info = 0;
  matvec(c, X, R.data());
  vec_loop(n, [&](int i) { R[i] = B[i] - R[i]; });
  while (true) {
    pcond(c, Q.data(), R.data());
    vec_loop(n, [&](int i) { Z[i] = Q[i]; });  // pcondrsubr = dummy copy
    rho = dot(n, R.data(), Z.data());
    if (rho == 0) {
      info = HUTI_CG_RHO;
      break;
    }
    if (iter_count == 1) {
      vec_loop(n, [&](int i) { P[i] = Z[i]; });
    } else {
      beta = rho / oldrho;
      vec_loop(n, [&](int i) { P[i] = Z[i] + beta * P[i]; });
    }
    matvec(c, P.data(), Q.data());
    alpha = rho / dot(n, P.data(), Q.data());
    vec_loop(n, [&](int i) { X[i] = X[i] + alpha * P[i]; });
    vec_loop(n, [&](int i) { R[i] = R[i] - alpha * Q[i]; });
    matvec(c, X, Z.data());
    vec_loop(n, [&](int i) { Z[i] = Z[i] - B[i]; });
    residual = nrm2(n, Z.data()) / rhsnorm;
    if (residual < tol) {
      info = HUTI_CONVERGENCE;
      break;
    }
    oldrho = rho;
    iter_count++;
    if (iter_count > maxit) {
      info = HUTI_MAXITER;
      break;
    }
  }
  *iters = iter_count;
  *resid = residual;
  return info;
}

// huti_dbicgstabsolv, hutiter/src/huti_bicgstab_D.F90:96-284 (stop HUTI_TRESID_SCALED_BYB)
int huti_bicgstab(const Ctx &c, double *X, const double *B, int maxit, double tol, int *iters,
                  double *resid) {
  const int n = c.n;
  std::vector<double> R(n), RTLD(n), P(n), V(n), T(n), T1V(n), T2V(n), S(n);
  int iter_count = 1;
  double rhsnorm = nrm2(n, B);
  double rho, oldrho = 1, omega = 1, alpha = 0, beta, residual = 0;
  int info = 0;
  matvec(c, X, R.data());
  vec_loop(n, [&](int i) { R[i] = B[i] - R[i]; });
  RTLD = R;
  std::fill(P.begin(), P.end(), 0.0);
  std::fill(V.begin(), V.end(), 0.0);
  while (true) {
    rho = dot(n, RTLD.data(), R.data());
    if (rho == 0) {
      info = HUTI_BICGSTAB_RHO;
      break;
    }
    beta = (rho * alpha) / (oldrho * omega);
    vec_loop(n, [&](int i) { P[i] = R[i] + beta * (P[i] - omega * V[i]); });
    pcond(c, V.data(), P.data());
    vec_loop(n, [&](int i) { T1V[i] = V[i]; });
    matvec(c, T1V.data(), V.data());
    alpha = rho / dot(n, RTLD.data(), V.data());
    vec_loop(n, [&](int i) { S[i] = R[i] - alpha * V[i]; });
    residual = nrm2(n, S.data());
    if (residual < HUTI_EPSILON) {
      vec_loop(n, [&](int i) { X[i] = X[i] + alpha * T1V[i]; });
      info = HUTI_BICGSTAB_SNORM;
      break;
    }
    pcond(c, T.data(), S.data());
    vec_loop(n, [&](int i) { T2V[i] = T[i]; });
    matvec(c, T2V.data(), T.data());
    omega = dot(n, T.data(), S.data()) / dot(n, T.data(), T.data());
    vec_loop(n, [&](int i) { X[i] = X[i] + alpha * T1V[i] + omega * T2V[i]; });
    vec_loop(n, [&](int i) { R[i] = S[i] - omega * T[i]; });
    matvec(c, X, T2V.data());
    vec_loop(n, [&](int i) { T1V[i] = T2V[i] - B[i]; });
    residual = nrm2(n, T1V.data()) / rhsnorm;
    if (residual < tol) {
      info = HUTI_CONVERGENCE;
      break;
    }
    if (omega == 0) {
      info = HUTI_BICGSTAB_OMEGA;
      break;
    }
    oldrho = rho;
    iter_count++;
    if (iter_count > maxit) {
      info = HUTI_MAXITER;
      break;
    }
  }
  *iters = iter_count;
  *resid = residual;
  return info;
}

// GCR with restart m, IterativeMethods.src:919-1055 (preconditioned search directions
// T1 = M^-1 r, modified Gram-Schmidt of A T1 against the stored ones, recursive residual
// stopping test ||r|| / ||b|| < tol)
int gcr(const Ctx &c, double *x, const double *b, int rounds, double tol, double maxtol, int m, int *iters,
        double *resid) {
  const int n = c.n;
  std::vector<double> r(n), T1(n), T2(n);
  std::vector<std::vector<double>> S(std::max(0, m - 1), std::vector<double>(n, 0.0)),
      V(std::max(0, m - 1), std::vector<double>(n, 0.0));
  matvec(c, x, r.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  const double bnorm = nrm2(n, b);
  double rnorm = nrm2(n, r.data());
  double residual = rnorm / bnorm;
  *iters = 0;
  *resid = residual;
  if (residual < tol) return HUTI_CONVERGENCE;
  if (residual > maxtol || residual != residual) return HUTI_DIVERGENCE;  // :959-961
  for (int k = 1; k <= rounds; ++k) {
    int j;
    if (k % m == 0) {
      j = m;
    } else {
      j = k % m;
      if (j == 1 && k > 1) {  // true residual at a restart
        matvec(c, x, r.data());
        for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
      }
    }
    pcond(c, T1.data(), r.data());
    matvec(c, T1.data(), T2.data());
    for (int i = 1; i <= j - 1; ++i) {
      const double beta = dot(n, V[i - 1].data(), T2.data());
      for (int t = 0; t < n; ++t) T1[t] = T1[t] - beta * S[i - 1][t];
      for (int t = 0; t < n; ++t) T2[t] = T2[t] - beta * V[i - 1][t];
    }
    const double alpha = nrm2(n, T2.data());
    for (int t = 0; t < n; ++t) T1[t] = 1.0 / alpha * T1[t];
    for (int t = 0; t < n; ++t) T2[t] = 1.0 / alpha * T2[t];
    const double beta = dot(n, T2.data(), r.data());
    for (int t = 0; t < n; ++t) x[t] = x[t] + beta * T1[t];
    for (int t = 0; t < n; ++t) r[t] = r[t] - beta * T2[t];
    if (j != m) {
      S[j - 1] = T1;
      V[j - 1] = T2;
    }
    rnorm = nrm2(n, r.data());
    residual = rnorm / bnorm;
    *iters = k;
    *resid = residual;
    if (residual < tol) return HUTI_CONVERGENCE;
    if (residual > maxtol || residual != residual) return HUTI_DIVERGENCE;  // :1047-1048
  }
  return HUTI_MAXITER;
}

// LU with partial pivoting of a small dense column-major matrix (dgetrf) and the solve with
// it (dgetrs 'n'), as RealBiCGStabl calls them on its (l-1) x (l-1) block
void small_lu(int m, double *a, int lda, int *piv) {
  for (int k = 0; k < m; ++k) {
    int p = k;
    for (int i = k + 1; i < m; ++i)
      if (std::fabs(a[i + k * lda]) > std::fabs(a[p + k * lda])) p = i;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < m; ++j) std::swap(a[k + j * lda], a[p + j * lda]);
    if (a[k + k * lda] != 0.0)
      for (int i = k + 1; i < m; ++i) a[i + k * lda] = a[i + k * lda] / a[k + k * lda];
    for (int j = k + 1; j < m; ++j)
      for (int i = k + 1; i < m; ++i) a[i + j * lda] = a[i + j * lda] - a[i + k * lda] * a[k + j * lda];
  }
}
void small_lu_solve(int m, const double *a, int lda, const int *piv, double *bv) {
  for (int k = 0; k < m; ++k)
    if (piv[k] != k) std::swap(bv[k], bv[piv[k]]);
  for (int k = 0; k < m; ++k)
    for (int i = k + 1; i < m; ++i) bv[i] = bv[i] - a[i + k * lda] * bv[k];
  for (int k = m - 1; k >= 0; --k) {
    bv[k] = bv[k] / a[k + k * lda];
    for (int i = 0; i < k; ++i) bv[i] = bv[i] - a[i + k * lda] * bv[k];
  }
}

// BiCGStab(l), IterativeMethods.src:559-834 (right preconditioned, convex polynomial part,
// reliable residual / solution updates with delta = 1e-2; stop on the recursive residual)
int bicgstabl(const Ctx &c, double *x_out, const double *b, int max_rounds, double tol, double maxtol, int l, int *iters,
              double *resid) {
  const int n = c.n;
  const double delta = 1.0e-2;
  std::vector<double> x(x_out, x_out + n), t(n, 0.0), rr(n), xp(n), bp(n);
  std::vector<std::vector<double>> r(l + 1, std::vector<double>(n, 0.0)), u(l + 1, std::vector<double>(n, 0.0));
  bool all_zero = true;
  for (int i = 0; i < n; ++i)
    if (x[i] != 0.0) all_zero = false;
  if (all_zero) x.assign(b, b + n);
  matvec(c, x.data(), r[0].data());
  for (int i = 0; i < n; ++i) r[0][i] = b[i] - r[0][i];
  const double bnrm = nrm2(n, b);
  const double rnrm0 = nrm2(n, r[0].data());
  double errorind = rnrm0 / bnrm;
  *iters = 0;
  *resid = errorind;
  if (errorind < tol) return HUTI_CONVERGENCE;
  if (errorind > maxtol) return HUTI_DIVERGENCE;  // IterativeMethods.src:626-629
  rr = r[0];
  bp = r[0];
  xp = x;
  double rnrm = rnrm0, mxnrmx = rnrm0, mxnrmr = rnrm0;
  std::fill(x.begin(), x.end(), 0.0);
  double alpha = 0.0, omega = 1.0, sigma = 1.0, rho0 = 1.0, rho1 = 0.0, beta = 0.0;
  const int L1 = l + 1;
  std::vector<double> Z(L1 * L1), ZZ(L1 * L1), y0(L1), yl(L1), y(L1);
  std::vector<int> piv(std::max(1, l - 1));
  auto symv = [&](const std::vector<double> &v, std::vector<double> &out) {
    for (int i = 0; i < L1; ++i) {
      double s = 0.0;
      for (int j = 0; j < L1; ++j) s = s + Z[i + j * L1] * v[j];
      out[i] = s;
    }
  };
  auto small_dot = [&](const std::vector<double> &a, const std::vector<double> &bb) {
    double s = 0.0;
    for (int i = 0; i < L1; ++i) s = s + a[i] * bb[i];
    return s;
  };
  int round = 0, info = HUTI_MAXITER;
  bool early = false;
  for (round = 1; round <= max_rounds; ++round) {
    // --- the BiCG part
    rho0 = -omega * rho0;
    for (int k = 1; k <= l; ++k) {
      rho1 = dot(n, rr.data(), r[k - 1].data());
      if (rho0 == 0.0 || rho1 != rho1) { info = HUTI_DIVERGENCE; early = true; break; }
      beta = alpha * (rho1 / rho0);
      rho0 = rho1;
      for (int j = 0; j <= k - 1; ++j)
        for (int i = 0; i < n; ++i) u[j][i] = r[j][i] - beta * u[j][i];
      pcond(c, t.data(), u[k - 1].data());
      matvec(c, t.data(), u[k].data());
      sigma = dot(n, rr.data(), u[k].data());
      if (sigma == 0.0 || sigma != sigma) { info = HUTI_DIVERGENCE; early = true; break; }
      alpha = rho1 / sigma;
      for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * u[0][i];
      for (int j = 0; j <= k - 1; ++j)
        for (int i = 0; i < n; ++i) r[j][i] = r[j][i] - alpha * u[j + 1][i];
      pcond(c, t.data(), r[k - 1].data());
      matvec(c, t.data(), r[k].data());
      rnrm = nrm2(n, r[0].data());
      mxnrmx = std::max(mxnrmx, rnrm);
      mxnrmr = std::max(mxnrmr, rnrm);
      errorind = rnrm / bnrm;
      if (errorind < tol) { info = HUTI_CONVERGENCE; early = true; break; }
      if (errorind != errorind) { info = HUTI_DIVERGENCE; early = true; break; }
    }
    if (early) break;
    // --- the convex polynomial part
    for (int i = 0; i < L1; ++i)
      for (int j = 0; j <= i; ++j) Z[i + j * L1] = dot(n, r[i].data(), r[j].data());
    for (int j = 1; j < L1; ++j)
      for (int i = 0; i < j; ++i) Z[i + j * L1] = Z[j + i * L1];
    ZZ = Z;
    // the (l-1) x (l-1) block rows/cols 2..l of ZZ
    std::vector<double> M((l - 1) * (l - 1));
    for (int j = 0; j < l - 1; ++j)
      for (int i = 0; i < l - 1; ++i) M[i + j * (l - 1)] = ZZ[(i + 1) + (j + 1) * L1];
    if (l > 1) small_lu(l - 1, M.data(), l - 1, piv.data());
    y0[0] = -1.0;
    for (int i = 1; i < l; ++i) y0[i] = Z[i + 0 * L1];
    if (l > 1) small_lu_solve(l - 1, M.data(), l - 1, piv.data(), &y0[1]);
    y0[l] = 0.0;
    yl[0] = 0.0;
    for (int i = 1; i < l; ++i) yl[i] = Z[i + l * L1];
    if (l > 1) small_lu_solve(l - 1, M.data(), l - 1, piv.data(), &yl[1]);
    yl[l] = -1.0;
    symv(y0, y);
    const double kappa0 = std::sqrt(small_dot(y0, y));
    symv(yl, y);
    const double kappal = std::sqrt(small_dot(yl, y));
    symv(y0, y);
    const double varrho = small_dot(yl, y) / (kappa0 * kappal);
    const double hatgamma = varrho / std::fabs(varrho) * std::max(std::fabs(varrho), 7e-1) * kappa0 / kappal;
    for (int i = 0; i < L1; ++i) y0[i] = y0[i] - hatgamma * yl[i];
    // --- update
    omega = y0[l];
    for (int j = 1; j <= l; ++j) {
      for (int i = 0; i < n; ++i) u[0][i] = u[0][i] - y0[j] * u[j][i];
      for (int i = 0; i < n; ++i) x[i] = x[i] + y0[j] * r[j - 1][i];
      for (int i = 0; i < n; ++i) r[0][i] = r[0][i] - y0[j] * r[j][i];
    }
    symv(y0, y);
    rnrm = std::sqrt(small_dot(y0, y));
    // --- the reliable update part
    mxnrmx = std::max(mxnrmx, rnrm);
    mxnrmr = std::max(mxnrmr, rnrm);
    const bool xpdt = rnrm < delta * rnrm0 && rnrm0 < mxnrmx;
    const bool rcmp = (rnrm < delta * mxnrmr && rnrm0 < mxnrmr) || xpdt;
    if (rcmp) {
      pcond(c, t.data(), x.data());
      matvec(c, t.data(), r[0].data());
      for (int i = 0; i < n; ++i) r[0][i] = bp[i] - r[0][i];
      mxnrmr = rnrm;
      if (xpdt) {
        for (int i = 0; i < n; ++i) xp[i] = xp[i] + t[i];
        std::fill(x.begin(), x.end(), 0.0);
        bp = r[0];
        mxnrmx = rnrm;
      }
    }
    errorind = rnrm / bnrm;
    if (errorind < tol) { info = HUTI_CONVERGENCE; break; }
    if (errorind > maxtol || errorind != errorind) { info = HUTI_DIVERGENCE; break; }  // :817-819
  }
  *iters = std::min(round, max_rounds);
  *resid = errorind;
  // x = M^-1 x + xp
  t = x;
  pcond(c, x.data(), t.data());
  for (int i = 0; i < n; ++i) x_out[i] = x[i] + xp[i];
  return info;
}

}  // namespace

// SolveLinearSystem (SolverUtils.src:7151-7525) for Linear System Solver = Iterative:
// zero-rhs short cut (:7309-7320), ScaleLinearSystem (:7344-7352), IterSolver
// (IterSolve.src:144-798: x=1e-8 when all zero :358-359, ILU0 factorization :575,
// HUTI call :774-778), BackScaleLinearSystem (:7446-7452).
extern "C" int orc_solve(int n, const int *rows, const int *cols, const int *diag,
                         const double *values_in, const double *b_in, double *x,
                         const orc_params *prm, orc_result *res) {
  orc_result r{};
  std::vector<double> values(values_in, values_in + (size_t)(rows[n] - 1));
  std::vector<double> b(b_in, b_in + n);
  double bnorm = 0.0;
  for (int i = 0; i < n; ++i) bnorm = bnorm + b[i] * b[i];
  bnorm = std::sqrt(bnorm);
  if (bnorm <= TINY_DP) {
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    r.info = HUTI_CONVERGENCE;
    if (res) *res = r;
    return r.info;
  }
  double t0 = now();
  std::vector<double> D(n);
  double rs = 1.0;
  if (prm->scale_system)
    orc_scale(n, rows, cols, diag, values.data(), b.data(), x, D.data(), &rs, 1);
  bool all_zero = true;
  for (int i = 0; i < n; ++i)
    if (x[i] != 0.0) all_zero = false;
  if (all_zero)
    for (int i = 0; i < n; ++i) x[i] = 1.0e-8;

  std::vector<double> ilu;
  std::vector<int> ir, ic, id;
  const int *irows = rows, *icols = cols, *idiag = diag;
  double tp = now();
  if (prm->precond == ORC_PREC_ILU0 && prm->ilu_order > 0) {  // ILU(n), CRS_IncompleteLU(A,n)
    const long long nz = orc_ilu_pattern(n, rows, cols, diag, prm->ilu_order, 0, nullptr, nullptr, nullptr);
    ir.resize(n + 1);
    ic.resize(nz);
    id.resize(n);
    orc_ilu_pattern(n, rows, cols, diag, prm->ilu_order, nz, ir.data(), ic.data(), id.data());
    irows = ir.data();
    icols = ic.data();
    idiag = id.data();
    ilu.assign(nz, 0.0);
    orc_iluk(n, rows, cols, values.data(), irows, icols, idiag, ilu.data());
  } else if (prm->precond == ORC_PREC_ILU0 && prm->nblocks > 1 && prm->block_starts) {
    // block-Jacobi ILU0: the matrix restricted to its diagonal blocks, factored whole (the
    // blocks are independent, so this equals factoring each block on its own)
    std::vector<int> blk(n);
    for (int k = 0; k < prm->nblocks; ++k)
      for (int i = prm->block_starts[k]; i < prm->block_starts[k + 1]; ++i) blk[i] = k;
    ir.assign(n + 1, 1);
    id.assign(n, 0);
    std::vector<double> bv;
    for (int i = 0; i < n; ++i) {
      for (int j = rows[i] - 1; j < rows[i + 1] - 1; ++j) {
        const int c = cols[j] - 1;
        if (blk[c] != blk[i]) continue;
        if (c == i) id[i] = (int)ic.size() + 1;
        ic.push_back(c + 1);
        bv.push_back(values[j]);
      }
      ir[i + 1] = (int)ic.size() + 1;
    }
    irows = ir.data();
    icols = ic.data();
    idiag = id.data();
    ilu.assign(bv.size(), 0.0);
    orc_ilu0(n, irows, icols, idiag, bv.data(), ilu.data());
  } else if (prm->precond == ORC_PREC_ILU0) {
    ilu.assign(values.size(), 0.0);
    orc_ilu0(n, rows, cols, diag, values.data(), ilu.data());
  } else if (prm->precond == ORC_PREC_ILUT) {  // CRS_ILUT(A, Linear System ILUT Tolerance)
    if (!ilut_rows(n, rows, cols, values.data(), prm->ilut_tol, ir, ic, id, ilu)) return -1;
    irows = ir.data();
    icols = ic.data();
    idiag = id.data();
  }
  r.seconds_precond_setup = now() - tp;
  // ILUT is applied by the same CRS_LUPrecondition as ILU(n), on its own structure
  const int apply = prm->precond == ORC_PREC_ILUT ? ORC_PREC_ILU0 : prm->precond;
  Ctx c{n, rows, cols, diag, values.data(), ilu.empty() ? nullptr : ilu.data(), apply,
        prm->omp_threads, irows, icols, idiag};
  struct BlasThreads {  // the vector operations' thread count for this solve only
    int saved;
    explicit BlasThreads(int t) : saved(t_blas_threads) { t_blas_threads = t > 0 ? t : 0; }
    ~BlasThreads() { t_blas_threads = saved; }
  } blas_threads_scope(prm->blas_threads);
  // HUTI_MAXTOLERANCE: Linear System Divergence Tolerance, HUGE when absent (IterSolve.src:364-366)
  const double maxtol = prm->divtol > 0.0 ? prm->divtol : std::numeric_limits<double>::max();
  if (prm->method == ORC_CG)
    r.info = huti_cg(c, x, b.data(), prm->max_iter, prm->tol, &r.iters, &r.residual);
  else if (prm->method == ORC_GCR)  // restart: Linear System GCR Restart, else Max Iterations
    r.info = gcr(c, x, b.data(), prm->max_iter, prm->tol, maxtol, prm->restart > 0 ? prm->restart : prm->max_iter,
                 &r.iters, &r.residual);
  else if (prm->method == ORC_BICGSTABL)  // BiCGstabl polynomial degree, default 2
    r.info = bicgstabl(c, x, b.data(), prm->max_iter, prm->tol, maxtol, prm->restart >= 2 ? prm->restart : 2,
                       &r.iters, &r.residual);
  else
    r.info = huti_bicgstab(c, x, b.data(), prm->max_iter, prm->tol, &r.iters, &r.residual);
  if (prm->scale_system) backscale(n, rows, cols, values.data(), b.data(), x, D.data(), rs);
  r.seconds_solve = now() - t0;
  if (res) *res = r;
  return r.info;
}
