// egpu_assembly.cu -- element assembly into the CRS matrix on the device.
//
// Replaces the bulk element loops of HeatSolve (modules/HeatSolve.src:655-985) and
// StressSolve (modules/StressSolve.src:815-1072) for linear isotropic diffusion and
// isotropic elasticity.  One warp computes one element: lanes < ngauss evaluate the
// geometry of one integration point each (ElementInfo / ElementMetric,
// ElementDescription.src:2586-3320, 6757-6884) into shared memory, then all lanes form
// the element matrix entries and add them to precomputed CRS positions.  Elements of one
// colour share no node, so the scatter needs no atomics; colours run one after another.
#include <algorithm>
#include <cmath>
#include <vector>

#include "egpu_internal.cuh"
#include "egpu_solve.h"

int egpu_color_elements(int nnodes, int nelem, int nen, const int *elem_nodes, std::vector<int> &color_of);

namespace egpu {

// reference element data: quadrature (Integration.src:281-295, 1446-1486, 84-91) and
// nodal basis (elements.def 808 :606-643, 504 :365-404, 303 :155-185)
template <int CODE>
struct Ref;

template <>
struct Ref<808> {
  static constexpr int NEN = 8, NGP = 8, DIM = 3;
  __device__ static void gp(int t, double &u, double &v, double &w, double &s) {
    const double a = 0.57735026918962576451;  // 1/sqrt(3)
    const int i = t >> 2, j = (t >> 1) & 1, k = t & 1;
    u = k ? a : -a;
    v = j ? a : -a;
    w = i ? a : -a;
    s = 1.0;
  }
  __device__ static void basis(double u, double v, double w, double *N, double (*dN)[3]) {
    const double nu[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const double nv[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const double nw[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const double a = 1.0 + nu[p] * u, b = 1.0 + nv[p] * v, c = 1.0 + nw[p] * w;
      N[p] = 0.125 * a * b * c;
      dN[p][0] = 0.125 * nu[p] * b * c;
      dN[p][1] = 0.125 * nv[p] * a * c;
      dN[p][2] = 0.125 * nw[p] * a * b;
    }
  }
};

template <>
struct Ref<504> {
  static constexpr int NEN = 4, NGP = 4, DIM = 3;
  __device__ static void gp(int t, double &u, double &v, double &w, double &s) {
    const double U[4] = {0.1757281246520584, 0.2445310270213291, 0.5556470949048655, 0.0240937534217468};
    const double V[4] = {0.5656137776620919, 0.0501800797762026, 0.1487681308666864, 0.2354380116950194};
    const double W[4] = {0.2180665126782654, 0.5635595064952189, 0.0350112499848832, 0.1833627308416330};
    u = U[t];
    v = V[t];
    w = W[t];
    s = 0.25 / 6.0;
  }
  __device__ static void basis(double u, double v, double w, double *N, double (*dN)[3]) {
    N[0] = 1.0 - u - v - w;
    N[1] = u;
    N[2] = v;
    N[3] = w;
    const double d[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int i = 0; i < 3; ++i) dN[p][i] = d[p][i];
  }
};

template <>
struct Ref<303> {
  static constexpr int NEN = 3, NGP = 3, DIM = 2;
  __device__ static void gp(int t, double &u, double &v, double &w, double &s) {
    const double U[3] = {0.16666666666666667, 0.66666666666666667, 0.16666666666666667};
    const double V[3] = {0.16666666666666667, 0.16666666666666667, 0.66666666666666667};
    u = U[t];
    v = V[t];
    w = 0.0;
    s = 0.33333333333333333 / 2.0;
  }
  __device__ static void basis(double u, double v, double, double *N, double (*dN)[3]) {
    N[0] = 1.0 - u - v;
    N[1] = u;
    N[2] = v;
    const double d[3][3] = {{-1, -1, 0}, {1, 0, 0}, {0, 1, 0}};
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int i = 0; i < 3; ++i) dN[p][i] = d[p][i];
  }
};

// geometry of one integration point: dBdx (NEN x 3), detJ*weight.  Returns false for a
// degenerate element (ElementMetric's DetG <= TINY test).
template <int CODE>
__device__ bool gp_geometry(int t, const double (*X)[3], int cdim, double *N, double (*dB)[3], double &s) {
  using R = Ref<CODE>;
  constexpr int NEN = R::NEN, DIM = R::DIM;
  double u, v, w, wt;
  R::gp(t, u, v, w, wt);
  double dN[NEN][3];
  R::basis(u, v, w, N, dN);
  double dx[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double acc = 0.0;
      if (i < DIM)
#pragma unroll
        for (int p = 0; p < NEN; ++p) acc += X[p][c] * dN[p][i];
      dx[c][i] = acc;
    }
  double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, GI[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int i = 0; i < DIM; ++i)
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      double acc = 0.0;
      for (int k = 0; k < cdim; ++k) acc += dx[k][i] * dx[k][j];
      G[i][j] = acc;
    }
  double detG;
  if (DIM == 2) {
    detG = G[0][0] * G[1][1] - G[0][1] * G[1][0];
    if (detG <= EGPU_TINY_DP) return false;
    GI[0][0] = G[1][1] / detG;
    GI[0][1] = -G[0][1] / detG;
    GI[1][0] = -G[1][0] / detG;
    GI[1][1] = G[0][0] / detG;
  } else {
    detG = G[0][0] * (G[1][1] * G[2][2] - G[1][2] * G[2][1]) + G[0][1] * (G[1][2] * G[2][0] - G[1][0] * G[2][2]) +
           G[0][2] * (G[1][0] * G[2][1] - G[1][1] * G[2][0]);
    if (detG <= EGPU_TINY_DP) return false;
    const double q = 1.0 / detG;
    GI[0][0] = q * (G[1][1] * G[2][2] - G[2][1] * G[1][2]);
    GI[1][0] = -q * (G[1][0] * G[2][2] - G[2][0] * G[1][2]);
    GI[2][0] = q * (G[1][0] * G[2][1] - G[2][0] * G[1][1]);
    GI[0][1] = -q * (G[0][1] * G[2][2] - G[2][1] * G[0][2]);
    GI[1][1] = q * (G[0][0] * G[2][2] - G[2][0] * G[0][2]);
    GI[2][1] = -q * (G[0][0] * G[2][1] - G[2][0] * G[0][1]);
    GI[0][2] = q * (G[0][1] * G[1][2] - G[1][1] * G[0][2]);
    GI[1][2] = -q * (G[0][0] * G[1][2] - G[1][0] * G[0][2]);
    GI[2][2] = q * (G[0][0] * G[1][1] - G[1][0] * G[0][1]);
  }
  s = sqrt(detG) * wt;
  double L[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) acc += dx[i][k] * GI[k][j];
      L[i][j] = acc;
    }
#pragma unroll
  for (int p = 0; p < NEN; ++p)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      if (j < cdim)
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc += dN[p][k] * L[j][k];
      dB[p][j] = acc;
    }
  return true;
}

constexpr int ASM_WARPS = 8;

// Diffusion: K_pq = sum_t s_t k_t dN_q.dN_p, f_p = sum_t s_t (sum_m load_m N_m) N_p
// (DiffuseConvectiveAnisotropic.src:334-344, 515-561, 569-612)
template <int CODE>
__global__ void __launch_bounds__(ASM_WARPS * 32, 3) k_assemble_poisson(
    int ne, const int *__restrict__ elist, const int *__restrict__ enodes, const double *__restrict__ xyz,
    int cdim, const double *__restrict__ elem_k, const double *__restrict__ nodal_k,
    const double *__restrict__ load, const int *__restrict__ perm, const int *__restrict__ slots,
    double *__restrict__ values, double *__restrict__ rhs) {
  using R = Ref<CODE>;
  constexpr int NEN = R::NEN, NGP = R::NGP;
  __shared__ double sh_dB[ASM_WARPS][NGP][NEN][3];
  __shared__ double sh_N[ASM_WARPS][NGP][NEN];
  __shared__ double sh_s[ASM_WARPS][NGP], sh_k[ASM_WARPS][NGP], sh_f[ASM_WARPS][NGP];
  // the element's node coordinates and nodal k / load, staged once per warp (lane p holds
  // node p's) instead of in every lane's registers
  __shared__ double sh_X[ASM_WARPS][NEN][3], sh_kn[ASM_WARPS][NEN], sh_ln[ASM_WARPS][NEN];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * ASM_WARPS + wib;
  if (w >= ne) return;
  const int e = elist[w];
  int node = 0;
  if (lane < NEN) {
    node = enodes[(size_t)e * NEN + lane];
    sh_kn[wib][lane] = elem_k ? elem_k[e] : (nodal_k ? nodal_k[node] : 1.0);
    sh_ln[wib][lane] = load ? load[node] : 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) sh_X[wib][lane][c] = xyz[(size_t)node * 3 + c];
  }
  __syncwarp();
  if (lane < NGP) {
    double N[NEN], dB[NEN][3], s;
    const bool ok = gp_geometry<CODE>(lane, sh_X[wib], cdim, N, dB, s);
    double kk = 0.0, ff = 0.0;
#pragma unroll
    for (int p = 0; p < NEN; ++p) {
      kk += sh_kn[wib][p] * N[p];
      ff += sh_ln[wib][p] * N[p];
    }
    sh_s[wib][lane] = ok ? s : 0.0;
    sh_k[wib][lane] = kk;
    sh_f[wib][lane] = ff;
#pragma unroll
    for (int p = 0; p < NEN; ++p) {
      sh_N[wib][lane][p] = N[p];
#pragma unroll
      for (int i = 0; i < 3; ++i) sh_dB[wib][lane][p][i] = dB[p][i];
    }
  }
  __syncwarp();
  const int *sl = slots + (size_t)e * NEN * NEN;
  for (int idx = lane; idx < NEN * NEN; idx += 32) {
    const int p = idx / NEN, q = idx % NEN;
    double K = 0.0;
#pragma unroll
    for (int t = 0; t < NGP; ++t) {
      double A = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i) A += sh_k[wib][t] * sh_dB[wib][t][q][i] * sh_dB[wib][t][p][i];
      K += sh_s[wib][t] * A;
    }
    const int slot = sl[idx];
    if (slot >= 0) values[slot] += K;
  }
  if (lane < NEN) {
    double F = 0.0;
#pragma unroll
    for (int t = 0; t < NGP; ++t) F += sh_s[wib][t] * (sh_f[wib][t] * sh_N[wib][t][lane]);
    const int r = perm[node];
    if (r >= 0) rhs[r] += F;
  }
}

// Isotropic elasticity (Stress.src:260-273, 366-439, 476-515): with c12 = E nu/((1+nu)(1-2nu)),
// c44 = E (1/2-nu)/((1+nu)(1-2nu)) the product G_p C B_q collapses to
//   K_(p,i),(q,j) = c12 a_i b_j + c44 (a_j b_i + delta_ij a.b),  a = dN_p/dx, b = dN_q/dx,
// which is already symmetric, so the reference's (K+K^T)/2 leaves it unchanged.
template <int CODE>
__global__ void __launch_bounds__(ASM_WARPS * 32) k_assemble_elastic(
    int ne, const int *__restrict__ elist, const int *__restrict__ enodes, const double *__restrict__ xyz,
    double c12, double c44, double bf0, double bf1, double bf2, const int *__restrict__ perm,
    const int *__restrict__ slots, double *__restrict__ values, double *__restrict__ rhs) {
  using R = Ref<CODE>;
  constexpr int NEN = R::NEN, NGP = R::NGP, ND = 3 * NEN;
  __shared__ double sh_dB[ASM_WARPS][NGP][NEN][3];
  __shared__ double sh_N[ASM_WARPS][NGP][NEN];
  __shared__ double sh_s[ASM_WARPS][NGP], sh_sn[ASM_WARPS][NGP];
  __shared__ double sh_X[ASM_WARPS][NEN][3];  // node coordinates, staged once per warp
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * ASM_WARPS + wib;
  if (w >= ne) return;
  const int e = elist[w];
  int node = 0;
  if (lane < NEN) {
    node = enodes[(size_t)e * NEN + lane];
#pragma unroll
    for (int c = 0; c < 3; ++c) sh_X[wib][lane][c] = xyz[(size_t)node * 3 + c];
  }
  __syncwarp();
  if (lane < NGP) {
    double N[NEN], dB[NEN][3], s;
    const bool ok = gp_geometry<CODE>(lane, sh_X[wib], 3, N, dB, s);
    double sn = 0.0;
#pragma unroll
    for (int p = 0; p < NEN; ++p) sn += N[p];
    sh_s[wib][lane] = ok ? s : 0.0;
    sh_sn[wib][lane] = sn;
#pragma unroll
    for (int p = 0; p < NEN; ++p) {
      sh_N[wib][lane][p] = N[p];
#pragma unroll
      for (int i = 0; i < 3; ++i) sh_dB[wib][lane][p][i] = dB[p][i];
    }
  }
  __syncwarp();
  const int *sl = slots + (size_t)e * ND * ND;
  for (int idx = lane; idx < ND * ND; idx += 32) {
    const int ra = idx / ND, cb = idx % ND;
    const int p = ra / 3, i = ra % 3, q = cb / 3, j = cb % 3;
    double K = 0.0;
#pragma unroll
    for (int t = 0; t < NGP; ++t) {
      const double *a = sh_dB[wib][t][p], *b = sh_dB[wib][t][q];
      double v = c12 * a[i] * b[j] + c44 * a[j] * b[i];
      if (i == j) v += c44 * (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]);
      K += sh_s[wib][t] * v;
    }
    const int slot = sl[idx];
    if (slot >= 0) values[slot] += K;
  }
  int node_of[NEN];
#pragma unroll
  for (int p = 0; p < NEN; ++p) node_of[p] = __shfl_sync(0xffffffffu, node, p);
  if (lane < ND) {
    const int p = lane / 3, i = lane % 3;
    const double bfi = i == 0 ? bf0 : (i == 1 ? bf1 : bf2);
    double F = 0.0;
#pragma unroll
    for (int t = 0; t < NGP; ++t) F += sh_s[wib][t] * ((bfi * sh_sn[wib][t]) * sh_N[wib][t][p]);
    const int r = perm[node_of[p]];
    if (r >= 0) rhs[3 * r + i] += F;
  }
}

// element -> CRS positions: slots[e][a][b] = position of (row(a), col(b)) in Cols,
// found by binary search in the row (rows are sorted, CRS_SortMatrix)
__global__ void k_slot_map(int nelem, int nen, int dofs, const int *__restrict__ enodes,
                           const int *__restrict__ perm, const int *__restrict__ rows,
                           const int *__restrict__ cols, int *__restrict__ slots, int *err) {
  const int nd = nen * dofs;
  const long long total = (long long)nelem * nd;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t / nd), a = (int)(t % nd);
    const int pn = perm[enodes[(size_t)e * nen + a / dofs]];
    int *out = slots + ((size_t)e * nd + a) * nd;
    if (pn < 0) {
      for (int b = 0; b < nd; ++b) out[b] = -1;
      continue;
    }
    const int row = pn * dofs + a % dofs;
    const int beg = rows[row], end = rows[row + 1];
    for (int b = 0; b < nd; ++b) {
      const int qn = perm[enodes[(size_t)e * nen + b / dofs]];
      int pos = -1;
      if (qn >= 0) {
        const int col = qn * dofs + b % dofs;
        int lo = beg, hi = end - 1;
        while (lo <= hi) {
          const int mid = (lo + hi) >> 1;
          const int c = cols[mid];
          if (c == col) {
            pos = mid;
            break;
          }
          if (c < col)
            lo = mid + 1;
          else
            hi = mid - 1;
        }
        if (pos < 0) atomicExch(err, 1);
      }
      out[b] = pos;
    }
  }
}

__global__ void k_fill_zero(double *p, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

// DefaultDirichletBCs (DefUtils.src:3530-4031) on the whole matrix in one pass:
// scale without rhs normalisation, constrained rows -> zero row, unit diagonal,
// b = val/D (SolverUtils.src:2465-2473), or symmetric elimination (CRS_SetSymmDirichlet,
// CRSMatrix.src:674-740), then back-scaling.  One thread per row keeps the reference's
// per-row order of right-hand-side updates.
__global__ void k_dirichlet(int n, const int *__restrict__ rows, const int *__restrict__ cols,
                            const int *__restrict__ diag, double *__restrict__ values, double *__restrict__ rhs,
                            const double *__restrict__ D, const unsigned char *__restrict__ cflag,
                            const double *__restrict__ cval, int symmetric) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double di = D[i];
    double bi = rhs[i] * di;
    if (cflag[i]) {
      for (int k = rows[i]; k < rows[i + 1]; ++k) values[k] = 0.0;
      values[diag[i]] = 1.0 / (di * di);
      bi = cval[i] / di;
    } else {
      for (int k = rows[i]; k < rows[i + 1]; ++k) {
        const int c = cols[k];
        const double dd = di * D[c];
        double v = values[k] * dd;
        if (symmetric && cflag[c]) {
          bi = bi - v * (cval[c] / D[c]);
          v = 0.0;
        }
        values[k] = v / dd;
      }
    }
    rhs[i] = bi / di * 1.0;
  }
}

// ScaleLinearSystem diagonal (SolverUtils.src:6500-6562) of the assembled matrix
__global__ void k_dirichlet_scale_diag(int n, const int *__restrict__ rows, const int *__restrict__ diag,
                                       const double *__restrict__ vals, double *__restrict__ D) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int j = diag[i];
    double d = j >= 0 ? vals[j] : 0.0;
    if (fabs(d) <= EGPU_TINY_DP) {
      double s = 0.0;
      for (int k = rows[i]; k < rows[i + 1]; ++k) s += fabs(vals[k]);
      d = s;
    }
    D[i] = fabs(d) > EGPU_TINY_DP ? 1.0 / sqrt(fabs(d)) : 1.0;
  }
}

__global__ void k_scatter_con(int ncon, const int *__restrict__ con_rows, const double *__restrict__ con_vals,
                              unsigned char *cflag, double *cval, int n, int *err) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncon; t += gridDim.x * blockDim.x) {
    const int r = con_rows[t] - 1;
    if (r < 0 || r >= n) {
      atomicExch(err, 1);
      continue;
    }
    cflag[r] = 1;
    cval[r] = con_vals ? con_vals[t] : 0.0;
  }
}

}  // namespace egpu

using namespace egpu;

static int grid_of(egpu_ctx *ctx, long long work, int block = 256) {
  long long g = (work + block - 1) / block;
  return (int)std::max(1LL, std::min(g, (long long)ctx->num_sms * 16));
}

extern "C" int egpu_assembly_bind(egpu_mat *A, int nnodes, const double *xyz, int cdim, int nelem, int code,
                                  const int *elem_nodes, const int *perm, int dofs) {
  if (!A || nnodes <= 0 || nelem <= 0 || !xyz || !elem_nodes || !perm) return EGPU_ERR_ARG;
  if (code != 808 && code != 504 && code != 303) return EGPU_ERR_ARG;
  if (dofs != 1 && !(dofs == 3 && code != 303)) return EGPU_ERR_ARG;
  if (cdim != 2 && cdim != 3) return EGPU_ERR_ARG;
  egpu_ctx *ctx = A->ctx;
  cudaSetDevice(ctx->device);
  const int nen = code % 100;
  AssemblyData &S = A->asmb;
  S.nnodes = nnodes;
  S.nelem = nelem;
  S.nen = nen;
  S.code = code;
  S.dofs = dofs;
  S.cdim = cdim;
  std::vector<int> en0((size_t)nelem * nen), p0(nnodes);
  for (size_t k = 0; k < en0.size(); ++k) {
    if (elem_nodes[k] < 1 || elem_nodes[k] > nnodes) return EGPU_ERR_ARG;
    en0[k] = elem_nodes[k] - 1;
  }
  for (int i = 0; i < nnodes; ++i) {
    p0[i] = perm[i] - 1;
    if (p0[i] >= 0 && (long long)(p0[i] + 1) * dofs > A->n) return EGPU_ERR_ARG;
  }
  std::vector<int> color_of;
  const int ncol = egpu_color_elements(nnodes, nelem, nen, elem_nodes, color_of);
  S.color_ptr.assign(ncol + 1, 0);
  for (int e = 0; e < nelem; ++e) S.color_ptr[color_of[e] + 1]++;
  for (int c = 0; c < ncol; ++c) S.color_ptr[c + 1] += S.color_ptr[c];
  std::vector<int> grouped(nelem), fill(S.color_ptr.begin(), S.color_ptr.end() - 1);
  for (int e = 0; e < nelem; ++e) grouped[fill[color_of[e]]++] = e;
  const int nd = nen * dofs;
  EGPU_CUDA_TRY(ctx, S.xyz.alloc((size_t)nnodes * 3));
  EGPU_CUDA_TRY(ctx, S.elem_nodes.alloc(en0.size()));
  EGPU_CUDA_TRY(ctx, S.perm.alloc(nnodes));
  EGPU_CUDA_TRY(ctx, S.color_elems.alloc(nelem));
  EGPU_CUDA_TRY(ctx, S.slots.alloc((size_t)nelem * nd * nd));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(S.xyz.p, xyz, (size_t)nnodes * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(S.elem_nodes.p, en0.data(), en0.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(S.perm.p, p0.data(), nnodes * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(S.color_elems.p, grouped.data(), nelem * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  int *err = (int *)(ctx->sync.p + 1);
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
  k_slot_map<<<grid_of(ctx, (long long)nelem * nd), 256, 0, ctx->stream>>>(nelem, nen, dofs, S.elem_nodes.p, S.perm.p,
                                                                          A->rows.p, A->cols.p, S.slots.p, err);
  ctx->launches++;
  int herr = 0;
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr) {
    egpu_set_error(ctx, "mesh and CRS pattern disagree: an element coupling has no matrix entry");
    return EGPU_ERR_ARG;
  }
  S.bound = true;
  return EGPU_OK;
}

extern "C" int egpu_assemble_poisson(egpu_mat *A, const double *elem_k, const double *nodal_k, const double *load) {
  if (!A || !A->asmb.bound || A->asmb.dofs != 1) return EGPU_ERR_STATE;
  egpu_ctx *ctx = A->ctx;
  cudaSetDevice(ctx->device);
  AssemblyData &S = A->asmb;
  DevBuf<double> dk, dn, dl;
  if (elem_k) {
    EGPU_CUDA_TRY(ctx, dk.alloc(S.nelem));
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(dk.p, elem_k, S.nelem * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  if (nodal_k) {
    EGPU_CUDA_TRY(ctx, dn.alloc(S.nnodes));
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(dn.p, nodal_k, S.nnodes * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  if (load) {
    EGPU_CUDA_TRY(ctx, dl.alloc(S.nnodes));
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(dl.p, load, S.nnodes * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  k_fill_zero<<<grid_of(ctx, A->nnz), 256, 0, ctx->stream>>>(A->values.p, A->nnz);
  k_fill_zero<<<grid_of(ctx, A->n), 256, 0, ctx->stream>>>(A->rhs.p, A->n);
  ctx->launches += 2;
  const int ncol = (int)S.color_ptr.size() - 1;
  for (int c = 0; c < ncol; ++c) {
    const int ne = S.color_ptr[c + 1] - S.color_ptr[c];
    if (!ne) continue;
    const int *el = S.color_elems.p + S.color_ptr[c];
    const int grid = (ne + ASM_WARPS - 1) / ASM_WARPS;
#define EGPU_ASM(CODE)                                                                                       \
  k_assemble_poisson<CODE><<<grid, ASM_WARPS * 32, 0, ctx->stream>>>(ne, el, S.elem_nodes.p, S.xyz.p, S.cdim, \
                                                                     dk.p, dn.p, dl.p, S.perm.p, S.slots.p,    \
                                                                     A->values.p, A->rhs.p)
    if (S.code == 808)
      EGPU_ASM(808);
    else if (S.code == 504)
      EGPU_ASM(504);
    else
      EGPU_ASM(303);
#undef EGPU_ASM
    ctx->launches++;
  }
  EGPU_CUDA_TRY(ctx, cudaGetLastError());
  EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  A->has_values = true;
  A->has_rhs = true;
  A->ilu_valid = false;
  return EGPU_OK;
}

extern "C" int egpu_assemble_elastic(egpu_mat *A, double young, double poisson, const double *bf) {
  if (!A || !A->asmb.bound || A->asmb.dofs != 3 || !bf) return EGPU_ERR_STATE;
  egpu_ctx *ctx = A->ctx;
  cudaSetDevice(ctx->device);
  AssemblyData &S = A->asmb;
  const double cs = young / ((1 + poisson) * (1 - 2 * poisson));
  const double c12 = poisson * cs, c44 = (0.5 - poisson) * cs;
  k_fill_zero<<<grid_of(ctx, A->nnz), 256, 0, ctx->stream>>>(A->values.p, A->nnz);
  k_fill_zero<<<grid_of(ctx, A->n), 256, 0, ctx->stream>>>(A->rhs.p, A->n);
  ctx->launches += 2;
  const int ncol = (int)S.color_ptr.size() - 1;
  for (int c = 0; c < ncol; ++c) {
    const int ne = S.color_ptr[c + 1] - S.color_ptr[c];
    if (!ne) continue;
    const int *el = S.color_elems.p + S.color_ptr[c];
    const int grid = (ne + ASM_WARPS - 1) / ASM_WARPS;
    if (S.code == 808)
      k_assemble_elastic<808><<<grid, ASM_WARPS * 32, 0, ctx->stream>>>(ne, el, S.elem_nodes.p, S.xyz.p, c12, c44, bf[0],
                                                                        bf[1], bf[2], S.perm.p, S.slots.p, A->values.p,
                                                                        A->rhs.p);
    else
      k_assemble_elastic<504><<<grid, ASM_WARPS * 32, 0, ctx->stream>>>(ne, el, S.elem_nodes.p, S.xyz.p, c12, c44, bf[0],
                                                                        bf[1], bf[2], S.perm.p, S.slots.p, A->values.p,
                                                                        A->rhs.p);
    ctx->launches++;
  }
  EGPU_CUDA_TRY(ctx, cudaGetLastError());
  EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  A->has_values = true;
  A->has_rhs = true;
  A->ilu_valid = false;
  return EGPU_OK;
}

extern "C" int egpu_dirichlet(egpu_mat *A, int ncon, const int *con_rows, const double *con_vals, int symmetric) {
  if (!A || ncon < 0 || (ncon > 0 && !con_rows)) return EGPU_ERR_ARG;
  egpu_ctx *ctx = A->ctx;
  cudaSetDevice(ctx->device);
  const int n = A->n;
  DevBuf<int> dr;
  DevBuf<double> dv, D, cval;
  DevBuf<unsigned char> cflag;
  EGPU_CUDA_TRY(ctx, cflag.alloc(n));
  EGPU_CUDA_TRY(ctx, cval.alloc(n));
  EGPU_CUDA_TRY(ctx, D.alloc(n));
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(cflag.p, 0, n, ctx->stream));
  int *err = (int *)(ctx->sync.p + 1);
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
  if (ncon > 0) {
    EGPU_CUDA_TRY(ctx, dr.alloc(ncon));
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(dr.p, con_rows, ncon * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    if (con_vals) {
      EGPU_CUDA_TRY(ctx, dv.alloc(ncon));
      EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(dv.p, con_vals, ncon * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    k_scatter_con<<<grid_of(ctx, ncon), 256, 0, ctx->stream>>>(ncon, dr.p, dv.p, cflag.p, cval.p, n, err);
    ctx->launches++;
  }
  // Linear System Dirichlet Scaling defaults to Linear System Scaling = True
  k_dirichlet_scale_diag<<<grid_of(ctx, n), 256, 0, ctx->stream>>>(n, A->rows.p, A->diag.p, A->values.p, D.p);
  k_dirichlet<<<grid_of(ctx, n), 256, 0, ctx->stream>>>(n, A->rows.p, A->cols.p, A->diag.p, A->values.p, A->rhs.p, D.p,
                                                        cflag.p, cval.p, symmetric);
  ctx->launches += 2;
  int herr = 0;
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr) {
    egpu_set_error(ctx, "Dirichlet row index out of range");
    return EGPU_ERR_ARG;
  }
  A->ilu_valid = false;
  return EGPU_OK;
}
