// egpu_noalloc.cu -- CG + Diagonal solve that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: code that must not trigger the
// implicit device-wide synchronisation of an allocation inside a time-critical loop, and
// hosts whose device memory is owned by another runtime (a CUDA Fortran or OpenACC data
// region around Elmer's arrays) that forbids hidden allocations.  For them this file
// provides one entry point whose scratch lives in a fixed, file-scope device array.
//
// Limits and sharing rules:
//   * systems of at most EGPU_NOALLOC_MAX_ROWS rows (larger n is rejected with EGPU_ERR_ARG);
//   * the array (about 2.4 MB) is held by every GPU that loads this library until the
//     process exits;
//   * every call on a device uses the same array: calls that overlap on the GPU race and
//     must be serialised by the caller; the counters that must start at zero are cleared
//     by each call, everything else is overwritten before it is read.
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress
//     with that device current) and caches it; make that first call before any stream
//     capture.  The cached address is not looked up again, so after cudaDeviceReset on
//     that device (which unloads the module and may place the array elsewhere) this entry
//     point must not be called;
//   * the caller's arrays are used in place and are checked on the device before any gather
//     goes through them; the caller's current device is restored on return.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <mutex>

#include "egpu_internal.cuh"

namespace {

constexpr int NA_MAXN = EGPU_NOALLOC_MAX_ROWS;
constexpr int NA_NVEC = 9;          // D0 D dv bs xs R Z P Q
constexpr int NA_PARTIALS = 8 * 1024;
// as unsigned ints at the tail, laid out as a context's control block (egpu_internal.cuh):
// barrier counter, error word, then from EGPU_CTL_WORD the wait bound and abort address,
// both kept at zero here (the default bound, no abort word)
constexpr int NA_COUNTERS = EGPU_SYNC_WORDS;

}  // namespace

// The scratch: NA_NVEC vectors of NA_MAXN doubles, partial sums, then counters.
static __device__ __align__(256) double g_noalloc_scratch[NA_NVEC * NA_MAXN + NA_PARTIALS + NA_COUNTERS / 2];

namespace {

enum { NS_BB = 0, NS_BD, NS_RHO, NS_PQ, NS_RR, NS_NSLOT };

struct NaArgs {
  int n;
  const int *rows, *cols, *diag;  // 1-based (Matrix_t), device memory
  const double *vals, *b;
  double *x;
  int precond, maxit;
  double tol;
  double *scratch;                // device address of g_noalloc_scratch
};

// v = (D A D) u for row i in the reference's row order (as the SELL path: a_ij*(D_i*D_j), then
// s = s + v*u with two roundings)
__device__ __forceinline__ double scaled_row(const NaArgs &a, const double *D0, int i, const double *u) {
  const double di = D0[i];
  double s = 0.0;
  for (int k = a.rows[i] - 1; k < a.rows[i + 1] - 1; ++k) {
    const int c = a.cols[k] - 1;
    const double v = a.vals[k] * (di * D0[c]);
    s = __dadd_rn(s, __dmul_rn(v, __ldcg(u + c)));
  }
  return s;
}

__device__ __forceinline__ double na_prec(double r, double d, int precond) {
  return (precond == EGPU_PREC_DIAGONAL && fabs(d) > EGPU_AEPS) ? r / d : r;
}

__global__ void __launch_bounds__(256) k_cg_noalloc(NaArgs a) {
  __shared__ double sm[32 * 4];
  const int n = a.n;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const int nb = gridDim.x;
  double *D0 = a.scratch, *D = D0 + NA_MAXN, *dv = D + NA_MAXN, *bs = dv + NA_MAXN, *X = bs + NA_MAXN,
         *R = X + NA_MAXN, *Z = R + NA_MAXN, *P = Z + NA_MAXN, *Q = P + NA_MAXN;
  double *partials = a.scratch + NA_NVEC * NA_MAXN;
  unsigned int *cnt = reinterpret_cast<unsigned int *>(partials + NA_PARTIALS);
  unsigned int *bar = cnt;
  int *err = reinterpret_cast<int *>(cnt + 1);
  unsigned int *xnz = cnt + 2;
  int *out_i = reinterpret_cast<int *>(cnt + 8);
  double *out_d = reinterpret_cast<double *>(cnt + 16);
  unsigned int epoch = 0;

  // The caller's Matrix_t arrays are used in place, so they are checked here before any
  // gather goes through them (egpu_matrix_bind checks the same on the host): Rows(1) = 1 and
  // non-decreasing, every Cols entry in 1..n, Diag either 0 (no stored diagonal) or inside its
  // row at the column of the row itself.  A violation sets EGPU_ERR_ARG and every block leaves
  // at the first grid barrier.  Only Rows(i), Rows(i+1) and entries they bound are read, and
  // an entry is read only after its row's bounds passed.
  for (int i = tid; i < n; i += nth) {
    const int r0 = a.rows[i], r1 = a.rows[i + 1];
    bool ok = r0 <= r1 && (i != 0 || r0 == 1) && r0 >= 1;
    for (int k = r0 - 1; ok && k < r1 - 1; ++k) {
      const int c = a.cols[k];
      ok = c >= 1 && c <= n;
    }
    const int d = a.diag[i];
    if (ok && d != 0) ok = d >= r0 && d < r1 && a.cols[d - 1] == i + 1;
    if (!ok) atomicExch(err, (int)EGPU_ERR_ARG);
  }
  if (!grid_barrier(bar, err, epoch)) return;

  // ScaleLinearSystem (SolverUtils.src:6500-6636): D0 = 1/sqrt|a_ii|, ||b||, ||D0 b||, x != 0
  {
    double acc[2] = {0.0, 0.0};
    bool nz = false;
    for (int i = tid; i < n; i += nth) {
      const int j = a.diag[i] - 1;
      double d = j >= 0 ? a.vals[j] : 0.0;
      if (fabs(d) <= EGPU_TINY_DP) {
        double s = 0.0;
        for (int k = a.rows[i] - 1; k < a.rows[i + 1] - 1; ++k) s += fabs(a.vals[k]);
        d = s;
      }
      const double di = fabs(d) > EGPU_TINY_DP ? 1.0 / sqrt(fabs(d)) : 1.0;
      D0[i] = di;
      dv[i] = j >= 0 ? a.vals[j] * (di * di) : 0.0;
      const double bi = a.b[i];
      acc[0] += bi * bi;
      const double s = bi * di;
      bs[i] = s;
      acc[1] += s * s;
      nz |= a.x[i] != 0.0;
    }
    if (__syncthreads_or(nz) && threadIdx.x == 0) atomicOr(xnz, 1u);
    block_sum<2>(acc, sm);
    if (threadIdx.x == 0) {
      partials[NS_BB * nb + blockIdx.x] = acc[0];
      partials[NS_BD * nb + blockIdx.x] = acc[1];
    }
  }
  if (!grid_barrier(bar, err, epoch)) return;
  const double borig = sqrt(reduce_partials(partials + NS_BB * nb, nb, sm));
  if (borig <= EGPU_TINY_DP) {  // solution trivially zero (SolverUtils.src:7309-7320)
    for (int i = tid; i < n; i += nth) a.x[i] = 0.0;
    if (tid == 0) {
      out_i[0] = EGPU_HUTI_CONVERGENCE;
      out_i[1] = 0;
      out_d[0] = 0.0;
    }
    return;
  }
  const double bnorm = sqrt(reduce_partials(partials + NS_BD * nb, nb, sm));
  const bool x_nonzero = (*(volatile unsigned int *)xnz & 1u) != 0;
  for (int i = tid; i < n; i += nth) {
    const double d = D0[i] * bnorm;
    D[i] = d;
    bs[i] = bs[i] / bnorm;
    X[i] = x_nonzero ? a.x[i] / d : 1.0e-8;  // IterSolve.src:358-359
  }
  if (!grid_barrier(bar, err, epoch)) return;

  // huti_dcgsolv (hutiter/src/huti_cg_D.F90:158-240), true-residual stopping test; the
  // residual of x_{k-1} is formed in the pass that computes A p_k
  {
    double acc[1] = {0.0};
    for (int i = tid; i < n; i += nth) {
      const double r = bs[i] - scaled_row(a, D0, i, X);
      R[i] = r;
      acc[0] += bs[i] * bs[i];
    }
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) partials[NS_BB * nb + blockIdx.x] = acc[0];
  }
  if (!grid_barrier(bar, err, epoch)) return;
  const double rhsnorm = sqrt(reduce_partials(partials + NS_BB * nb, nb, sm));
  {
    double acc[1] = {0.0};
    for (int i = tid; i < n; i += nth) {
      const double z = na_prec(R[i], dv[i], a.precond);
      Z[i] = z;
      acc[0] += R[i] * z;
    }
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) partials[NS_RHO * nb + blockIdx.x] = acc[0];
  }
  if (!grid_barrier(bar, err, epoch)) return;
  int k = 1, info = 0, iters = 0;
  double rho, oldrho = 1.0, residual = 0.0;
  while (true) {
    rho = reduce_partials(partials + NS_RHO * nb, nb, sm);
    const double beta = rho / oldrho;
    for (int i = tid; i < n; i += nth) P[i] = (k == 1) ? Z[i] : Z[i] + beta * P[i];
    if (!grid_barrier(bar, err, epoch)) return;
    {
      double acc[2] = {0.0, 0.0};
      for (int i = tid; i < n; i += nth) {
        const double q = scaled_row(a, D0, i, P);
        Q[i] = q;
        acc[0] += P[i] * q;
        if (k > 1) {
          const double r = scaled_row(a, D0, i, X) - bs[i];
          acc[1] += r * r;
        }
      }
      block_sum<2>(acc, sm);
      if (threadIdx.x == 0) {
        partials[NS_PQ * nb + blockIdx.x] = acc[0];
        partials[NS_RR * nb + blockIdx.x] = acc[1];
      }
    }
    if (!grid_barrier(bar, err, epoch)) return;
    const double pq = reduce_partials(partials + NS_PQ * nb, nb, sm);
    if (k > 1) {
      residual = sqrt(reduce_partials(partials + NS_RR * nb, nb, sm)) / rhsnorm;
      if (residual < a.tol) { info = EGPU_HUTI_CONVERGENCE; iters = k - 1; break; }
      if (k > a.maxit) { info = EGPU_HUTI_MAXITER; iters = k; break; }
    }
    if (rho == 0.0) { info = EGPU_HUTI_CG_RHO; iters = k; break; }
    const double alpha = rho / pq;
    {
      double acc[1] = {0.0};
      for (int i = tid; i < n; i += nth) {
        X[i] = X[i] + alpha * P[i];
        const double r = R[i] - alpha * Q[i];
        R[i] = r;
        const double z = na_prec(r, dv[i], a.precond);
        Z[i] = z;
        acc[0] += r * z;
      }
      block_sum<1>(acc, sm);
      if (threadIdx.x == 0) partials[NS_RHO * nb + blockIdx.x] = acc[0];
    }
    if (!grid_barrier(bar, err, epoch)) return;
    oldrho = rho;
    ++k;
  }
  // BackScaleLinearSystem x part (SolverUtils.src:6794-6796)
  for (int i = tid; i < n; i += nth) a.x[i] = X[i] * D[i];
  if (tid == 0) {
    out_i[0] = info;
    out_i[1] = iters;
    out_d[0] = residual;
  }
}

std::mutex g_mu;
double *g_addr[64] = {nullptr};

int noalloc_solve(int device, int n, const int *rows_dev, const int *cols_dev, const int *diag_dev,
                  const double *values_dev, const double *b_dev, double *x_dev, const egpu_params *prm,
                  egpu_result *res);

}  // namespace

extern "C" int egpu_cg_noalloc(int device, int n, const int *rows_dev, const int *cols_dev, const int *diag_dev,
                               const double *values_dev, const double *b_dev, double *x_dev,
                               const egpu_params *prm, egpu_result *res) {
  if (!prm || !rows_dev || !cols_dev || !diag_dev || !values_dev || !b_dev || !x_dev) return EGPU_ERR_ARG;
  if (n < 1 || n > NA_MAXN) return EGPU_ERR_ARG;
  if (prm->method != EGPU_CG || prm->max_iter < 1 ||
      (prm->precond != EGPU_PREC_DIAGONAL && prm->precond != EGPU_PREC_NONE) || !prm->scale_system)
    return EGPU_ERR_ARG;
  if (device < 0 || device >= 64) return EGPU_ERR_ARG;
  // the caller's current device is put back on every return: hosts that manage their own
  // device (CUDA Fortran, OpenACC) keep it
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return EGPU_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return EGPU_ERR_CUDA;
  const int rc = noalloc_solve(device, n, rows_dev, cols_dev, diag_dev, values_dev, b_dev, x_dev, prm, res);
  if (prev != device) cudaSetDevice(prev);
  return rc;
}

namespace {

int noalloc_solve(int device, int n, const int *rows_dev, const int *cols_dev, const int *diag_dev,
                  const double *values_dev, const double *b_dev, double *x_dev, const egpu_params *prm,
                  egpu_result *res) {
  double *scratch = nullptr;
  {
    // set-up, once per device, with that device current: the host-side name of the array is
    // not a device address; look the address up and keep it
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return EGPU_ERR_CUDA;
      g_addr[device] = static_cast<double *>(p);
    }
    scratch = g_addr[device];
  }
  // counters that must start at zero: barrier count, error flag, x != 0 flag, and the
  // control words (default wait bound, no abort word)
  unsigned int *cnt = reinterpret_cast<unsigned int *>(scratch + NA_NVEC * NA_MAXN + NA_PARTIALS);
  if (cudaMemsetAsync(cnt, 0, (EGPU_CTL_WORD + 4) * sizeof(unsigned int), 0) != cudaSuccess) return EGPU_ERR_CUDA;
  int num_sms = 0, bps = 0;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_cg_noalloc, 256, 0) != cudaSuccess || bps < 1)
    return EGPU_ERR_CUDA;
  const int grid = std::min(num_sms * std::min(bps, 2), NA_PARTIALS / NS_NSLOT);
  NaArgs a{n, rows_dev, cols_dev, diag_dev, values_dev, b_dev, x_dev, prm->precond, prm->max_iter, prm->tol, scratch};
  void *args[] = {&a};
  const auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_cg_noalloc, dim3(grid), dim3(256), args, 0, 0);
  unsigned int h[24] = {0};
  if (e == cudaSuccess) e = cudaMemcpy(h, cnt, sizeof(h), cudaMemcpyDeviceToHost);  // waits for the kernel
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (e != cudaSuccess) return EGPU_ERR_CUDA;
  if (h[1]) return (int)h[1];
  egpu_result r{};
  r.info = reinterpret_cast<int *>(h + 8)[0];
  r.iters = reinterpret_cast<int *>(h + 8)[1];
  r.residual = reinterpret_cast<double *>(h + 16)[0];
  r.seconds = ms * 1e-3;
  r.seconds_krylov = ms * 1e-3;
  r.krylov_launches = 1;
  if (res) *res = r;
  return r.info;
}

}  // namespace
