// egpu_tri_cta.cu -- host side of the level-synchronous single-block ILU0 solves.
//
// The sync-free solves (egpu_krylov.cuh) spread a level over the whole GPU and pay a
// cross-SM publish/observe round trip per dependency level.  On meshes whose levels are
// narrow (a few hundred rows) and whose dependencies reach only a few levels back, one
// block running the levels in order out of shared memory is faster: its per-level cost is
// a __syncthreads, and the factor entries stream in through cp.async ahead of use.  This
// file builds that schedule (ELL blocks per level, ring-buffer slots, staging windows),
// fills it with the factor values after every factorisation, and decides per solve which
// of the two solves to run.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "egpu_solve.h"
#include "egpu_tri_plan.h"

namespace egpu {

namespace {

// dynamic shared memory of the single block (227 KB per block on sm_100, less the
// kernels' static shared memory and a margin)
constexpr size_t CTA_SMEM_MAX = 200 * 1024;

int tri_mode_env() {
  // EGPU_TRI_MODE: "syncfree" never uses the single-block solve, "block" uses it whenever
  // the schedule fits, anything else chooses by the cost estimate
  const char *m = std::getenv("EGPU_TRI_MODE");
  if (!m) return 0;
  if (!std::strcmp(m, "syncfree")) return 1;
  if (!std::strcmp(m, "block")) return 2;
  return 0;
}

// Estimated seconds of one M^-1 application, from B200 measurements of the solves on hex
// meshes (Poisson and 3-DOF elasticity): sync-free, about 0.9 us per dependency level (a
// cross-SM publish/observe round trip) plus 0.8 ns per row; node-block sync-free, about
// 1.7 us per block level plus 0.65 ns per row; single block, about 0.6 us per level plus
// 4 ns per row (its entries streamed and summed by one SM), plus the extra grid barrier.
double est_syncfree(int nlev_lo, int nlev_up, int n) { return 0.9e-6 * (nlev_lo + nlev_up) + 0.8e-9 * 2.0 * n; }
double est_nodeblock(int nlev_lo, int nlev_up, int n) { return 1.7e-6 * (nlev_lo + nlev_up) + 0.65e-9 * 2.0 * n; }
double est_block(int nlev_lo, int nlev_up, int n) { return 0.6e-6 * (nlev_lo + nlev_up) + 4e-9 * 2.0 * n + 3e-6; }

}  // namespace

// node-block sync-free solve (bl / bu block levels) instead of the row schedule (nlo / nup
// row levels, sync-free or single block)?  EGPU_TRI_NODE_BLOCKS=0 never, =1 always.
bool tri_prefer_node_blocks(int nlo, int nup, int bl, int bu, int n) {
  if (const char *e = std::getenv("EGPU_TRI_NODE_BLOCKS")) {
    if (!std::strcmp(e, "0")) return false;
    if (!std::strcmp(e, "1")) return true;
  }
  const int mode = tri_mode_env();
  if (mode == 2) return false;
  const double blk = est_nodeblock(bl, bu, n);
  if (blk >= est_syncfree(nlo, nup, n)) return false;
  return mode == 1 || blk < est_block(nlo, nup, n);
}

__global__ void k_cta_fill(long long nl, long long nu, const int *__restrict__ lsrc, const int *__restrict__ usrc,
                           const double *__restrict__ lo, const double *__restrict__ up,
                           const float *__restrict__ lo32, const float *__restrict__ up32, double *clo, double *cup,
                           float *clo32, float *cup32) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nl + nu;
       t += (long long)gridDim.x * blockDim.x) {
    if (t < nl) {
      const int s = lsrc[t];
      clo[t] = s >= 0 ? lo[s] : 0.0;
      clo32[t] = s >= 0 ? lo32[s] : 0.0f;
    } else {
      const long long k = t - nl;
      const int s = usrc[k];
      cup[k] = s >= 0 ? up[s] : 0.0;
      cup32[k] = s >= 0 ? up32[s] : 0.0f;
    }
  }
}

// Build the single-block schedule next to the sync-free one.  lo / up: slot orders;
// lp, lc / upp, uc: packed strictly-lower / strictly-upper entries per slot.
int build_cta_schedule(egpu_mat *A, const std::vector<int> &rows, const std::vector<int> &cols,
                       const std::vector<int> &diag, const std::vector<int> &lo, const std::vector<int> &up,
                       const std::vector<int> &lp, const std::vector<int> &lc, const std::vector<int> &upp,
                       const std::vector<int> &uc) {
  egpu_ctx *ctx = A->ctx;
  TriSchedule &S = A->tri;
  const int n = A->n;
  S.cta_ok[0] = S.cta_ok[1] = false;
  const int mode = tri_mode_env();
  if (mode == 1 || n == 0) return EGPU_OK;
  plan::Plan P;
  plan::make_plan(n, rows, cols, diag, lo, up, lp, lc, upp, uc, CTA_SMEM_MAX, P);
  if (!P.ok) return EGPU_OK;
  bool any = false;
  for (int v = 0; v < 2; ++v)
    if (P.fits[v] && (mode == 2 || est_block(P.lo.nlev, P.up.nlev, n) < est_syncfree(P.lo.nlev, P.up.nlev, n)))
      any = true;
  if (!any) return EGPU_OK;
  if (!plan::plan_arrays(P, n, lo, up, lp, lc, upp, uc)) {
    egpu_set_error(ctx, "internal: level-synchronous schedule dependency out of range");
    return EGPU_ERR_ARG;
  }
  auto upload = [&](const plan::TriPlan &T, CtaTriHost &H) -> int {
    std::vector<int4> lev(std::max<size_t>(1, T.lev.size()), make_int4(0, 0, 0, 0));
    for (size_t L = 0; L < T.lev.size(); ++L) lev[L] = make_int4(T.lev[L].x, T.lev[L].y, T.lev[L].z, T.lev[L].w);
    EGPU_CUDA_TRY(ctx, H.lev.alloc(lev.size()));
    EGPU_CUDA_TRY(ctx, H.ridx.alloc(T.nent));
    EGPU_CUDA_TRY(ctx, H.src.alloc(T.nent));
    EGPU_CUDA_TRY(ctx, H.map.alloc(T.map.size()));
    EGPU_CUDA_TRY(ctx, cudaMemcpy(H.lev.p, lev.data(), lev.size() * sizeof(int4), cudaMemcpyHostToDevice));
    EGPU_CUDA_TRY(ctx, cudaMemcpy(H.ridx.p, T.ridx.data(), T.nent * sizeof(uint16_t), cudaMemcpyHostToDevice));
    EGPU_CUDA_TRY(ctx, cudaMemcpy(H.src.p, T.src.data(), T.nent * sizeof(int), cudaMemcpyHostToDevice));
    EGPU_CUDA_TRY(ctx, cudaMemcpy(H.map.p, T.map.data(), T.map.size() * sizeof(int), cudaMemcpyHostToDevice));
    H.nlev = T.nlev;
    H.nent = T.nent;
    return EGPU_OK;
  };
  int rc = upload(P.lo, S.cta_lo);
  if (!rc) rc = upload(P.up, S.cta_up);
  if (rc) return rc;
  EGPU_CUDA_TRY(ctx, S.pos_lo.alloc(P.pos_lo.size()));
  EGPU_CUDA_TRY(ctx, S.pos_up.alloc(P.pos_up.size()));
  EGPU_CUDA_TRY(ctx, cudaMemcpy(S.pos_lo.p, P.pos_lo.data(), P.pos_lo.size() * sizeof(int), cudaMemcpyHostToDevice));
  EGPU_CUDA_TRY(ctx, cudaMemcpy(S.pos_up.p, P.pos_up.data(), P.pos_up.size() * sizeof(int), cudaMemcpyHostToDevice));
  S.cta_rs = P.rs;
  for (int v = 0; v < 2; ++v) {
    S.cta_ok[v] = P.fits[v];
    S.cta_pd[v] = P.pd[v];
    S.cta_sb[v] = P.sb[v];
    S.cta_sr[v] = P.sr[v];
    S.cta_smem[v] = P.smem[v];
  }
  return EGPU_OK;
}

// the factors in the ELL layout, after every factorisation
int cta_fill_values(egpu_mat *A) {
  const TriSchedule &S = A->tri;
  if (!S.cta_ok[0] && !S.cta_ok[1]) return EGPU_OK;
  egpu_ctx *ctx = A->ctx;
  const long long nl = S.cta_lo.nent, nu = S.cta_up.nent;
  EGPU_CUDA_TRY(ctx, A->cta_lo_vals.alloc(nl));
  EGPU_CUDA_TRY(ctx, A->cta_up_vals.alloc(nu));
  EGPU_CUDA_TRY(ctx, A->cta_lo_vals32.alloc(nl));
  EGPU_CUDA_TRY(ctx, A->cta_up_vals32.alloc(nu));
  const long long tot = nl + nu;
  const int grid = (int)std::max(1LL, std::min((tot + 255) / 256, (long long)ctx->num_sms * 8));
  k_cta_fill<<<grid, 256, 0, ctx->stream>>>(nl, nu, S.cta_lo.src.p, S.cta_up.src.p, A->lo_vals.p, A->up_vals.p,
                                             A->lo_vals32.p, A->up_vals32.p, A->cta_lo_vals.p, A->cta_up_vals.p,
                                             A->cta_lo_vals32.p, A->cta_up_vals32.p);
  ctx->launches++;
  EGPU_CUDA_TRY(ctx, cudaGetLastError());
  return EGPU_OK;
}

// threads of the block taking part in the level-synchronous solve: enough for the widest
// level, a multiple of 32, at most the block (EGPU_TRI_THREADS overrides)
int cta_threads(const egpu_mat *A) {
  int nt = 512;
  if (const char *e = std::getenv("EGPU_TRI_THREADS")) nt = std::atoi(e);
  nt = std::max(32, std::min(EGPU_KBLOCK, nt));
  return nt / 32 * 32;
}

// single-block solve for this precision (v = 0 FP64, 1 FP32)?
bool cta_use(const egpu_mat *A, int v) {
  const TriSchedule &S = A->tri;
  if (!S.cta_ok[v] || !A->cta_lo_vals.p) return false;
  const int mode = tri_mode_env();
  if (mode == 1) return false;
  if (mode == 2) return true;
  return est_block(S.cta_lo.nlev, S.cta_up.nlev, A->n) < est_syncfree(S.cta_lo.nlev, S.cta_up.nlev, A->n);
}

}  // namespace egpu
