// egpu_solve.h -- internal solve entry points shared by the translation units.
#pragma once

#include "egpu_internal.cuh"

// ILU(n) fill structure (egpu_pattern.cpp), 0-based; order 0 returns the input
void egpu_ilu_structure(int n, const std::vector<int> &rows, const std::vector<int> &cols,
                        const std::vector<int> &diag, int order, std::vector<int> &orows, std::vector<int> &ocols,
                        std::vector<int> &odiag);

// threshold ILU factors on the host (egpu_pattern.cpp), 0-based, inverted U diagonal
bool egpu_ilut_host(int n, const std::vector<int> &rows, const std::vector<int> &cols,
                    const std::vector<double> &vals, double tol, std::vector<int> &ir, std::vector<int> &ic,
                    std::vector<int> &id, std::vector<double> &iv);

namespace egpu {

// inner tolerance of one FP32 segment of the mixed-precision solve; 0 picks it by
// preconditioner.  Segments continue each other's recurrences (reliable updating), so short
// segments keep the FP64 iteration count while the FP64 true residual is refreshed often:
// tuned on B200, 1e-2 with Diagonal / none (CG 128^3: 417 FP32 iterations against 378 in
// FP64) and 3e-2 with ILU0 (BiCGStab 32^3: 19 against 19).
inline double inner_tol_of(const egpu_params *p) {
  if (p->inner_tol > 0) return p->inner_tol;
  return (p->precond == EGPU_PREC_ILU0 || p->precond == EGPU_PREC_ILUT) ? 3e-2 : 1e-2;
}

int ensure_ctx_scratch(egpu_ctx *ctx);
int reset_sync(egpu_ctx *ctx);
int scale_matrix(egpu_mat *A, bool scale_system);
int ensure_ilu_structure(egpu_mat *A, int order);
int ensure_tri_schedule(egpu_mat *A);
int ilu_factor(egpu_mat *A, int order);
// the ILU structure code of threshold ILU (A->ilu_order; ILU(n) uses 0..9)
constexpr int ILU_ORDER_T = 100;
inline bool is_ilu(int precond) { return precond == EGPU_PREC_ILU0 || precond == EGPU_PREC_ILUT; }
int ilut_factor(egpu_mat *A, double tol);
// the factor the parameters ask for: ILU(n) or ILUT
int precond_factor(egpu_mat *A, const egpu_params *p);
int solve_fp64(egpu_mat *A, const double *b_dev, double *x_dev, const egpu_params *prm,
               egpu_result *res);
int solve_mixed(egpu_mat *A, const double *b_dev, double *x_dev, const egpu_params *prm,
                egpu_result *res);
// FP64 Krylov continuation on an already scaled system (used by the mixed path's
// stagnation fallback): xs in/out, bs scaled rhs; preconditioner state must be current.
int krylov_fp64_scaled(egpu_mat *A, const double *bs, double *xs, const egpu_params *prm, int *info,
                       int *iters, double *residual);

// scale b into bs and the initial guess x into xs (ScaleLinearSystem, x = 1e-8 rule);
// *bnorm_s = ||bs||, or -1 when b is zero (solution trivially zero).  Synchronises.
int rhs_scale(egpu_mat *A, const double *b_dev, const double *x_dev, double *bs, double *xs, bool scale_system,
              double *bnorm_s);
// FP32 SELL values, diagonal and (optionally) ILU0 factors for the inner solver
int prepare_fp32_public(egpu_mat *A, bool with_ilu, bool sweeps);
int unit_diagonal_fp32(egpu_mat *A, int *unit);

// level-synchronous single-block ILU0 solves (egpu_tri_cta.cu)
int build_cta_schedule(egpu_mat *A, const std::vector<int> &rows, const std::vector<int> &cols,
                       const std::vector<int> &diag, const std::vector<int> &lo, const std::vector<int> &up,
                       const std::vector<int> &lp, const std::vector<int> &lc, const std::vector<int> &upp,
                       const std::vector<int> &uc);
int cta_fill_values(egpu_mat *A);
bool tri_prefer_node_blocks(int nlo, int nup, int bl, int bu, int n);
bool cta_use(const egpu_mat *A, int v);
int cta_threads(const egpu_mat *A);

}  // namespace egpu
