// egpu_batch.cuh -- persistent batched FP32 inner Krylov kernel over many systems.
//
// Every system keeps its own device-resident data (an egpu_mat: SELL-32 FP32 copy of the
// scaled matrix, diagonal, ILU0 factors, level orders, FP32 work vectors); the kernel
// reads them through a table of SysDesc.  A launch runs at most kmax iterations of every
// active system and returns; Krylov state and per-system scalars stay in device memory,
// so the next launch continues where this one stopped and new systems can be admitted
// between launches (continuous batching).
//
// Work assignment: at the top of every iteration every block decides, for all systems,
// the per-system scalars and state transitions (identical inputs give identical
// decisions in every block), compacts the systems that have work this iteration, and
// takes a contiguous share of their SELL slices (re-balanced each iteration, so converged
// systems free their share).  A warp handles one slice (32 rows) of one system.
// Per-system dot products: warp sum per slice -> shared-memory accumulation per system ->
// one global atomic per (block, system); read after the next grid barrier, cleared one
// phase later.  Sums are therefore reproducible to rounding, not bitwise.
//
// Inner solve of A d = r (x0 = 0) stopping on ||r_k|| <= tol ||r_0|| (recursive residual):
//   CG        huti_cg_D.F90:158-240
//   BiCGStab  huti_bicgstab_D.F90:171-267
#pragma once

#include "egpu_internal.cuh"
#include "egpu_krylov.cuh"

namespace egpu {

constexpr int BATCH_MAX_SYS = 512;

enum { ST_IDLE = 0, ST_INIT = 1, ST_RUN = 2, ST_DONE = 3 };

struct SysDesc {
  int n, nslices;
  int unit_diag;           // CG + Jacobi on a scaled diagonal that is 1.0f everywhere: Z is R
  const int *sell_ptr, *sell_w;
  const int16_t *scols16;  // col - row
  const int *scols;        // absolute column (when scols16 is null)
  const float *svals, *dvals, *ilu;
  const int *rows, *cols, *diag, *lower_order, *upper_order;
  const int *lo_ptr, *lo_cols, *up_ptr, *up_cols;   // ILU0 factors packed in solve order
  const float *lo_vals, *up_vals, *up_dinv;
  // ILU0 by Jacobi sweeps (BatchArgs::sweeps > 0): the factors in the SELL layout, the
  // inverted U diagonal in row order, per slice the k ranges of the strictly-lower ([0, x))
  // and strictly-upper ([y, w)) entries
  const float *isvals, *idinv;
  const int2 *swr;
  float *w;                // work vectors, stride ldw
  long long ldw;
  const float *b;          // inner right-hand side (r / ||r||)
  float *x;                // inner solution d
};

// per-system state, double-buffered by iteration parity: blocks read [it & 1] and the
// system's designated block writes [(it + 1) & 1]
struct SysState {
  int status, k, info, iters;
  double rho, oldrho, alpha, omega, r0norm, residual;
  // reliable updating: resume != 0 continues the previous segment's recurrences (keeps
  // P, V, RTLD, alpha, omega) with rho_{k-1} = carry_rho (already in the new residual scale)
  int resume, pad;
  double carry_rho;
  double eta;              // CG: (p, A p) of the last direction (single-reduction recurrence)
};

// accumulator slots per system.  CG sums gamma, delta, (r, r) and (z, s) into one of two
// sets by iteration parity (BA_RHO/BA_PQ/BA_RR/BA_SS or BA_CG1..+3): a set is cleared in the
// iteration after the one whose top read it, with a grid barrier between.
enum { BA_BB = 0, BA_RHO, BA_RR, BA_PQ, BA_SS, BA_TS, BA_TT, BA_CG1, BA_NSLOT = BA_CG1 + 4 };

struct BatchArgs {
  int nsys;
  const SysDesc *sys;
  SysState *state;          // 2 * nsys
  double *acc;              // BA_NSLOT * nsys
  int method, precond, kmax;
  int exit_on_done;         // end the launch after an iteration in which a system finished
  double tol;
  int maxit;
  int tri_warps_per_block;
  int tri_group;            // rows per warp in the sync-free solves (1, 2, 4 or 8)
  int spw;                  // SELL slices (of 32 rows) a warp sums at once in the SpMV phases (1 or 2)
  int sweeps;               // BiCGStab + ILU0: Jacobi sweeps per triangle (0: sync-free exact solves)
  unsigned int *bar;
  int *err;
  int *it_done;             // iterations run by this launch (written by block 0)
};

struct BatchShared {
  int act[BATCH_MAX_SYS];        // systems with work this iteration
  unsigned char fresh[BATCH_MAX_SYS];  // 1: this inner solve started from zero, 0: resumed
  int pre[BATCH_MAX_SYS + 1];    // prefix of their slice counts
  int status[BATCH_MAX_SYS];     // status decided for this iteration
  int kk[BATCH_MAX_SYS];
  float sa[BATCH_MAX_SYS], sb[BATCH_MAX_SYS];  // per-phase scalars (beta, alpha, omega)
  double red[BATCH_MAX_SYS * 4];               // per-block per-system accumulators (4 each)
  int nact, total;
  int any_done;                  // a system finished at this iteration's top
};

__device__ __forceinline__ void batch_acc_add(BatchShared &sh, int s_local, int v, double x) {
  atomicAdd(&sh.red[4 * s_local + v], x);
}

}  // namespace egpu
