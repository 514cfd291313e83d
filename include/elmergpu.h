/*
 * elmergpu.h -- C ABI of the B200 linear-system path for ElmerSolver.
 *
 * Drop-in seam: the library replaces IterSolver (fem/src/IterSolve.src:144-798) for
 *   Linear System Solver = Iterative
 *   Linear System Iterative Method = BiCGStab | CG
 *   Linear System Preconditioning  = ILU0 | Diagonal | None
 * and the bulk assembly loop of HeatSolve/StressSolve (modules/HeatSolve.src:655-985,
 * modules/StressSolve.src:815-1072) for linear Poisson and isotropic elasticity.
 *
 * Every pointer argument is a plain host pointer unless the name ends in _dev (device
 * memory on the context's GPU).  CRS arrays use Elmer's Matrix_t convention
 * (fem/src/Types.src:155-228): Rows(n+1), Cols(nnz), Diag(n), 1-based int32; Values
 * double.  The library copies what it needs, never frees or keeps caller memory, and
 * writes only the output arrays named in each call.
 *
 * Return values: >0 is a HUTI status (hutiter/src/huti_fdefs.h:18-52; 1 = converged);
 * 0 is success for calls that do not iterate; <0 is a library error (EGPU_ERR_*).
 * No exception crosses the ABI.  A context is used by one host thread at a time.
 */
#ifndef ELMERGPU_H
#define ELMERGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------- */
#define EGPU_OK 0
#define EGPU_ERR_ARG (-1)      /* invalid argument */
#define EGPU_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define EGPU_ERR_ALLOC (-3)    /* device allocation failed */
#define EGPU_ERR_TIMEOUT (-4)  /* a bounded device-side wait expired (kernel returned) */
#define EGPU_ERR_STATE (-5)    /* call out of order (e.g. solve before values exist) */
#define EGPU_ERR_BUDGET (-6)   /* admission refused: footprint exceeds the HBM budget */
#define EGPU_ERR_ABORT (-7)    /* the host raised the context's abort word (egpu_abort) */

/* HUTI status values returned by the solve calls (huti_fdefs.h:18-52) */
#define EGPU_HUTI_CONVERGENCE 1
#define EGPU_HUTI_MAXITER 2
#define EGPU_HUTI_DIVERGENCE 3
#define EGPU_HUTI_CG_RHO 20
#define EGPU_HUTI_BICGSTAB_RHO 35
#define EGPU_HUTI_BICGSTAB_SNORM 36
#define EGPU_HUTI_BICGSTAB_OMEGA 37

/* ---- keyword surface (IterSolve.src:221-420) ------------------------------------ */
enum { EGPU_CG = 1, EGPU_BICGSTAB = 2, EGPU_GCR = 3, EGPU_BICGSTABL = 4 }; /* Linear System Iterative Method */
/* Linear System Preconditioning: None, Diagonal, ILU0 / ILUn (with ilu_order), ILUT (with
 * ilut_tol; IterSolve.src:384-388, CRS_ILUT CRSMatrix.src:2849-3044) */
enum { EGPU_PREC_NONE = 0, EGPU_PREC_DIAGONAL = 1, EGPU_PREC_ILU0 = 2, EGPU_PREC_ILUT = 3 };
enum { EGPU_FP64 = 0, EGPU_MIXED = 1 };  /* FP64 drop-in | FP32 inner Krylov in FP64 refinement */

typedef struct {
  int method;             /* EGPU_CG | EGPU_BICGSTAB | EGPU_GCR | EGPU_BICGSTABL */
  int precond;            /* EGPU_PREC_* */
  int max_iter;           /* Linear System Max Iterations (required, >= 1) */
  double tol;             /* Linear System Convergence Tolerance (true residual / ||b||) */
  int scale_system;       /* Linear System Scaling (Elmer default 1) */
  int precision;          /* EGPU_FP64 | EGPU_MIXED */
  int refactorize;        /* Linear System Refactorize (Elmer default 1) */
  int precond_recompute;  /* Linear System Precondition Recompute (Elmer default 1) */
  /* mixed precision only */
  double inner_tol;       /* relative reduction of the FP32 inner residual per segment
                             (each segment continues the previous one's recurrences from the
                             FP64 true residual); 0 (the default): 1e-2 with Diagonal / none,
                             3e-2 with ILU0 */
  int inner_max_iter;     /* cap on inner iterations per refinement */
  int max_refinements;    /* cap on FP64 refinement steps */
  /* with EGPU_PREC_ILU0: fill order n of ILU(n) (Linear System Preconditioning = ILUn /
   * Linear System ILU Order, IterSolve.src:420-575); 0 = ILU0 (the default), at most 9 */
  int ilu_order;
  /* EGPU_GCR: Linear System GCR Restart (0: Max Iterations, IterSolve.src:298-304);
   * EGPU_BICGSTABL: BiCGstabl polynomial degree (0: 2, :306-310).  Both run in FP64 whatever
   * the precision, stopping on the recursive residual as the reference's internal methods do. */
  int restart;
  /* EGPU_PREC_ILUT: Linear System ILUT Tolerance (0 when absent, as in the reference: no entry
   * dropped).  Entries with |ILU(i,j)| < tol * ||A(i,:)||_2 are dropped after the row's full
   * elimination.  The factor's structure depends on the values, so it is computed on the host
   * (as the reference does) and applied on the device; not available to cloned matrices
   * (batches, the server). */
  double ilut_tol;
  /* Linear System Divergence Tolerance (IterSolve.src:364-366; 0 when absent: no bound, as the
   * reference's HUGE).  EGPU_GCR and EGPU_BICGSTABL stop with HUTI_DIVERGENCE (3) when the
   * residual ratio exceeds it (IterativeMethods.src:626-629, 817-819, 959-961, 1047-1048);
   * HUTI's CG and BiCGStab do not read it, as in the reference. */
  double divtol;
  /* mixed precision, BiCGStab + ILU0 (order 0): the FP32 inner solves apply the factors by
   * this many Jacobi sweeps per triangle (y <- v - L y, z <- D^-1 (y - U z)) instead of
   * exact triangular solves, trading the solves' dependency levels (latency-bound) for
   * parallel passes over the factors; the FP64 refinement still stops on the true residual.
   * 0: exact solves; < 0 (egpu_params_default): the library measures exact solves against
   * two sweeps on the matrix and keeps the faster (see egpu_result.precision_used).  The
   * FP64 drop-in always solves exactly, as CRS_LUSolve. */
  int ilu_sweeps;
} egpu_params;

typedef struct {
  int info;               /* HUTI status */
  int iters;              /* HUTI_ITERS (FP64) / total inner iterations (mixed) */
  int refinements;        /* FP64 refinement steps (mixed); 0 for FP64 */
  double residual;        /* last ||A x - b|| / ||b|| of the scaled system */
  double seconds;         /* device time of the solve, CUDA events */
  double seconds_setup;   /* scaling + preconditioner construction part of seconds */
  double seconds_krylov;  /* device time inside the persistent Krylov kernels */
  int krylov_launches;    /* number of persistent Krylov kernel launches */
  /* the path that ran: EGPU_FP64, or EGPU_MIXED.  A CG / BiCGStab mixed request is a request
   * for the fastest path at the same tolerance.  The candidates: the mixed solve as asked,
   * with ilu_sweeps < 0 (BiCGStab + ILU0) also the mixed solve with two Jacobi sweeps, and the
   * FP64 drop-in.  On each matrix the first solve is not timed (one-time set-up), then every
   * candidate not yet timed runs once (the caller's own FP64 solves count), and after that a
   * mixed request takes the fastest mixed candidate, or the FP64 drop-in when its latest time
   * is below 0.85 of that one.  The times outlive value updates.  EGPU_MIXED_AUTO=0 keeps the
   * mixed solve as asked. */
  int precision_used;
  int ilu_sweeps_used;    /* Jacobi sweeps per triangle of the mixed solve that ran (0: exact) */
} egpu_result;

/* fills p with Elmer's defaults for the given method/preconditioner */
void egpu_params_default(egpu_params *p, int method, int precond);

/* ---- context --------------------------------------------------------------------- */
typedef struct egpu_ctx egpu_ctx;
typedef struct egpu_mat egpu_mat;

int egpu_create(int device, egpu_ctx **out);
void egpu_destroy(egpu_ctx *ctx);
const char *egpu_last_error(const egpu_ctx *ctx);
/* number of this library's kernel launches since the context was created */
long long egpu_kernel_launches(const egpu_ctx *ctx);
/* the cudaStream_t every call of this context runs on (for callers' CUDA events) */
void *egpu_stream(const egpu_ctx *ctx);
/* Failure detection, no counterpart in the reference (whose IterSolver has only its status
 * exits, IterSolve.src:784-792).  Every device-side wait of this context's kernels (grid
 * barriers, sync-free dependency waits, factorisation flags) is bounded: after `seconds`
 * (0: the default of 2 s) the kernel records EGPU_ERR_TIMEOUT, unwinds and the call returns
 * it; the context stays usable. */
int egpu_set_wait_limit(egpu_ctx *ctx, double seconds);
/* Cancellation: raise != 0 sets the context's host-mapped abort word, which the running
 * kernels poll (block 0 every 256th grid barrier, block 1 during long barrier waits); the call in flight
 * and every later call return EGPU_ERR_ABORT until egpu_abort(ctx, 0).  Makes no CUDA call
 * and may be called from any host thread while a solve runs. */
int egpu_abort(egpu_ctx *ctx, int raise);
/* Self-test of the bounded waits: which = 0 launches two blocks of which one never arrives at
 * the grid barrier; which = 1 waits for a value that nothing publishes.  Returns the status
 * the kernel recorded: EGPU_ERR_TIMEOUT once the wait bound has passed (EGPU_ERR_ABORT if the
 * abort word is raised). */
int egpu_wait_selftest(egpu_ctx *ctx, int which);
/* Device blocks freed by the library (matrix copies, work vectors, factors) stay in a
 * process-wide cache per device, at most 24 GB each, for the next matrix of a similar size.
 * egpu_cached_bytes: bytes held for `device` (all devices if device < 0).
 * egpu_release_cached_memory: synchronises and frees them (all devices if device < 0);
 * returns the bytes given back to the driver. */
long long egpu_cached_bytes(int device);
long long egpu_release_cached_memory(int device);

/* ---- sparsity pattern: CreateMatrix (ElementUtils.src:698-930) -------------------
 * MakeListMatrix + OptimizeBandwidth (BandwidthOptimize.src:108-355) +
 * CRS_CreateMatrix/InitializeMatrix/CRS_SortMatrix for a mesh whose nodes are all
 * active.  Two calls: first with rows/cols/diag == NULL to get n and nnz, then with
 * buffers of those sizes.  perm (nnodes) receives Elmer's Perm (node -> row block). */
int egpu_pattern_create(int nnodes, int nelem, int nen, const int *elem_nodes, int dofs,
                        int optimize_bw, int *n_out, long long *nnz_out, int *perm,
                        int *rows, int *cols, int *diag);

/* ---- matrix binding (replaces the Matrix_t handed to IterSolver) ----------------- */
int egpu_matrix_bind(egpu_ctx *ctx, int n, const int *rows, const int *cols, const int *diag,
                     const double *values, egpu_mat **out);
/* same pattern, new Values (nonlinear / time steps) */
int egpu_matrix_update_values(egpu_mat *A, const double *values);
int egpu_matrix_values_download(egpu_mat *A, double *values);
int egpu_matrix_rhs_download(egpu_mat *A, double *rhs);
void egpu_matrix_free(egpu_mat *A);
/* No counterpart in the reference's C interface (Elmer reuses Solver % Matrix across steps):
 * a matrix sharing proto's pattern, SELL layout, level orders and bound mesh (read-only)
 * with its own Values, right-hand side and solve buffers.  proto may be freed before its
 * clones; the shared data goes with the last of them. */
int egpu_matrix_clone(egpu_mat *proto, egpu_mat **out);
/* Builds the preconditioner's one-time structures before the first solve (for ILU(n) the
 * fill structure and the level schedules of the triangular solves; nothing for Diagonal /
 * None), so that the first IterSolver call on a pattern costs what later ones do.  Clones
 * share their prototype's. */
int egpu_matrix_prepare(egpu_mat *A, const egpu_params *prm);
/* device bytes a solve of A holds beyond the shared pattern, for the given preconditioner */
long long egpu_matrix_footprint(const egpu_mat *A, int precond);

/* ---- IterSolver replacement (SolveLinearSystem semantics, SolverUtils.src:7151-7525):
 * zero-rhs short cut, symmetric scaling, x = 1e-8 when x is all zero, ILU0 factored on
 * the scaled matrix, HUTI true-residual stopping test, back-scaling.  b, x host. */
int egpu_iter_solve(egpu_mat *A, const double *b, double *x, const egpu_params *prm,
                    egpu_result *res);
/* same with b_dev, x_dev in device memory; b_dev == NULL uses the assembled RHS */
int egpu_iter_solve_dev(egpu_mat *A, const double *b_dev, double *x_dev, const egpu_params *prm,
                        egpu_result *res);

/* ---- preconditioner state (Matrix_t ILUValues, CRSMatrix.src:2157-2388, 3259-3270) ----
 * egpu_ilu0_build factors ILU0 of the matrix (scaled as SolveLinearSystem scales it when
 * scale_system != 0) on the device; egpu_ilu0_download copies the factors (same layout as
 * Values, inverted U diagonal) and the DiagScaling vector (NULL to skip);
 * egpu_lu_precondition applies u = (LU)^-1 v with the device factors (pcondProc). */
int egpu_ilu0_build(egpu_mat *A, int scale_system);
/* the same for ILU(order), order 0..9 (CRS_IncompleteLU(A, order)) */
int egpu_ilu_build(egpu_mat *A, int scale_system, int order);
/* ILU(n) structure of a Matrix_t pattern (CRS_IncompleteLU(A, n), CRSMatrix.src:2196-2218:
 * InitializeILU1 applied n times), host only, index base as given.  Returns the number of
 * entries; ilu_rows (n+1), ilu_cols and ilu_diag (n) are written when cap >= it. */
long long egpu_ilu_pattern(int n, const int *rows, const int *cols, const int *diag, int order, long long cap,
                           int *ilu_rows, int *ilu_cols, int *ilu_diag);
/* threshold ILU (CRS_ILUT, CRSMatrix.src:2849-3044) of the (optionally scaled) matrix: host
 * factorisation, device schedules and packed factors as for ILU(n); egpu_ilu_download reads
 * the result */
int egpu_ilut_build(egpu_mat *A, int scale_system, double tol);
/* the matrix's current ILU factors on their structure (1-based, as egpu_ilu_pattern
 * returns it), inverted U diagonal; NULL arrays are skipped.  Returns the number of entries. */
int egpu_ilu_download(egpu_mat *A, int *ilu_rows, int *ilu_cols, int *ilu_diag, double *ilu_values);
int egpu_ilu0_download(egpu_mat *A, double *ilu_values, double *diag_scaling);
int egpu_lu_precondition(egpu_mat *A, const double *v, double *u);
/* the same on device vectors (v_dev != u_dev), on the context's stream; returns when applied.
 * ParLUPrec (SParIterPrecond.src:86-146) of a rank's block in the row-sharded solve */
int egpu_lu_precondition_dev(egpu_mat *A, const double *v_dev, double *u_dev);
/* The triangular-solve schedule built for the matrix's ILU structure (diagnostics): info[0]
 * rows per sync-free slot group (> 1: node-block solve), [1] / [2] lower / upper dependency
 * levels (of slot groups), [3] most rows in one level, [4] / [5] single-block schedule usable
 * for FP64 / FP32.  EGPU_ERR_STATE before the first factorisation.  No reference
 * counterpart (the reference's CRS_LUSolve has no schedule). */
int egpu_tri_info(egpu_mat *A, int info[6]);

/* ---- Matrix Vector Proc hook (CRSMatrix.src:3555-3559, Load.c:734-747) ----------- */
int egpu_mv(egpu_mat *A, const double *u, double *v);
int egpu_mv_dev(egpu_mat *A, const double *u_dev, double *v_dev);
/* exact MatVecSubr signature; *spmv is the per-matrix handle slot A%SpMV; the
 * matrix is (re)uploaded when *reinit != 0 or *spmv == NULL.  The signature has no status:
 * when the product cannot be formed (no device, rejected arrays) v is filled with NaN. */
void egpu_matvec_subr(void **spmv, int *n, int *rows, int *cols, double *values, double *u,
                      double *v, int *reinit);

/* ---- assembly seam (HeatSolve / StressSolve bulk loops) --------------------------
 * Binds the mesh to the matrix pattern: coords (nnodes x 3, row-major), element
 * connectivity (nelem x nen, 1-based), element code (808 | 504 | 303), Perm.
 * Builds the element colouring and the element -> CRS slot map on the device. */
int egpu_assembly_bind(egpu_mat *A, int nnodes, const double *xyz, int cdim, int nelem,
                       int code, const int *elem_nodes, const int *perm, int dofs);
/* DiffuseConvectiveCompose diffusion branch: conductivity per element (elem_k, nelem)
 * or per node (nodal_k, nnodes) or 1; nodal heat source*density (load, nnodes) or 0.
 * Zeroes and fills Values and the RHS on the device. */
int egpu_assemble_poisson(egpu_mat *A, const double *elem_k, const double *nodal_k,
                          const double *load);
/* StressCompose, isotropic 3D (dofs = 3) with a constant body force */
int egpu_assemble_elastic(egpu_mat *A, double young, double poisson, const double *body_force3);
/* DefaultDirichletBCs: con_rows 1-based matrix rows, con_vals values (NULL = 0),
 * symmetric = Linear System Symmetric (CRS_SetSymmDirichlet) */
int egpu_dirichlet(egpu_mat *A, int ncon, const int *con_rows, const double *con_vals,
                   int symmetric);

/* ---- allocation-free CG ------------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot let the library allocate
 * device memory: code whose device memory belongs to another runtime (CUDA Fortran or
 * OpenACC data regions around Elmer's arrays) and code that cannot afford the implicit
 * synchronisation of cudaMalloc inside its loop.  Solves like egpu_iter_solve_dev with
 * method CG, preconditioner Diagonal or None and system scaling on, taking the caller's
 * Matrix_t arrays (1-based Rows/Cols/Diag, Values) and b, x in device memory; x is the
 * initial guess on entry.  All scratch is one fixed device array inside the library
 * (about 2.4 MB, held by every GPU that loads the library until the process exits), so:
 * n is limited to EGPU_NOALLOC_MAX_ROWS (larger n returns EGPU_ERR_ARG); calls that
 * overlap on the GPU race on that array; the first call on a device looks up the array's
 * device address and should come before any stream capture.  That address is kept for the
 * life of the process: after cudaDeviceReset on the device this entry point must not be
 * called again.  The Matrix_t arrays are checked on the device before use (Rows(1) = 1 and
 * non-decreasing, Cols in 1..n, Diag 0 or the row's own diagonal entry); a violation returns
 * EGPU_ERR_ARG.  Runs on the legacy default stream, returns when the solve has finished and
 * leaves the caller's current device as it found it. */
#define EGPU_NOALLOC_MAX_ROWS 32768
int egpu_cg_noalloc(int device, int n, const int *rows_dev, const int *cols_dev, const int *diag_dev,
                    const double *values_dev, const double *b_dev, double *x_dev, const egpu_params *prm,
                    egpu_result *res);

/* ---- batched / continuous-batching solve (no counterpart in the reference; extends
 * SolveSystem to many independent systems).  Every system is scaled and preconditioned
 * like egpu_iter_solve and solved in mixed precision (FP32 inner Krylov, FP64 iterative
 * refinement to prm->tol on the true residual); all resident systems share one persistent
 * launch per chunk of inner iterations, with per-system convergence masks.
 *   egpu_batch_create   parameters are fixed for the batch (method, preconditioner, tol...)
 *   egpu_batch_add      host Matrix_t arrays + rhs; the batch owns the device copy
 *   egpu_batch_add_matrix  a bound/assembled matrix (b_dev NULL: its assembled rhs); borrowed
 *   egpu_batch_step     one refinement check + one chunk; lists the systems that finished
 *   egpu_batch_solve    steps until every resident system has finished.  With CG and no
 *                       preconditioner or Diagonal, when no system is inside an inner solve,
 *                       it runs every system's whole solve in one cooperative launch instead:
 *                       each system on a team of CTAs of its own (one CTA when small), with
 *                       team barriers, no grid barrier and no host round trip between
 *                       refinements (EGPU_BATCH_TEAMS=0 keeps the stepwise path)
 *   egpu_batch_last_launch  device milliseconds of the latest batched launch (the team
 *                       solver's one launch, or the latest chunk of egpu_batch_step)
 *   egpu_batch_remove   frees a finished system's slot
 * Returns the slot id (>= 0) from the add calls, EGPU_ERR_BUDGET when all slots are used. */
typedef struct egpu_batch egpu_batch;
int egpu_batch_create(egpu_ctx *ctx, const egpu_params *prm, egpu_batch **out);
int egpu_batch_add(egpu_batch *B, int n, const int *rows, const int *cols, const int *diag,
                   const double *values, const double *rhs);
int egpu_batch_add_matrix(egpu_batch *B, egpu_mat *A, const double *b_dev);
int egpu_batch_set_chunk(egpu_batch *B, int chunk_iters);
/* on != 0: a launch returns as soon as some system finishes its inner segment, so that system
 * is refined or retired at once (lower latency for short requests, more launches) */
int egpu_batch_set_latency_mode(egpu_batch *B, int on);
int egpu_batch_step(egpu_batch *B, int *finished, int *nfinished);
int egpu_batch_pending(egpu_batch *B);
int egpu_batch_solve(egpu_batch *B, egpu_result *per_system);
int egpu_batch_last_launch(egpu_batch *B, double *ms);
int egpu_batch_result(egpu_batch *B, int sys, egpu_result *res);
int egpu_batch_solution(egpu_batch *B, int sys, double *x);
int egpu_batch_remove(egpu_batch *B, int sys);
/* Autotuner: runs real steps of the resident systems with each candidate configuration
 * (inner iterations per launch, persistent-kernel blocks per SM, rows per warp in the SpMV
 * phases, sync-free triangular-solve participants) and keeps the fastest by nonzeros x
 * iterations per device second.  Systems that finish while tuning are listed by the next
 * egpu_batch_step. */
typedef struct {
  int chunk_iters, blocks_per_sm, tri_mult, candidates;
  double rate;  /* nonzeros x inner iterations per second of the kept configuration */
  int slices_per_warp;  /* rows per warp in the SpMV phases: 1 or 2 SELL slices of 32 rows (0 in
                           egpu_batch_set_config: keep) */
} egpu_batch_config;
int egpu_batch_tune(egpu_batch *B, egpu_batch_config *cfg);
/* applies a configuration (e.g. one egpu_batch_tune chose for an earlier batch of the same kind) */
int egpu_batch_set_config(egpu_batch *B, const egpu_batch_config *cfg);
void egpu_batch_free(egpu_batch *B);

/* ---- solve server (no counterpart in the reference; the serving extension of SolveSystem,
 * SolverUtils.src:7531, for a stream of independent systems).  The server owns its own
 * context and a batch, and runs a host worker thread: it admits submitted requests in
 * arrival order while their device footprint fits hbm_budget_bytes and a batch slot is free
 * (at most max_resident at once; one request larger than the budget runs alone), prepares
 * them (clone of the registered pattern's resident prototype; Values and RHS from the
 * request, or GPU assembly + Dirichlet rows), steps the batch (egpu_batch_step: mixed
 * precision, prm's method / preconditioner / tolerance) and retires converged systems.
 * Every entry point may be called from any thread.
 *   egpu_server_pattern       registers a Matrix_t pattern (1-based Rows/Cols/Diag); once per mesh
 *   egpu_server_pattern_mesh  binds the mesh to a pattern (as egpu_assembly_bind) for
 *                             egpu_server_submit_poisson
 *   egpu_server_submit        Values (nnz) and RHS (n) from the host, copied at the call
 *   egpu_server_submit_poisson  per-element / per-node conductivity, nodal load (NULL: as in
 *                             egpu_assemble_poisson), 1-based Dirichlet rows set to zero
 *   egpu_server_poll          1 and the solution (x, n values; NULL to skip) and result when
 *                             the request has finished, releasing it; 0 while it has not
 *   egpu_server_wait          egpu_server_poll blocking up to timeout_s (EGPU_ERR_TIMEOUT)
 * A finished request's res.seconds is its latency from submission to completion and
 * res.seconds_setup its time in the queue; res.info is its HUTI status, or a negative
 * library error when its preparation or the batch failed. */
typedef struct egpu_server egpu_server;
typedef struct {
  long long queued, resident, done, steps;
  double used_bytes;
  /* worker thread's wall time so far: preparing admitted requests (clone, device assembly,
   * scaling, factorisation), batch steps, retiring finished requests (results, solution
   * copies, device memory returned) */
  double seconds_prepare, seconds_step, seconds_retire;
  /* kernel launches of the server's context so far; request inputs copied host -> device
   * (Values, RHS, conductivities, loads, Dirichlet rows) and solutions device -> host, bytes */
  long long kernel_launches;
  double bytes_h2d, bytes_d2h;
  /* admitted requests put back in the queue because a device allocation failed while others
   * were resident (each is prepared again when admitted again) */
  long long requeues;
} egpu_server_stats;
int egpu_server_create(int device, const egpu_params *prm, double hbm_budget_bytes, int chunk_iters,
                       int max_resident, egpu_server **out);
int egpu_server_pattern(egpu_server *S, int n, const int *rows, const int *cols, const int *diag, int *pattern);
int egpu_server_pattern_mesh(egpu_server *S, int pattern, int nnodes, const double *xyz, int cdim, int nelem,
                             int code, const int *elem_nodes, const int *perm, int dofs);
int egpu_server_submit(egpu_server *S, int pattern, const double *values, const double *rhs, long long *request);
int egpu_server_submit_poisson(egpu_server *S, int pattern, const double *elem_k, const double *nodal_k,
                               const double *load, int ncon, const int *con_rows, int symmetric,
                               long long *request);
int egpu_server_poll(egpu_server *S, long long request, double *x, egpu_result *res);
int egpu_server_wait(egpu_server *S, long long request, double timeout_s, double *x, egpu_result *res);
int egpu_server_info(egpu_server *S, egpu_server_stats *st);
void egpu_server_free(egpu_server *S);

#ifdef __cplusplus
}
#endif
#endif /* ELMERGPU_H */
