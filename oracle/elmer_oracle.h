/*
 * elmer_oracle.h -- CPU restatement of ElmerSolver's linear-system path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the GPU library
 * (elmerfem_b200/libelmergpu.so): it is linked by the tests, by smoke() and by
 * the CPU-baseline leg of bench.py, never by the product.  Each function restates
 * the Fortran routine cited beside it, in the same operation order, with
 * floating-point contraction disabled (-ffp-contract=off).
 *
 * Conventions follow Elmer's Matrix_t (fem/src/Types.src:155-228): Rows(n+1),
 * Cols(nnz), Diag(n) are 1-based int32; Values are double.
 */
#ifndef ELMER_ORACLE_H
#define ELMER_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- sparsity pattern: MakeListMatrix + OptimizeBandwidth + CRS_CreateMatrix/InitializeMatrix */
typedef struct orc_pattern orc_pattern;

orc_pattern *orc_pattern_create(int nnodes, int nelem, int nen, const int *elem_nodes,
                                int dofs, int optimize_bw, int use_optimized_always);
void orc_pattern_info(const orc_pattern *p, int *n, long long *nnz, int *hbw_before,
                      int *hbw_after, int *start_node, int *rejected);
void orc_pattern_copy(const orc_pattern *p, int *perm, int *rows, int *cols, int *diag);
void orc_pattern_free(orc_pattern *p);

/* ---- element assembly (HeatSolve / StressSolve bulk loops) */
/* elem_k: per-element conductivity (nelem) or NULL for nodal_k; nodal_k: per-node
 * conductivity or NULL (then k=1); load: per-node heat source * density (or NULL = 0). */
void orc_assemble_poisson(int nnodes, const double *xyz, int cdim, int nelem, int code,
                          const int *elem_nodes, const double *elem_k, const double *nodal_k,
                          const double *load, const int *perm, int n, const int *rows,
                          const int *cols, const int *diag, double *values, double *rhs);
void orc_assemble_elastic(int nnodes, const double *xyz, int nelem, int code,
                          const int *elem_nodes, double young, double poisson,
                          const double *body_force3, const int *perm, int n, const int *rows,
                          const int *cols, const int *diag, double *values, double *rhs);

/* ---- Dirichlet conditions (DefaultDirichletBCs): scale(no rhs) -> set rows -> backscale */
void orc_dirichlet(int n, const int *rows, const int *cols, const int *diag, double *values,
                   double *rhs, int ncon, const int *con_rows, const double *con_vals,
                   int symmetric, int scale);

/* ---- linear solve (SolveLinearSystem -> IterSolver -> HUTI) */
enum { ORC_CG = 1, ORC_BICGSTAB = 2, ORC_GCR = 3, ORC_BICGSTABL = 4 };
enum { ORC_PREC_NONE = 0, ORC_PREC_DIAGONAL = 1, ORC_PREC_ILU0 = 2, ORC_PREC_ILUT = 3 };
typedef struct {
  int method;          /* ORC_CG | ORC_BICGSTAB */
  int precond;         /* ORC_PREC_* */
  int max_iter;        /* Linear System Max Iterations */
  double tol;          /* Linear System Convergence Tolerance */
  int scale_system;    /* Linear System Scaling (default 1) */
  int omp_threads;     /* threads for the SpMV loop (CRSMatrix.src:3565), <=0: all */
  int ilu_order;       /* ORC_PREC_ILU0 with ilu_order n > 0: ILU(n) (Linear System ILU Order) */
  int restart;         /* GCR: Linear System GCR Restart (0: Max Iterations); BiCGStab(l): degree l */
  double ilut_tol;     /* ORC_PREC_ILUT: Linear System ILUT Tolerance (0 when absent, as ListGetCReal) */
  double divtol;       /* GCR / BiCGStab(l): Linear System Divergence Tolerance (<= 0: HUGE, as when absent) */
  int blas_threads;    /* threads for the vector operations: 0 serial (netlib BLAS, the checker's
                          setting), t > 0 t static chunks (a threaded BLAS; the timed baseline) */
  /* ORC_PREC_ILU0 with nblocks > 1: block-Jacobi ILU0 of a row partition (the parallel
   * preconditioner, ParILU0 SParIterPrecond.src:234-301, which factors each partition's
   * InsideMatrix): rows [block_starts[k], block_starts[k+1]) (0-based, nblocks + 1 entries)
   * form block k, and the factor is CRS_IncompleteLU of the matrix with every entry coupling
   * two blocks removed */
  const int *block_starts;
  int nblocks;
} orc_params;
typedef struct {
  int info;            /* HUTI status code (huti_fdefs.h) */
  int iters;
  double residual;     /* last ||Ax-b||/||b|| on the scaled system */
  double seconds_solve;/* scale + IterSolver + backscale */
  double seconds_precond_setup;
} orc_result;

/* values/b are not modified (the routine works on copies, as the reference's
 * scaling and back-scaling leave A and b restored). x: in = initial guess, out = solution. */
int orc_solve(int n, const int *rows, const int *cols, const int *diag, const double *values,
              const double *b, double *x, const orc_params *prm, orc_result *res);

/* ---- primitives for unit parity */
void orc_spmv(int n, const int *rows, const int *cols, const double *values, const double *u,
              double *v, int omp_threads);
void orc_ilu0(int n, const int *rows, const int *cols, const int *diag, const double *values,
              double *ilu_values);
void orc_lusolve(int n, const int *rows, const int *cols, const int *diag,
                 const double *ilu_values, double *b);
/* ILU(n) structure: InitializeILU1 (CRSMatrix.src:2391-2497) applied n times to the matrix
 * pattern (CRS_IncompleteLU :2196-2218).  1-based arrays.  Returns the number of entries;
 * the arrays are written when cap >= that number. */
long long orc_ilu_pattern(int n, const int *rows, const int *cols, const int *diag, int order, long long cap,
                          int *ilu_rows, int *ilu_cols, int *ilu_diag);
/* CRS_IncompleteLU LU branch (:2312-2366) on the ILU(n) structure: the matrix values
 * (rows/cols/values) enter the dense row, the structure's flags decide which entries are
 * kept; inverted U diagonal (:2359-2366). */
void orc_iluk(int n, const int *rows, const int *cols, const double *values, const int *ilu_rows,
              const int *ilu_cols, const int *ilu_diag, double *ilu_values);
/* CRS_ILUT (CRSMatrix.src:2849-3044): threshold ILU with the drop test
 * |ILU(i,j)| >= tol * ||A(i,:)||_2 after the row's full elimination; inverted U diagonal.
 * 1-based output, written when cap >= the returned entry count; -1 if a row has no diagonal. */
long long orc_ilut(int n, const int *rows, const int *cols, const double *values, double tol, long long cap,
                   int *ilu_rows, int *ilu_cols, int *ilu_diag, double *ilu_values);
void orc_scale(int n, const int *rows, const int *cols, const int *diag, double *values,
               double *b, double *x, double *diag_scaling, double *rhs_scaling, int rhs_scale);
double orc_compute_norm(int n, const double *x);
/* dependency levels of the lower-triangular part (row i after every j<i with a_ij != 0) */
int orc_lower_levels(int n, const int *rows, const int *cols, const int *diag, int *level);

#ifdef __cplusplus
}
#endif
#endif
