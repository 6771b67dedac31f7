/* Test infrastructure (oracle): PETSc-3.5-semantics restarted GMRES + Jacobi. */
#ifndef APC_ORACLE_GMRES_PETSC_H
#define APC_ORACLE_GMRES_PETSC_H
#ifdef __cplusplus
extern "C" {
#endif

/* PETSc KSPConvergedReason values */
enum {
  ORACLE_KSP_CONVERGED_RTOL = 2,
  ORACLE_KSP_CONVERGED_ATOL = 3,
  ORACLE_KSP_DIVERGED_NULL = -2,
  ORACLE_KSP_DIVERGED_ITS = -3,
  ORACLE_KSP_DIVERGED_DTOL = -4,
  ORACLE_KSP_DIVERGED_BREAKDOWN = -5,
  ORACLE_KSP_DIVERGED_NANORINF = -9
};

typedef struct oracle_gmres_params {
  int restart;   /* -ksp_gmres_restart */
  double rtol;   /* -ksp_rtol */
  double atol;   /* -ksp_atol */
  double dtol;   /* -ksp_divtol */
  int max_it;    /* -ksp_max_it */
  /* outputs */
  int its;
  double rnorm;
  int reason;
  /* host threads of the vector and matrix loops: <= 1 runs them serially, in the order
     the parity tests pin; more spread them over OpenMP threads as PETSc spreads them
     over MPI ranks (sums then depend on the thread count) */
  int threads;
} oracle_gmres_params;

void oracle_gmres_defaults(oracle_gmres_params *p);

/* Solve A x = b (CSR, columns sorted per row) with left-Jacobi GMRES(restart). */
int oracle_gmres_csr(int n, const int *rowptr, const int *col, const double *val,
                     const double *b, double *x, oracle_gmres_params *p);

#ifdef __cplusplus
}
#endif
#endif
