/* Test infrastructure (oracle): LAPACK-style Householder least squares. */
#ifndef APC_ORACLE_LSQ_HOUSEHOLDER_H
#define APC_ORACLE_LSQ_HOUSEHOLDER_H
#ifdef __cplusplus
extern "C" {
#endif

/* Row-major dgels('N') for m >= n.  On return B's first n rows hold the
 * least-squares solution.  Returns 0, or k > 0 when R(k,k) == 0 (LAPACK info). */
int oracle_dgels_rowmajor(int m, int n, int nrhs, double *A, int lda, double *B, int ldb);

#ifdef __cplusplus
}
#endif
#endif
