/*
 * Test infrastructure (oracle): stand-in for the one LAPACKE call the reference makes
 * (LAPACKE_dgels at solver.cpp:106 and solver.cpp:342), backed by the Householder
 * restatement in lsq_householder.c.  LAPACK 3.5.0 is not vendored in the reference.
 */
#ifndef APC_SHIM_LAPACKE_H
#define APC_SHIM_LAPACKE_H

#include "../lsq_householder.h"

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

static inline lapack_int LAPACKE_dgels(int layout, char trans, lapack_int m, lapack_int n,
                                       lapack_int nrhs, double *a, lapack_int lda, double *b,
                                       lapack_int ldb) {
  if (layout != LAPACK_ROW_MAJOR || trans != 'N') return -1;
  return oracle_dgels_rowmajor(m, n, nrhs, a, lda, b, ldb);
}

#endif
